// api.cu -- C ABI of the projection engine: plans, the reference-compatible
// setup()/showSetup()/gpuPrj() entry points, and error reporting.
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <algorithm>
#include <condition_variable>
#include <mutex>
#include <thread>
#include <vector>

#include <unistd.h>

#include "ctprj_internal.h"
#include "footprint.cuh"

namespace ctprj {

static thread_local char t_err[512] = "";

int set_error(int status, const char *fmt, ...)
{
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(t_err, sizeof t_err, fmt, ap);
    va_end(ap);
    return status;
}

int cuda_error(cudaError_t e, const char *what)
{
    if (e == cudaSuccess) return CTPRJ_OK;
    if (e == cudaErrorMemoryAllocation)
        return set_error(CTPRJ_ENOMEM, "%s: %s", what, cudaGetErrorString(e));
    return set_error(CTPRJ_ECUDA, "%s: %s", what, cudaGetErrorString(e));
}

// View angle of view i exactly as the reference forms it (prj/cpuPrj.c:342):
// ((float)(2 i) * pi_f) / (float)prjFull in float arithmetic.
double view_angle(int i, int P)
{
    volatile float th = (float)(2 * i) * kRefPiF;
    th = th / (float)P;
    return (double)th;
}

// View of symmetric image j for base view b: (q_j P/4 + s_j b) mod P, with
// (q, s) = (0,+)(1,+)(2,+)(3,+)(2,-)(3,-)(4,-)(1,-) (prj/cpuPrj.c:403-460,
// :117-157).
int view_of(int j, int b, int P)
{
    static const int q[8] = {0, 1, 2, 3, 2, 3, 4, 1};
    static const int sg[8] = {1, 1, 1, 1, -1, -1, -1, -1};
    int v = (q[j] * (P / 4) + sg[j] * b) % P;
    return v < 0 ? v + P : v;
}

int validate_geometry(const ctprj_geometry *g)
{
    if (!g) return set_error(CTPRJ_EINVAL, "geometry is NULL");
    if (g->n < 1 || g->prjWidth < 1 || g->np < 1)
        return set_error(CTPRJ_EINVAL, "n, prjWidth and np must be positive (n=%d prjWidth=%d np=%d)",
                         g->n, g->prjWidth, g->np);
    if (g->prjFull < 4 || g->prjFull % 4 != 0)
        return set_error(CTPRJ_EINVAL, "prjFull must be a positive multiple of 4 (prjFull=%d)",
                         g->prjFull);
    if (g->np > g->prjFull)
        return set_error(CTPRJ_EINVAL, "np (%d) exceeds prjFull (%d)", g->np, g->prjFull);
    if (!(g->dSize > 0.0f) || !std::isfinite(g->dSize))
        return set_error(CTPRJ_EINVAL, "dSize must be positive and finite");
    if (!(g->effectiveRate > 0.0f) || !std::isfinite(g->effectiveRate))
        return set_error(CTPRJ_EINVAL, "effectiveRate must be positive and finite");
    if (!std::isfinite(g->d)) return set_error(CTPRJ_EINVAL, "d must be finite");
    if ((long long)g->n * g->n >= (1LL << 31) || (long long)g->np * g->prjWidth >= (1LL << 31) ||
        (long long)g->prjFull * g->prjWidth >= (1LL << 31))
        return set_error(CTPRJ_ERANGE, "image or sinogram exceeds 2^31 elements");
    if (g->n > 65536 || g->prjWidth > 65536)
        return set_error(CTPRJ_ERANGE, "n and prjWidth are limited to 65536");
    return CTPRJ_OK;
}

Geo make_geo(const ctprj_geometry &gm)
{
    Geo g;
    g.n = gm.n;
    g.W = gm.prjWidth;
    g.np = gm.np;
    g.P = gm.prjFull;
    g.pC = gm.prjWidth / 2;
    g.half = (gm.n - 1) / 2;
    g.h2 = gm.n / 2;
    g.fan = gm.d > 0.0f;
    g.dSize = gm.dSize;
    g.beamWidth = (double)gm.dSize * (double)gm.effectiveRate;
    g.d = gm.d;
    g.beamWidthF = (float)g.beamWidth;
    g.dF = gm.d;
    g.invEr = 1.0f / gm.effectiveRate;
    g.effRate = gm.effectiveRate;
    return g;
}

// forward ray set (prj/cpuPrj.c:326-332, :469-475, :632-644): base views
// b <= prjFull/8, the first ray and the rays per base view
void fwd_ray_set(const Geo &g, int *nb, int *k0, int *nk)
{
    *nb = g.np < g.P / 8 + 1 ? g.np : g.P / 8 + 1;
    *k0 = (g.W % 2 == 0) ? 1 : 0;
    *nk = g.fan ? (g.W % 2 == 0 ? g.W - 1 : g.W) : (g.W % 2 == 0 ? g.W / 2 : (g.W + 1) / 2);
}

void fill_fwd_views(const Geo &g, int nb, FwdView *fv)
{
    for (int b = 0; b < nb; ++b) {
        const double th = view_angle(b, g.P);
        fv[b].c = cos(th);
        fv[b].s = sin(th);
        const bool mirror = b > 0 && (float)b < (float)g.P * 0.125f;
        for (int j = 0; j < 8; ++j) {
            const int v = view_of(j, b, g.P);
            fv[b].out[j] = ((j < 4 || mirror) && v < g.np) ? v : -1;
        }
    }
}

void fill_det_table(const Geo &g, DetEntry *de)
{
    for (int k = 0; k < g.W; ++k) {
        DetEntry &e = de[k];
        e.t = (double)(k - g.pC) * g.dSize;
        if (g.fan) {
            const double bq = sqrt(g.d * g.d + e.t * e.t);
            e.cB = g.d / bq;
            e.sB = e.t / bq;
            e.invbq = (float)(1.0 / bq);
        } else {
            e.cB = 1.0;
            e.sB = 0.0;
            e.invbq = 0.0f;
        }
        e.cBf = (float)e.cB;
        e.sBf = (float)e.sB;
        e.pad = 0;
    }
}

template <class T>
static int upload(T **dst, const std::vector<T> &src)
{
    int st = cuda_error(cudaMalloc((void **)dst, sizeof(T) * (src.empty() ? 1 : src.size())),
                        "table allocation");
    if (st) return st;
    if (!src.empty())
        st = cuda_error(cudaMemcpy(*dst, src.data(), sizeof(T) * src.size(), cudaMemcpyHostToDevice),
                        "table upload");
    return st;
}

static void free_plan(ctprj_plan *p)
{
    if (!p) return;
    cudaFree(p->d_fview);
    cudaFree(p->d_bview);
    cudaFree(p->d_det);
    cudaFree(p->d_quad);
    cudaFree(p->d_count);
    cudaFree(p->d_ramp);
    cudaFree(p->d_fsino);
    cudaFree(p->d_mimg);
    cudaFree(p->d_msino);
    delete p;
}

struct DeviceGuard {
    int prev = -1;
    bool changed = false;
    int status = CTPRJ_OK;
    explicit DeviceGuard(int dev)
    {
        if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
        if (dev >= 0 && dev != prev) {
            status = cuda_error(cudaSetDevice(dev), "cudaSetDevice");
            changed = status == CTPRJ_OK;
        }
    }
    ~DeviceGuard()
    {
        if (changed && prev >= 0) cudaSetDevice(prev);
    }
};

static int build_plan(const ctprj_geometry *geom, int device, ctprj_plan **out)
{
    int st = validate_geometry(geom);
    if (st) return st;
    ctprj_plan *p = new (std::nothrow) ctprj_plan();
    if (!p) return set_error(CTPRJ_ENOMEM, "host allocation failed");
    memset(p, 0, sizeof *p);
    p->geom = *geom;
    if (device < 0 && cudaGetDevice(&device) != cudaSuccess) device = 0;
    p->device = device;
    p->g = make_geo(*geom);
    const Geo &g = p->g;
    const int W = g.W, P = g.P, np = g.np;

    fwd_ray_set(g, &p->nb, &p->k0, &p->nk);
    p->nv = g.fan ? P : P / 2;

    std::vector<FwdView> fv(p->nb);
    fill_fwd_views(g, p->nb, fv.data());
    std::vector<BwdView> bv(p->nv);
    for (int i = 0; i < p->nv; ++i) {
        BwdView &e = bv[i];
        const double th = view_angle(i, P);
        e.c = cos(th);
        e.s = sin(th);
        e.cf = (float)e.c;
        e.sf = (float)e.s;
        const Footprint f = make_footprint(e.cf, e.sf);
        e.h = f.h; e.b1 = f.b1; e.b2 = f.b2; e.w = f.w; e.iw2 = f.iw2; e.pad = 0;
        e.cnt4 = e.cnt8 = 0;
        for (int j = 0; j < 8; ++j) {
            const int v = view_of(j, i, P);
            e.row[j] = v < np ? v * W : -1;
            int v2 = (v + P / 2) % P;
            e.row2[j] = (!g.fan && v2 < np) ? v2 * W : -1;
            const int reads = (e.row[j] >= 0) + (e.row2[j] >= 0);
            e.cnt8 += reads;
            if (j < 4) e.cnt4 += reads;
        }
    }
    std::vector<DetEntry> de(W);
    fill_det_table(g, de.data());

    DeviceGuard dg(device);
    if ((st = dg.status)) { delete p; return st; }
    if ((st = upload(&p->d_fview, fv)) || (st = upload(&p->d_bview, bv)) ||
        (st = upload(&p->d_det, de)) ||
        (st = cuda_error(cudaMalloc((void **)&p->d_quad, sizeof(float4) * quad_elems(g.n)),
                         "scratch allocation")) ||
        (st = cuda_error(cudaMalloc((void **)&p->d_count, sizeof(unsigned long long)),
                         "counter allocation"))) {
        free_plan(p);
        return st;
    }
    // backprojection kernel: staged tiles sized to the widest tile shadow of
    // this geometry, or the unstaged kernel when a shadow exceeds 64 detectors
    // or CTPRJ_BWD_KERNEL=direct asks for it (kept for comparison)
    int span = 0;
    if ((st = backward_max_span(p, &span))) {
        free_plan(p);
        return st;
    }
    const char *bk = getenv("CTPRJ_BWD_KERNEL");
    p->bwd_seg = span <= 32 ? 32 : (span <= 64 ? 64 : 0);
    if (bk && strcmp(bk, "direct") == 0) p->bwd_seg = 0;
    *out = p;
    return CTPRJ_OK;
}

}  // namespace ctprj

using namespace ctprj;

// ------------------------------------------------------------------ plan API

extern "C" int ctprj_plan_create(const ctprj_geometry *geom, int device, ctprj_plan **plan)
{
    if (!plan) return set_error(CTPRJ_EINVAL, "plan output pointer is NULL");
    *plan = nullptr;
    return build_plan(geom, device, plan);
}

extern "C" void ctprj_plan_destroy(ctprj_plan *plan)
{
    if (!plan) return;
    DeviceGuard dg(plan->device);
    free_plan(plan);
}

extern "C" int ctprj_forward(ctprj_plan *plan, const float *d_img, float *d_sino, void *stream)
{
    if (!plan || !d_img || !d_sino) return set_error(CTPRJ_EINVAL, "NULL plan or buffer");
    DeviceGuard dg(plan->device);
    if (dg.status) return dg.status;
    cudaStream_t s = (cudaStream_t)stream;
    int st = launch_quad(d_img, plan->d_quad, plan->g.n, s);
    if (st) return st;
    return launch_forward(plan, plan->d_quad, d_sino, nullptr, s);
}

extern "C" int ctprj_backward(ctprj_plan *plan, const float *d_sino, float *d_img, void *stream)
{
    if (!plan || !d_img || !d_sino) return set_error(CTPRJ_EINVAL, "NULL plan or buffer");
    DeviceGuard dg(plan->device);
    if (dg.status) return dg.status;
    return launch_backward(plan, d_sino, d_img, 0, nullptr, (cudaStream_t)stream);
}

extern "C" int ctprj_count_updates(ctprj_plan *plan, long long *fwd, long long *bwd, void *stream)
{
    if (!plan) return set_error(CTPRJ_EINVAL, "NULL plan");
    DeviceGuard dg(plan->device);
    if (dg.status) return dg.status;
    cudaStream_t s = (cudaStream_t)stream;
    unsigned long long h[2] = {0, 0};
    int st;
    for (int pass = 0; pass < 2; ++pass) {
        if ((st = cuda_error(cudaMemsetAsync(plan->d_count, 0, sizeof(unsigned long long), s),
                             "counter reset")))
            return st;
        st = pass == 0 ? launch_forward(plan, nullptr, nullptr, plan->d_count, s)
                       : launch_backward(plan, nullptr, nullptr, 0, plan->d_count, s);
        if (st) return st;
        if ((st = cuda_error(cudaMemcpyAsync(&h[pass], plan->d_count, sizeof(unsigned long long),
                                             cudaMemcpyDeviceToHost, s),
                             "counter readback")) ||
            (st = cuda_error(cudaStreamSynchronize(s), "counter sync")))
            return st;
    }
    if (fwd) *fwd = (long long)h[0];
    if (bwd) *bwd = (long long)h[1];
    return CTPRJ_OK;
}

extern "C" const char *ctprj_error_string(int status)
{
    switch (status) {
    case CTPRJ_OK: return "success";
    case CTPRJ_EINVAL: return "invalid argument";
    case CTPRJ_ENOTSETUP: return "setup() has not completed successfully";
    case CTPRJ_ENOMEM: return "out of memory";
    case CTPRJ_ECUDA: return "CUDA error";
    case CTPRJ_ERANGE: return "size out of range";
    case CTPRJ_ETIMEOUT: return "device wait timed out";
    default: return "unknown status";
    }
}

extern "C" const char *ctprj_last_error(void) { return t_err; }

// ----------------------------------------------- reference-compatible entry points

static std::mutex g_mu;
static struct prjConf g_conf;
extern "C" {
struct prjConf *pConf = &g_conf;
}
static ctprj_plan *g_plan = nullptr;
static float *g_dimg = nullptr, *g_dsino = nullptr;
// page-locked, mapped staging for pageable caller buffers (allocated on first
// use, as large as the larger of the image and the sinogram)
static float *g_stage = nullptr;
static size_t g_stage_bytes = 0;
static int g_status = CTPRJ_ENOTSETUP;
static char g_msg[512] = "setup() has not been called";

// prj/gpuPrj.cu:833-847: on a multi-GPU node the reference runs on the device
// with the most multiprocessors.  The environment variable CTPRJ_DEVICE, when
// set to a valid ordinal, selects the device instead (one process per GPU).
static int pick_device()
{
    int n = 0, best = 0, best_sm = -1;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n < 1) return -1;
    if (const char *env = getenv("CTPRJ_DEVICE")) {
        char *end = nullptr;
        long d = strtol(env, &end, 10);
        if (end != env && d >= 0 && d < n) return (int)d;
    }
    for (int d = 0; d < n; ++d) {
        int sm = 0;
        if (cudaDeviceGetAttribute(&sm, cudaDevAttrMultiProcessorCount, d) == cudaSuccess &&
            sm > best_sm) {
            best_sm = sm;
            best = d;
        }
    }
    return best;
}

static void release_global()
{
    if (g_plan) {
        DeviceGuard dg(g_plan->device);
        cudaFree(g_dimg);
        cudaFree(g_dsino);
        if (g_stage) cudaFreeHost(g_stage);
        free_plan(g_plan);
    }
    g_plan = nullptr;
    g_dimg = g_dsino = nullptr;
    g_stage = nullptr;
    g_stage_bytes = 0;
}

// Host copies of pageable caller buffers to and from the staging buffer, split
// over a few threads: one thread copies at about a quarter of what four reach
// (a driver-staged copy of pageable memory runs at about 20 GB/s, four host
// threads into page-locked memory at about 60).  The workers are started on
// first use and parked between copies; the calling thread takes a share.
class HostCopier {
public:
    static HostCopier &get()
    {
        static HostCopier c;
        return c;
    }
    // Copies `bytes` from src to dst, each thread (the workers and the caller)
    // its own contiguous share in pieces of at most `piece` bytes; after each
    // piece, sent(offset, length) when given (called from that thread; its
    // nonzero return is kept and returned).  The next job starts only when
    // each worker has reported this one.
    using Sent = int (*)(void *ctx, size_t offset, size_t length);
    int copy(void *dst, const void *src, size_t bytes, size_t piece = 0, Sent sent = nullptr,
             void *ctx = nullptr)
    {
        Job j = {(char *)dst, (const char *)src, bytes, workers_.size() + 1, piece ? piece : bytes, sent, ctx};
        // small copies, and a forked child (which has none of the parent's
        // workers), stay on the calling thread
        if (j.parts == 1 || bytes < (2u << 20) || getpid() != pid_) {
            j.parts = 1;
            return part(j, 0);
        }
        {
            std::lock_guard<std::mutex> lk(m_);
            job_ = j;
            done_ = 0;
            status_ = 0;
            ++gen_;
        }
        cv_.notify_all();
        const int mine = part(j, 0);
        std::unique_lock<std::mutex> lk(m_);
        done_cv_.wait(lk, [&] { return done_ == workers_.size(); });
        return mine ? mine : status_;
    }
    ~HostCopier()
    {
        {
            std::lock_guard<std::mutex> lk(m_);
            stop_ = true;
        }
        cv_.notify_all();
        for (auto &t : workers_) t.join();
    }

private:
    struct Job {
        char *dst;
        const char *src;
        size_t bytes, parts, piece;
        Sent sent;
        void *ctx;
    };
    HostCopier()
    {
        const unsigned hw = std::thread::hardware_concurrency();
        const unsigned n = hw >= 8 ? 3 : (hw >= 4 ? 1 : 0);   // plus the caller
        for (unsigned i = 0; i < n; ++i) workers_.emplace_back([this, i] { loop(i + 1); });
        pid_ = getpid();
    }
    static int part(const Job &j, size_t i)
    {
        const size_t a = j.bytes * i / j.parts, b = j.bytes * (i + 1) / j.parts;
        int st = 0;
        for (size_t o = a; o < b && !st; o += j.piece) {
            const size_t len = std::min(j.piece, b - o);
            memcpy(j.dst + o, j.src + o, len);
            if (j.sent) st = j.sent(j.ctx, o, len);
        }
        return st;
    }
    void loop(size_t idx)
    {
        unsigned seen = 0;
        for (;;) {
            Job j;
            {
                std::unique_lock<std::mutex> lk(m_);
                cv_.wait(lk, [&] { return stop_ || gen_ != seen; });
                if (stop_) return;
                seen = gen_;
                j = job_;
            }
            const int st = part(j, idx);
            {
                std::lock_guard<std::mutex> lk(m_);
                if (st && !status_) status_ = st;
                ++done_;
            }
            done_cv_.notify_one();
        }
    }
    std::vector<std::thread> workers_;
    std::mutex m_;
    std::condition_variable cv_, done_cv_;
    Job job_ = {nullptr, nullptr, 0, 1, 1, nullptr, nullptr};
    size_t done_ = 0;
    int status_ = 0;
    unsigned gen_ = 0;
    bool stop_ = false;
    pid_t pid_ = 0;
};

extern "C" void setup(int n, int prjWidth, int np, int prjFull, float dSize, float effectiveRate,
                      float d)
{
    std::lock_guard<std::mutex> lk(g_mu);
    g_conf.n = n;
    g_conf.prjWidth = prjWidth;
    g_conf.np = np;
    g_conf.prjFull = prjFull;
    g_conf.dSize = dSize;
    g_conf.effectiveRate = effectiveRate;
    g_conf.d = d;
    g_conf.cmd = 0;
    g_conf.imgSize = (unsigned)n * (unsigned)n;
    g_conf.sinoSize = (unsigned)prjWidth * (unsigned)np;
    release_global();
    ctprj_geometry gm = {n, prjWidth, np, prjFull, dSize, effectiveRate, d};
    int dev = pick_device();
    if (dev < 0) {
        g_status = set_error(CTPRJ_ECUDA, "no CUDA device");
    } else {
        g_status = build_plan(&gm, dev, &g_plan);
        if (g_status == CTPRJ_OK) {
            DeviceGuard dg(dev);
            g_status = cuda_error(cudaMalloc((void **)&g_dimg, sizeof(float) * (size_t)n * n),
                                  "image buffer");
            if (!g_status)
                g_status = cuda_error(
                    cudaMalloc((void **)&g_dsino, sizeof(float) * (size_t)np * prjWidth),
                    "sinogram buffer");
            if (g_status) release_global();
        }
    }
    snprintf(g_msg, sizeof g_msg, "%s", g_status ? ctprj_last_error() : "");
}

extern "C" void showSetup(void)
{
    printf("config.n=%d\n", g_conf.n);
    printf("config.prjWidth=%d\n", g_conf.prjWidth);
    printf("config.np=%d\n", g_conf.np);
    printf("config.prjFull=%d\n", g_conf.prjFull);
    printf("config.dSize=%g\n", g_conf.dSize);
    printf("config.effectiveRate=%g\n", g_conf.effectiveRate);
    printf("config.d=%g\n", g_conf.d);
}

int ctprj_fbp_device(ctprj_plan *plan, const float *d_sino, float *d_img, cudaStream_t s);

// The device address of a host buffer the GPU can write directly (page-locked
// and mapped, as every cudaHostAlloc / cudaHostRegister buffer is under
// unified addressing), or NULL for pageable memory.
static float *mapped_alias(void *host)
{
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, host) != cudaSuccess) {
        cudaGetLastError();
        return nullptr;
    }
    return a.type == cudaMemoryTypeHost ? (float *)a.devicePointer : nullptr;
}

// The staging buffer, grown to at least `bytes` (g_mu held)
static int stage(size_t bytes)
{
    if (g_stage_bytes >= bytes) return CTPRJ_OK;
    if (g_stage) cudaFreeHost(g_stage);
    g_stage = nullptr;
    g_stage_bytes = 0;
    int st = cuda_error(cudaHostAlloc((void **)&g_stage, bytes, cudaHostAllocMapped), "staging buffer");
    if (!st) g_stage_bytes = bytes;
    return st;
}

// Upload of a caller buffer: straight from page-locked memory, or through the
// staging buffer, each 1 MiB piece sent as soon as it has been copied in (the
// host threads copy while the copy engine sends).  The device and stream of a
// piece's transfer are the calling thread's: every thread sets the device.
struct UploadCtx {
    char *dev;
    const char *stage;
    cudaStream_t s;
    int device;
};

static int send_piece(void *p, size_t off, size_t len)
{
    const UploadCtx &u = *(const UploadCtx *)p;
    if (cudaSetDevice(u.device) != cudaSuccess) return cuda_error(cudaGetLastError(), "upload device");
    return cuda_error(cudaMemcpyAsync(u.dev + off, u.stage + off, len, cudaMemcpyHostToDevice, u.s), "upload");
}

static int upload(float *dev, const float *host, size_t bytes, cudaStream_t s, const char *what)
{
    if (mapped_alias((void *)host)) return cuda_error(cudaMemcpyAsync(dev, host, bytes, cudaMemcpyHostToDevice, s), what);
    int st = stage(std::max(sizeof(float) * g_conf.imgSize, sizeof(float) * g_conf.sinoSize));
    if (st) return st;
    UploadCtx u = {(char *)dev, (const char *)g_stage, s, g_plan->device};
    st = HostCopier::get().copy(g_stage, host, bytes, 1u << 20, send_piece, &u);
    // the failing piece's message is on the thread that sent it
    return st ? set_error(st, "%s: a host-to-device copy failed", what) : CTPRJ_OK;
}

// prj/gpuPrj.cu:899-958: upload the input, run the pass, download the result,
// return when the result is in the caller's buffer.  The result goes straight
// over the bus into page-locked memory as the kernel produces it: the caller's
// buffer when it is page-locked, else the staging buffer (after the input has
// left it), copied out by the host threads when the pass is done.
extern "C" int gpuPrj(float *img, float *sino, char cmd)
{
    std::lock_guard<std::mutex> lk(g_mu);
    if (g_status != CTPRJ_OK) return set_error(g_status, "%s", g_msg);
    if (!img || !sino) return set_error(CTPRJ_EINVAL, "NULL image or sinogram pointer");
    DeviceGuard dg(g_plan->device);
    if (dg.status) return dg.status;
    const size_t ib = sizeof(float) * g_conf.imgSize, sb = sizeof(float) * g_conf.sinoSize;
    cudaStream_t s = 0;
    int st;
    float *result = nullptr;   // the caller's pageable result buffer
    size_t rb = 0;
    if (cmd & FWD_BIT) {
        float *out = mapped_alias(sino);
        if ((st = upload(g_dimg, img, ib, s, "image upload"))) return st;
        if (!out) {
            if ((st = stage(std::max(ib, sb)))) return st;
            out = mapped_alias(g_stage);
            result = sino;
            rb = sb;
        }
        if ((st = ctprj_forward(g_plan, g_dimg, out, s))) return st;
    } else if (cmd & (BWD_BIT | FBP_BIT)) {
        float *out = mapped_alias(img);
        if ((st = upload(g_dsino, sino, sb, s, "sinogram upload"))) return st;
        if (!out) {
            if ((st = stage(std::max(ib, sb)))) return st;
            out = mapped_alias(g_stage);
            result = img;
            rb = ib;
        }
        if ((st = (cmd & BWD_BIT) ? ctprj_backward(g_plan, g_dsino, out, s)
                                  : ctprj_fbp_device(g_plan, g_dsino, out, s)))
            return st;
    } else {
        return CTPRJ_OK;   // the reference does nothing for other commands
    }
    if ((st = cuda_error(cudaStreamSynchronize(s), "gpuPrj synchronize"))) return st;
    if (result) HostCopier::get().copy(result, g_stage, rb);
    return CTPRJ_OK;
}

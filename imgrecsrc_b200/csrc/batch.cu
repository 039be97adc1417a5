// batch.cu -- many slices of different geometries in one persistent launch,
// captured in CUDA graphs, with launch shapes chosen by a tuner.
//
// Each slice has its own plan (tables, scratch).  A batched forward is one
// batched quad-image pass plus one persistent forward kernel over the blocks of all
// slices; a batched backprojection is one persistent kernel over the tiles of
// all slices (projector.cu, k_*_batch).  Results are identical to the slices'
// own ctprj_forward / ctprj_backward: the block bodies are the same.
//
// The tuner times the candidate launch shapes on the bound buffers -- forward
// block of 2, 4 or 8 views x 32 rays, backprojection batches of 8 or 16 views
// per staged tile, full or half residency, slices handed out largest first or
// in order -- and keeps the fastest; results are cached in a text file keyed by
// the device and the batch's geometries.
#include <algorithm>
#include <cstdio>
#include <cstring>
#include <numeric>
#include <string>
#include <vector>

#include "ctprj_internal.h"
#include "../../include/ctprj_batch.h"

using namespace ctprj;

struct BatchConfig {
    int fwd_views = 4;     // 2, 4, 8
    int fwd_occ = 1;       // 1 full residency, 2 half
    int fwd_order = 1;     // 1 largest slice first, 0 as given
    int bwd_vb = 8;        // views per staged batch (16 only with 32-detector staging)
    int bwd_occ = 1;
    int bwd_order = 1;
};

struct ctprj_batch {
    int device = 0;
    int n = 0;
    std::vector<ctprj_geometry> geoms;
    std::vector<ctprj_plan *> plans;
    std::vector<BatchSlice> hs;
    BatchSlice *d_slices = nullptr;
    int *d_order_f = nullptr, *d_order_b = nullptr;
    long long *d_fprefix = nullptr, *d_bprefix = nullptr, *d_tprefix = nullptr;
    unsigned long long *d_counter = nullptr;   // [0] forward, [1] backward
    int *d_status = nullptr;                   // streaming: per slice, 1 = timed out
    long long ftotal = 0, btotal = 0, ttotal = 0;
    int seg = 0;                  // staging capacity used by the batched backprojection
    int bound = 0;                // buffers bound
    BatchConfig cfg;
    cudaGraphExec_t gexec[2] = {nullptr, nullptr};
    int sms = 148;
};

namespace {

struct Dev {
    int prev = -1, dev;
    explicit Dev(int d) : dev(d)
    {
        cudaGetDevice(&prev);
        if (prev != dev) cudaSetDevice(dev);
    }
    ~Dev()
    {
        if (prev >= 0 && prev != dev) cudaSetDevice(prev);
    }
};

long long fwd_items(const ctprj_plan *p, int V)
{
    return (long long)((p->nb + V - 1) / V) * ((p->nk + 31) / 32);
}

long long bwd_items(const ctprj_plan *p)
{
    const int T = (p->g.half + 1 + 15) / 16;
    return (long long)T * (T + 1) / 2;
}

// slice work estimate for ordering: updates ~ n^2 * views
double slice_cost(const ctprj_geometry &g) { return (double)g.n * g.n * g.np; }

void free_graphs(ctprj_batch *b)
{
    for (int i = 0; i < 2; ++i)
        if (b->gexec[i]) {
            cudaGraphExecDestroy(b->gexec[i]);
            b->gexec[i] = nullptr;
        }
}

// work lists for the current configuration
int upload_lists(ctprj_batch *b)
{
    const int n = b->n;
    std::vector<int> of(n), ob(n);
    std::iota(of.begin(), of.end(), 0);
    std::iota(ob.begin(), ob.end(), 0);
    auto bigger = [&](int a, int c) { return slice_cost(b->geoms[a]) > slice_cost(b->geoms[c]); };
    if (b->cfg.fwd_order) std::stable_sort(of.begin(), of.end(), bigger);
    if (b->cfg.bwd_order) std::stable_sort(ob.begin(), ob.end(), bigger);
    std::vector<long long> fp(n + 1, 0), bp(n + 1, 0), tp(n + 1, 0);
    for (int i = 0; i < n; ++i) {
        fp[i + 1] = fp[i] + fwd_items(b->plans[of[i]], b->cfg.fwd_views);
        bp[i + 1] = bp[i] + bwd_items(b->plans[ob[i]]);
        tp[i + 1] = tp[i] + quad_tiles(b->geoms[i].n);
    }
    b->ftotal = fp[n];
    b->btotal = bp[n];
    b->ttotal = tp[n];
    int st;
    if ((st = cuda_error(cudaMemcpy(b->d_order_f, of.data(), sizeof(int) * n, cudaMemcpyHostToDevice), "batch lists")) ||
        (st = cuda_error(cudaMemcpy(b->d_order_b, ob.data(), sizeof(int) * n, cudaMemcpyHostToDevice), "batch lists")) ||
        (st = cuda_error(cudaMemcpy(b->d_fprefix, fp.data(), sizeof(long long) * (n + 1), cudaMemcpyHostToDevice), "batch lists")) ||
        (st = cuda_error(cudaMemcpy(b->d_bprefix, bp.data(), sizeof(long long) * (n + 1), cudaMemcpyHostToDevice), "batch lists")) ||
        (st = cuda_error(cudaMemcpy(b->d_tprefix, tp.data(), sizeof(long long) * (n + 1), cudaMemcpyHostToDevice), "batch lists")))
        return st;
    free_graphs(b);
    return CTPRJ_OK;
}

BatchArgs fwd_args(const ctprj_batch *b)
{
    BatchArgs a;
    a.slices = b->d_slices;
    a.nslices = b->n;
    a.order = b->d_order_f;
    a.prefix = b->d_fprefix;
    a.total = b->ftotal;
    a.tprefix = b->d_tprefix;
    a.ttotal = b->ttotal;
    a.counter = b->d_counter;
    return a;
}

BatchArgs bwd_args(const ctprj_batch *b)
{
    BatchArgs a = fwd_args(b);
    a.order = b->d_order_b;
    a.prefix = b->d_bprefix;
    a.total = b->btotal;
    a.counter = b->d_counter + 1;
    return a;
}

int ctas(const ctprj_batch *b, int kind, int param, int occ)
{
    int per = 1;
    if (batch_max_ctas(kind, param, &per) || per < 1) per = 1;
    per = std::max(1, per / occ);
    return per * b->sms;
}

int enqueue_forward(ctprj_batch *b, cudaStream_t s)
{
    int st;
    if ((st = cuda_error(cudaMemsetAsync(b->d_counter, 0, sizeof(unsigned long long), s), "batch counter")))
        return st;
    const BatchArgs a = fwd_args(b);
    if ((st = launch_quad_batch(a, s))) return st;
    return launch_forward_batch(a, b->cfg.fwd_views, ctas(b, 0, b->cfg.fwd_views, b->cfg.fwd_occ), s);
}

int bwd_param(const ctprj_batch *b) { return (b->seg <= 32 ? 3200 : 6400) + b->cfg.bwd_vb; }

int enqueue_backward(ctprj_batch *b, cudaStream_t s)
{
    int st;
    if ((st = cuda_error(cudaMemsetAsync(b->d_counter + 1, 0, sizeof(unsigned long long), s), "batch counter")))
        return st;
    const int seg = b->seg <= 32 ? 32 : 64;
    const int vb = seg == 32 ? b->cfg.bwd_vb : 8;
    return launch_backward_batch(bwd_args(b), seg, vb, ctas(b, 1, bwd_param(b), b->cfg.bwd_occ), s);
}

unsigned long long signature(const ctprj_batch *b)
{
    unsigned long long h = 1469598103934665603ULL;   // FNV-1a
    auto mix = [&](const void *p, size_t len) {
        const unsigned char *c = (const unsigned char *)p;
        for (size_t i = 0; i < len; ++i) {
            h ^= c[i];
            h *= 1099511628211ULL;
        }
    };
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, b->device) == cudaSuccess) mix(prop.name, strlen(prop.name));
    for (const auto &g : b->geoms) mix(&g, sizeof g);
    return h;
}

}  // namespace

extern "C" int ctprj_batch_create(const ctprj_geometry *geoms, int nslices, int device,
                                  ctprj_batch **out)
{
    if (!geoms || !out || nslices < 1) return set_error(CTPRJ_EINVAL, "invalid batch arguments");
    *out = nullptr;
    if (device < 0 && cudaGetDevice(&device) != cudaSuccess) device = 0;
    Dev dv(device);
    ctprj_batch *b = new ctprj_batch();
    b->device = device;
    b->n = nslices;
    b->geoms.assign(geoms, geoms + nslices);
    cudaDeviceGetAttribute(&b->sms, cudaDevAttrMultiProcessorCount, device);
    int st = CTPRJ_OK;
    for (int i = 0; i < nslices && !st; ++i) {
        ctprj_plan *p = nullptr;
        st = ctprj_plan_create(&geoms[i], device, &p);
        if (!st) b->plans.push_back(p);
    }
    if (!st) {
        b->hs.resize(nslices);
        for (int i = 0; i < nslices; ++i) {
            BatchSlice &h = b->hs[i];
            memset(&h, 0, sizeof h);
            h.fp = make_fwd_params(b->plans[i]);
            h.bp = make_bwd_params(b->plans[i]);
            h.quad = b->plans[i]->d_quad;
            h.tiled = b->plans[i]->bwd_seg > 0;
            b->seg = std::max(b->seg, b->plans[i]->bwd_seg);
        }
        // every staged slice must fit the batch's staging capacity
        for (int i = 0; i < nslices; ++i)
            if (b->plans[i]->bwd_seg > 32) b->hs[i].tiled = (b->seg == 64);
        const int n = nslices;
        if (!(st = cuda_error(cudaMalloc((void **)&b->d_slices, sizeof(BatchSlice) * n), "batch tables")) &&
            !(st = cuda_error(cudaMalloc((void **)&b->d_order_f, sizeof(int) * n), "batch tables")) &&
            !(st = cuda_error(cudaMalloc((void **)&b->d_order_b, sizeof(int) * n), "batch tables")) &&
            !(st = cuda_error(cudaMalloc((void **)&b->d_fprefix, sizeof(long long) * (n + 1)), "batch tables")) &&
            !(st = cuda_error(cudaMalloc((void **)&b->d_bprefix, sizeof(long long) * (n + 1)), "batch tables")) &&
            !(st = cuda_error(cudaMalloc((void **)&b->d_tprefix, sizeof(long long) * (n + 1)), "batch tables")) &&
            !(st = cuda_error(cudaMalloc((void **)&b->d_counter, 2 * sizeof(unsigned long long)), "batch tables")) &&
            !(st = cuda_error(cudaMalloc((void **)&b->d_status, sizeof(int) * n), "batch tables")))
            st = upload_lists(b);
    }
    if (st) {
        ctprj_batch_destroy(b);
        return st;
    }
    *out = b;
    return CTPRJ_OK;
}

extern "C" void ctprj_batch_destroy(ctprj_batch *b)
{
    if (!b) return;
    Dev dv(b->device);
    free_graphs(b);
    for (auto *p : b->plans) ctprj_plan_destroy(p);
    cudaFree(b->d_slices);
    cudaFree(b->d_order_f);
    cudaFree(b->d_order_b);
    cudaFree(b->d_fprefix);
    cudaFree(b->d_bprefix);
    cudaFree(b->d_tprefix);
    cudaFree(b->d_counter);
    cudaFree(b->d_status);
    delete b;
}

extern "C" int ctprj_batch_bind(ctprj_batch *b, const float *const *d_imgs, float *const *d_sinos,
                                const float *const *d_bsinos, float *const *d_bimgs)
{
    if (!b) return set_error(CTPRJ_EINVAL, "NULL batch");
    Dev dv(b->device);
    for (int i = 0; i < b->n; ++i) {
        b->hs[i].img = d_imgs ? d_imgs[i] : nullptr;
        b->hs[i].sino = d_sinos ? d_sinos[i] : nullptr;
        b->hs[i].bsino = d_bsinos ? d_bsinos[i] : nullptr;
        b->hs[i].bimg = d_bimgs ? d_bimgs[i] : nullptr;
    }
    b->bound = (d_imgs && d_sinos ? 1 : 0) | (d_bsinos && d_bimgs ? 2 : 0);
    free_graphs(b);
    return cuda_error(cudaMemcpy(b->d_slices, b->hs.data(), sizeof(BatchSlice) * b->n,
                                 cudaMemcpyHostToDevice),
                      "batch bind");
}

extern "C" int ctprj_batch_forward(ctprj_batch *b, void *stream)
{
    if (!b || !(b->bound & 1)) return set_error(CTPRJ_EINVAL, "batch has no forward buffers bound");
    Dev dv(b->device);
    cudaStream_t s = (cudaStream_t)stream;
    if (b->gexec[0]) return cuda_error(cudaGraphLaunch(b->gexec[0], s), "batch graph launch");
    return enqueue_forward(b, s);
}

extern "C" int ctprj_batch_backward(ctprj_batch *b, void *stream)
{
    if (!b || !(b->bound & 2)) return set_error(CTPRJ_EINVAL, "batch has no backward buffers bound");
    Dev dv(b->device);
    cudaStream_t s = (cudaStream_t)stream;
    if (b->gexec[1]) return cuda_error(cudaGraphLaunch(b->gexec[1], s), "batch graph launch");
    return enqueue_backward(b, s);
}

extern "C" int ctprj_batch_capture(ctprj_batch *b, void *stream)
{
    if (!b || !b->bound) return set_error(CTPRJ_EINVAL, "batch has no buffers bound");
    Dev dv(b->device);
    cudaStream_t s = (cudaStream_t)stream;
    free_graphs(b);
    for (int w = 0; w < 2; ++w) {
        if (!(b->bound & (1 << w))) continue;
        cudaGraph_t graph = nullptr;
        int st = cuda_error(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal), "begin capture");
        if (st) return st;
        const int est = w == 0 ? enqueue_forward(b, s) : enqueue_backward(b, s);
        st = cuda_error(cudaStreamEndCapture(s, &graph), "end capture");
        if (est || st) {
            if (graph) cudaGraphDestroy(graph);
            return est ? est : st;
        }
        st = cuda_error(cudaGraphInstantiate(&b->gexec[w], graph, 0), "graph instantiate");
        cudaGraphDestroy(graph);
        if (st) return st;
    }
    return CTPRJ_OK;
}

extern "C" int ctprj_batch_config(ctprj_batch *b, char *buf, int len)
{
    if (!b || !buf || len < 1) return set_error(CTPRJ_EINVAL, "invalid arguments");
    snprintf(buf, len, "fwd_views=%d fwd_occ=%d fwd_order=%d bwd_vb=%d bwd_occ=%d bwd_order=%d seg=%d",
             b->cfg.fwd_views, b->cfg.fwd_occ, b->cfg.fwd_order, b->cfg.bwd_vb, b->cfg.bwd_occ,
             b->cfg.bwd_order, b->seg);
    return CTPRJ_OK;
}

static float time_ms(ctprj_batch *b, int which, cudaStream_t s, int reps)
{
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    float best = 1e30f;
    for (int r = 0; r < reps + 1; ++r) {
        cudaEventRecord(e0, s);
        const int st = which == 0 ? enqueue_forward(b, s) : enqueue_backward(b, s);
        cudaEventRecord(e1, s);
        cudaEventSynchronize(e1);
        float ms = 0.0f;
        cudaEventElapsedTime(&ms, e0, e1);
        if (st) ms = 1e30f;
        if (r > 0) best = std::min(best, ms);   // the first run warms up
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return best;
}

extern "C" int ctprj_batch_autotune(ctprj_batch *b, void *stream, const char *cache_path)
{
    if (!b || b->bound != 3) return set_error(CTPRJ_EINVAL, "autotune needs forward and backward buffers bound");
    Dev dv(b->device);
    cudaStream_t s = (cudaStream_t)stream;
    const unsigned long long sig = signature(b);
    if (cache_path) {
        if (FILE *f = fopen(cache_path, "r")) {
            unsigned long long key;
            BatchConfig c;
            int found = 0;
            while (fscanf(f, "%llx %d %d %d %d %d %d", &key, &c.fwd_views, &c.fwd_occ, &c.fwd_order,
                          &c.bwd_vb, &c.bwd_occ, &c.bwd_order) == 7)
                if (key == sig) {
                    b->cfg = c;
                    found = 1;
                }
            fclose(f);
            if (found) return upload_lists(b);
        }
    }
    BatchConfig best = b->cfg;
    float best_f = 1e30f, best_b = 1e30f;
    for (int views : {2, 4, 8})
        for (int occ : {1, 2})
            for (int order : {1, 0}) {
                b->cfg.fwd_views = views;
                b->cfg.fwd_occ = occ;
                b->cfg.fwd_order = order;
                int st = upload_lists(b);
                if (st) return st;
                const float t = time_ms(b, 0, s, 2);
                if (t < best_f) {
                    best_f = t;
                    best.fwd_views = views;
                    best.fwd_occ = occ;
                    best.fwd_order = order;
                }
            }
    b->cfg.fwd_views = best.fwd_views;
    b->cfg.fwd_occ = best.fwd_occ;
    b->cfg.fwd_order = best.fwd_order;
    for (int vb : {8, 16})
        for (int occ : {1, 2})
            for (int order : {1, 0}) {
                if (vb == 16 && b->seg > 32) continue;
                b->cfg.bwd_vb = vb;
                b->cfg.bwd_occ = occ;
                b->cfg.bwd_order = order;
                int st = upload_lists(b);
                if (st) return st;
                const float t = time_ms(b, 1, s, 2);
                if (t < best_b) {
                    best_b = t;
                    best.bwd_vb = vb;
                    best.bwd_occ = occ;
                    best.bwd_order = order;
                }
            }
    b->cfg = best;
    int st = upload_lists(b);
    if (st) return st;
    if (cache_path)
        if (FILE *f = fopen(cache_path, "a")) {
            fprintf(f, "%llx %d %d %d %d %d %d\n", sig, best.fwd_views, best.fwd_occ, best.fwd_order,
                    best.bwd_vb, best.bwd_occ, best.bwd_order);
            fclose(f);
        }
    return cuda_error(cudaGetLastError(), "autotune");
}

// ----------------------------------------------------------------- streaming

extern "C" int ctprj_stream_flags_create(int n, int **host_flags, int **dev_flags)
{
    if (n < 1 || !host_flags || !dev_flags) return set_error(CTPRJ_EINVAL, "invalid arguments");
    int *h = nullptr;
    int st = cuda_error(cudaHostAlloc((void **)&h, sizeof(int) * n, cudaHostAllocMapped), "flag allocation");
    if (st) return st;
    memset(h, 0, sizeof(int) * n);
    int *d = nullptr;
    if ((st = cuda_error(cudaHostGetDevicePointer((void **)&d, h, 0), "flag mapping"))) {
        cudaFreeHost(h);
        return st;
    }
    *host_flags = h;
    *dev_flags = d;
    return CTPRJ_OK;
}

extern "C" void ctprj_stream_flags_destroy(int *host_flags)
{
    if (host_flags) cudaFreeHost(host_flags);
}

extern "C" int ctprj_batch_stream_backward(ctprj_batch *b, const int *dev_flags, double timeout_s,
                                           int *status, void *stream)
{
    if (!b || !(b->bound & 2) || !dev_flags)
        return set_error(CTPRJ_EINVAL, "batch has no backward buffers bound or no flags");
    if (!(timeout_s > 0) || timeout_s > 60)
        return set_error(CTPRJ_EINVAL, "timeout must be in (0, 60] seconds");
    Dev dv(b->device);
    cudaStream_t s = (cudaStream_t)stream;
    int st;
    if ((st = cuda_error(cudaMemsetAsync(b->d_counter + 1, 0, sizeof(unsigned long long), s), "batch counter")) ||
        (st = cuda_error(cudaMemsetAsync(b->d_status, 0, sizeof(int) * b->n, s), "stream status")))
        return st;
    const int seg = b->seg <= 32 ? 32 : 64;
    const int vb = seg == 32 ? b->cfg.bwd_vb : 8;
    if ((st = launch_backward_stream(bwd_args(b), seg, vb, ctas(b, 1, bwd_param(b), b->cfg.bwd_occ),
                                     dev_flags, b->d_status,
                                     (unsigned long long)(timeout_s * 1e9), s)))
        return st;
    std::vector<int> h(b->n, 0);
    if ((st = cuda_error(cudaMemcpyAsync(h.data(), b->d_status, sizeof(int) * b->n, cudaMemcpyDeviceToHost, s), "stream status")) ||
        (st = cuda_error(cudaStreamSynchronize(s), "stream synchronize")))
        return st;
    int late = 0;
    for (int i = 0; i < b->n; ++i) {
        if (status) status[i] = h[i];
        late += h[i] != 0;
    }
    if (late) return set_error(CTPRJ_ETIMEOUT, "%d of %d slices were not published within %.3g s", late, b->n, timeout_s);
    return CTPRJ_OK;
}

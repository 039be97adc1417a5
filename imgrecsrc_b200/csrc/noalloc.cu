// noalloc.cu -- forward projection for callers that may not allocate device
// memory.
//
// Some callers cannot call cudaMalloc: code that runs inside another
// framework's memory pool or allocator (where a foreign cudaMalloc would
// fragment or bypass the pool, or is forbidden outright), real-time loops that
// must not block on allocation, and embedders that have already reserved every
// byte of the GPU.  ctprj_forward_noalloc serves them: the caller passes only
// the geometry, the input image and the output sinogram, and the call uses
// neither cudaMalloc nor cudaFree nor any allocating library routine.  The
// scratch the forward pass needs -- the quad image (the eight symmetric
// copies of each pixel, twice the image's size) and the ray/view tables --
// lives in the file-scope arrays below, which every GPU that loads this
// library holds until the process exits (about 8.5 MiB).
//
// Limits: n <= 1024, prjWidth <= 4096, prjFull <= 8192 (so at most 1025 base
// views).  Larger geometries are rejected with CTPRJ_ERANGE; they need the
// plan API.
//
// All calls share these arrays.  Each call overwrites every element it later
// reads (the quad image is rebuilt for the geometry and the tables are copied
// in full for the geometry), so nothing has to start at zero, but calls whose
// work overlaps on the GPU -- on different streams, or from different host
// threads -- race on the shared arrays and must be serialised by the caller.
//
// The first call on each device looks up the device addresses of the arrays
// (cudaGetSymbolAddress, with that device current); make that first call
// before any stream capture.
#include <cmath>
#include <cstring>
#include <mutex>

#include "ctprj_internal.h"

namespace ctprj {

constexpr int kNoAllocMaxN = 1024;
constexpr int kNoAllocMaxW = 4096;
constexpr int kNoAllocMaxP = 8192;
constexpr int kNoAllocMaxViews = kNoAllocMaxP / 8 + 1;
constexpr int kNoAllocMaxDevices = 64;

// quad image of an n <= kNoAllocMaxN image: (half + 1) x (2 half + 1) float4
static __device__ __align__(256) float4 g_noalloc_quad[(kNoAllocMaxN / 2 + 1) * (kNoAllocMaxN + 1)];
static __device__ __align__(256) FwdView g_noalloc_view[kNoAllocMaxViews];
static __device__ __align__(256) DetEntry g_noalloc_det[kNoAllocMaxW];

struct NoAllocSymbols {
    float4 *quad;
    FwdView *view;
    DetEntry *det;
};

static std::mutex g_noalloc_mu;
static bool g_noalloc_ready[kNoAllocMaxDevices];
static NoAllocSymbols g_noalloc_sym[kNoAllocMaxDevices];
// host staging of the tables (static, so that no host allocation is made either)
static FwdView g_host_view[kNoAllocMaxViews];
static DetEntry g_host_det[kNoAllocMaxW];

// Device addresses of the scratch arrays on the current device, looked up on
// the first call there.  The array names are host-side stand-ins; only these
// addresses may be handed to a kernel.
static int noalloc_symbols(int dev, NoAllocSymbols *out)
{
    if (dev < 0 || dev >= kNoAllocMaxDevices)
        return set_error(CTPRJ_ERANGE, "device ordinal %d beyond the %d supported", dev,
                         kNoAllocMaxDevices);
    if (!g_noalloc_ready[dev]) {
        NoAllocSymbols s;
        int st;
        if ((st = cuda_error(cudaGetSymbolAddress((void **)&s.quad, g_noalloc_quad),
                             "cudaGetSymbolAddress(scratch image)")) ||
            (st = cuda_error(cudaGetSymbolAddress((void **)&s.view, g_noalloc_view),
                             "cudaGetSymbolAddress(view table)")) ||
            (st = cuda_error(cudaGetSymbolAddress((void **)&s.det, g_noalloc_det),
                             "cudaGetSymbolAddress(detector table)")))
            return st;
        g_noalloc_sym[dev] = s;
        g_noalloc_ready[dev] = true;
    }
    *out = g_noalloc_sym[dev];
    return CTPRJ_OK;
}

// the reference's float-formed view angle (prj/cpuPrj.c:342)
static double noalloc_view_angle(int i, int P)
{
    volatile float th = (float)(2 * i) * kRefPiF;
    th = th / (float)P;
    return (double)th;
}

static int noalloc_view_of(int j, int b, int P)
{
    static const int q[8] = {0, 1, 2, 3, 2, 3, 4, 1};
    static const int sg[8] = {1, 1, 1, 1, -1, -1, -1, -1};
    int v = (q[j] * (P / 4) + sg[j] * b) % P;
    return v < 0 ? v + P : v;
}

}  // namespace ctprj

using namespace ctprj;

extern "C" int ctprj_forward_noalloc(const ctprj_geometry *geom, const float *d_img,
                                     float *d_sino, void *stream)
{
    if (!geom || !d_img || !d_sino) return set_error(CTPRJ_EINVAL, "NULL geometry or buffer");
    const ctprj_geometry &gm = *geom;
    if (gm.n < 1 || gm.prjWidth < 1 || gm.np < 1 || gm.prjFull < 4 || gm.prjFull % 4 != 0 ||
        gm.np > gm.prjFull || !(gm.dSize > 0.0f) || !(gm.effectiveRate > 0.0f) ||
        !std::isfinite(gm.dSize) || !std::isfinite(gm.effectiveRate) || !std::isfinite(gm.d))
        return set_error(CTPRJ_EINVAL, "invalid geometry (n=%d prjWidth=%d np=%d prjFull=%d)", gm.n,
                         gm.prjWidth, gm.np, gm.prjFull);
    if (gm.n > kNoAllocMaxN || gm.prjWidth > kNoAllocMaxW || gm.prjFull > kNoAllocMaxP)
        return set_error(CTPRJ_ERANGE,
                         "ctprj_forward_noalloc is limited to n <= %d, prjWidth <= %d and "
                         "prjFull <= %d (got n=%d prjWidth=%d prjFull=%d); use the plan API",
                         kNoAllocMaxN, kNoAllocMaxW, kNoAllocMaxP, gm.n, gm.prjWidth, gm.prjFull);

    // a plan on the stack whose tables and scratch are the static arrays
    ctprj_plan p;
    memset(&p, 0, sizeof p);
    p.geom = gm;
    Geo &g = p.g;
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
    p.nb = gm.np < gm.prjFull / 8 + 1 ? gm.np : gm.prjFull / 8 + 1;
    p.k0 = (g.W % 2 == 0) ? 1 : 0;
    p.nk = g.fan ? (g.W % 2 == 0 ? g.W - 1 : g.W) : (g.W % 2 == 0 ? g.W / 2 : (g.W + 1) / 2);

    int dev = 0;
    int st = cuda_error(cudaGetDevice(&dev), "cudaGetDevice");
    if (st) return st;
    p.device = dev;
    cudaStream_t s = (cudaStream_t)stream;

    std::lock_guard<std::mutex> lk(g_noalloc_mu);
    NoAllocSymbols sym;
    if ((st = noalloc_symbols(dev, &sym))) return st;
    for (int b = 0; b < p.nb; ++b) {
        const double th = noalloc_view_angle(b, g.P);
        g_host_view[b].c = cos(th);
        g_host_view[b].s = sin(th);
        const bool mirror = b > 0 && (float)b < (float)g.P * 0.125f;
        for (int j = 0; j < 8; ++j) {
            const int v = noalloc_view_of(j, b, g.P);
            g_host_view[b].out[j] = ((j < 4 || mirror) && v < g.np) ? v : -1;
        }
    }
    for (int k = 0; k < g.W; ++k) {
        DetEntry &e = g_host_det[k];
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
    // pageable-memory copies return once the host tables have been staged, so
    // the static host buffers may be refilled by the next call
    if ((st = cuda_error(cudaMemcpyAsync(sym.view, g_host_view, sizeof(FwdView) * (size_t)p.nb,
                                         cudaMemcpyHostToDevice, s),
                         "view table upload")) ||
        (st = cuda_error(cudaMemcpyAsync(sym.det, g_host_det, sizeof(DetEntry) * (size_t)g.W,
                                         cudaMemcpyHostToDevice, s),
                         "detector table upload")))
        return st;
    p.d_fview = sym.view;
    p.d_det = sym.det;
    p.d_quad = sym.quad;
    if ((st = launch_quad(d_img, sym.quad, g.n, s))) return st;
    return launch_forward(&p, sym.quad, d_sino, nullptr, s);
}

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
// before any stream capture.  The addresses are kept for the life of the
// process: a caller that tears the device's context down (cudaDeviceReset)
// and then calls again would hand the kernels stale addresses, so callers of
// this entry point must not reset the device.  A call on a stream that is
// being captured returns CTPRJ_EINVAL: its table uploads read static host
// buffers that every later call overwrites.
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

}  // namespace ctprj

using namespace ctprj;

extern "C" int ctprj_forward_noalloc(const ctprj_geometry *geom, const float *d_img,
                                     float *d_sino, void *stream)
{
    if (!d_img || !d_sino) return set_error(CTPRJ_EINVAL, "NULL image or sinogram");
    int st = validate_geometry(geom);
    if (st) return st;
    const ctprj_geometry &gm = *geom;
    if (gm.n > kNoAllocMaxN || gm.prjWidth > kNoAllocMaxW || gm.prjFull > kNoAllocMaxP)
        return set_error(CTPRJ_ERANGE,
                         "ctprj_forward_noalloc is limited to n <= %d, prjWidth <= %d and "
                         "prjFull <= %d (got n=%d prjWidth=%d prjFull=%d); use the plan API",
                         kNoAllocMaxN, kNoAllocMaxW, kNoAllocMaxP, gm.n, gm.prjWidth, gm.prjFull);
    cudaStream_t s = (cudaStream_t)stream;
    // The table uploads below read the static host tables, which the next call
    // overwrites: a captured upload would replay whatever a later call left
    // there, so a call on a capturing stream is refused.
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    if ((st = cuda_error(cudaStreamIsCapturing(s, &cap), "cudaStreamIsCapturing"))) return st;
    if (cap != cudaStreamCaptureStatusNone)
        return set_error(CTPRJ_EINVAL, "ctprj_forward_noalloc was called on a stream that is being captured");

    // a plan on the stack whose tables and scratch are the static arrays
    ctprj_plan p;
    memset(&p, 0, sizeof p);
    p.geom = gm;
    p.g = make_geo(gm);
    const Geo &g = p.g;
    fwd_ray_set(g, &p.nb, &p.k0, &p.nk);

    int dev = 0;
    if ((st = cuda_error(cudaGetDevice(&dev), "cudaGetDevice"))) return st;
    p.device = dev;

    std::lock_guard<std::mutex> lk(g_noalloc_mu);
    NoAllocSymbols sym;
    if ((st = noalloc_symbols(dev, &sym))) return st;
    fill_fwd_views(g, p.nb, g_host_view);
    fill_det_table(g, g_host_det);
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

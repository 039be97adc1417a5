// ctprj_internal.h -- plan layout, geometry tables and kernel parameter
// blocks shared by the host code and the sm_100a kernels.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "../../include/ctprj.h"

namespace ctprj {

// The reference's pi is the float literal 3.14159265359f (prj/prj.h:9) and view
// angles are formed in float arithmetic, fl(fl(2i * pi_f) / prjFull), in both of
// its precisions (prj/cpuPrj.c:342).  View tables are built on the host from
// exactly that value, with cos/sin evaluated in double.
constexpr float kRefPiF = 3.14159265359f;

// Forward base view (0 <= b <= prjFull/8): its direction and, for each of the
// eight symmetric images j (order of prj/cpuPrj.c:383-397), the sinogram row it
// is written to, or -1.  Images 4..7 also mirror the detector.
struct FwdView {
    double c, s;
    int out[8];
};

// Backward base view i (all views for fan beam, the first half for parallel
// beam, prj/cpuPrj.c:76, :213): direction, the sinogram row offsets
// (view * prjWidth, or -1) read for each image j, and for parallel beam the
// rows of the opposite views (view + prjFull/2) read with the detector
// mirrored.  shape = footprint of the parallel ray (unused for fan beam).
struct BwdView {
    double c, s;
    float cf, sf;
    float h, b1, b2, w, iw2, pad;
    int row[8];
    int row2[8];
    int cnt4, cnt8;   // valid reads per weight for 4 / 8 distinct images
};

// Detector k: t = (k - prjWidth/2) * dSize and, for fan beam, the direction
// of its ray relative to the central ray (cos B = d/bq, sin B = t/bq).
struct DetEntry {
    double t, cB, sB;
    float cBf, sBf, invbq, pad;
};

struct Geo {
    int n, W, np, P;
    int pC, half, h2;        // prjWidth/2, (n-1)/2, n/2
    int fan;
    double dSize, beamWidth, d;
    float beamWidthF, dF, invEr;
    float effRate;
};

// Polychromatic epilogue of the fused forward pass (bhc.cu).
struct BhcArgs {
    const double *tab;        // spline table, J * kSplStride doubles
    const double *Ie;         // spectrum coefficients, J doubles
    int J;
    double Ts;                // pixel size: s = Ts * (A x)
    const float *imea;        // measured intensity / I0 per ray (np * prjWidth)
    float *s_out, *w_out;     // per-ray s and r dBL/ds (the backprojected weight); NULL: not kept
    double *r_out;            // per-ray r = df/dBL in FP64: the spectrum gradient sums it over
                              // all rays with cancellation, which single precision would not survive
    double *part;             // per-block partial sums of the likelihood terms
    int noise;                // kNoisePoisson or kNoiseGaussian
    float *proj_out;          // the plain projection of each entry (np * prjWidth); NULL: not kept
};

enum { kModePlain = 0, kModeCount = 1, kModeBhc = 2 };

struct FwdParams {
    Geo g;
    int nb, k0, nk;           // base views, first ray, rays per base view
    int zero_col0;            // even prjWidth: detector 0 written as zero
    int sms;                  // multiprocessors of the plan's device
    const FwdView *view;
    const DetEntry *det;
    BhcArgs bhc;
};

struct BwdParams {
    Geo g;
    int nv;                   // base views looped over
    int tiles_side;
    int zero_axes;            // even n: row 0 and column 0 written as zero
    float scale;              // output scale: FBP PI_f/np/dSize^2, BHC gradient Ts, else 1
    int fast_shadow;          // fan: pixel shadows from the first-order expansion (staged kernel)
    int win;                  // staged kernel: 3 detectors per pixel and view hold every shadow; 0: range
    const BwdView *view;
    const DetEntry *det;
};
// One slice of a batch (batch.cu): its plan's parameter blocks and buffers.
struct BatchSlice {
    FwdParams fp;
    BwdParams bp;
    const float *img;       // forward input
    float4 *quad;           // forward scratch: the quad image (the slice plan's)
    float *sino;            // forward output
    const float *bsino;     // backward input
    float *bimg;            // backward output
    int tiled;              // backward: 1 staged tiles, 0 unstaged
};

// Work lists of a batched launch: items of the slices in `order`, item e
// belonging to the slice at position i when prefix[i] <= e < prefix[i + 1].
struct BatchArgs {
    const BatchSlice *slices;
    int nslices;
    const int *order;
    const long long *prefix;       // forward blocks or backward tiles
    long long total;
    const long long *tprefix;      // quad-image tiles (natural order)
    long long ttotal;
    unsigned long long *counter;   // work counter, zero before each launch
};

}  // namespace ctprj

struct ctprj_plan {
    ctprj_geometry geom;
    int device;
    ctprj::Geo g;
    int nb, k0, nk;           // forward ray set (prj/cpuPrj.c:326-332, :469-475)
    int nv;                   // backward view count
    int bwd_seg;              // staged detectors per view and tile (32, 64), 0: unstaged
    ctprj::FwdView *d_fview;
    ctprj::BwdView *d_bview;
    ctprj::DetEntry *d_det;
    float4 *d_quad;           // scratch: quad image, quad_elems(n) float4
    unsigned long long *d_count;
    // FBP: ramp-filter taps and pre-weights (2*prjWidth), then, where the rows
    // are filtered by FFTs, the twiddles and response of the 2^fbp_log-point
    // transform; filtered-sinogram scratch
    float *d_ramp;
    float *d_fsino;
    int fbp_log;
    // MATLAB-layout entry points: image and sinogram scratch (allocated on first use)
    float *d_mimg;
    float *d_msino;
};

// polychromatic model on a plan (bhc.cu, bhc_loop.cu)
struct ctprj_bhc {
    ctprj_plan *plan;
    int J;
    double Ts;
    double *d_tab;            // spline table, J * kSplStride doubles
    float *d_s, *d_w;         // per-ray state, np * prjWidth each
    double *d_r;
    double *d_part;           // per-block partials
    int part_cap;             // doubles in d_part
    int saved;                // the per-ray state holds the last forward's values
    int noise;                // kNoisePoisson or kNoiseGaussian
    double *d_tab2;           // second-derivative table, J * kSpl2Stride doubles
    float *d_hsino;           // Hessian scratch, np * prjWidth floats (lazily)
};

namespace ctprj {

// out[c] = sum over b < nrows of part[b * stride + c] for c < ncols, in FP64
// and in an order fixed by the launch shape alone (results repeat bit for bit).
// One block: with few columns each column is summed by the whole block (rows
// strided over the threads, then a fixed tree), with many by one thread each.
__device__ __forceinline__ void sum_partials(const double *__restrict__ part, int nrows, int stride,
                                             int ncols, double *__restrict__ out)
{
    if (ncols >= (int)blockDim.x / 4) {
        for (int c = threadIdx.x; c < ncols; c += blockDim.x) {
            double t = 0.0;
            for (int b = 0; b < nrows; ++b) t += part[(size_t)b * stride + c];
            out[c] = t;
        }
        return;
    }
    __shared__ double red[1024];
    for (int c = 0; c < ncols; ++c) {
        double t = 0.0;
        for (int b = threadIdx.x; b < nrows; b += blockDim.x) t += part[(size_t)b * stride + c];
        red[threadIdx.x] = t;
        __syncthreads();
        for (int h = blockDim.x / 2; h > 0; h >>= 1) {
            if ((int)threadIdx.x < h) red[threadIdx.x] += red[threadIdx.x + h];
            __syncthreads();
        }
        if (threadIdx.x == 0) out[c] = red[0];
        __syncthreads();
    }
}

// makes a plan's device current for the lifetime of the guard
struct PlanDevice {
    int prev = -1;
    int dev;
    explicit PlanDevice(int d) : dev(d)
    {
        cudaGetDevice(&prev);
        if (prev != dev) cudaSetDevice(dev);
    }
    ~PlanDevice()
    {
        if (prev >= 0 && prev != dev) cudaSetDevice(prev);
    }
};

int set_error(int status, const char *fmt, ...);
int cuda_error(cudaError_t e, const char *what);

// geometry and host-side tables of a plan (api.cu), shared by every entry
// point that builds them (plans and the allocation-free forward)
int validate_geometry(const ctprj_geometry *g);
Geo make_geo(const ctprj_geometry &gm);
double view_angle(int i, int P);
int view_of(int j, int b, int P);
void fwd_ray_set(const Geo &g, int *nb, int *k0, int *nk);
void fill_fwd_views(const Geo &g, int nb, FwdView *fv);   // fv[nb]
void fill_det_table(const Geo &g, DetEntry *de);          // de[prjWidth]

// buffers of the TV proximal map (tv.cu): D, P1, P2 double-buffered, R1, R2
// (8 images), per-block FP64 partials and the device-side iteration state
struct TvWorkspace {
    float *buf = nullptr;
    double *part = nullptr;
    void *state = nullptr;
    int rows = 0, cols = 0, blocks = 0;
    int alloc(int m, int n, cudaStream_t s);
    void release(cudaStream_t s);
};
// D = argmin ||X - xobs||^2 + 2 lambda TV(X), lb <= X <= ub (tv.cu)
int tv_denoise(TvWorkspace &ws, const float *xobs, int m, int n, double lambda, double lb, double ub,
               int iso, int max_iter, double eps, float *out, int *iterations, cudaStream_t s);
// *d_out = TV(x) in FP64 (device)
int tv_value(TvWorkspace &ws, const float *x, int m, int n, int iso, double *d_out, cudaStream_t s);

// buffers of the wavelet ADMM proximal map (wavelet.cu): LL scratch (half an
// image), s (two), nu; per-block FP64 partials; the device-side ADMM state
struct WvltProx {
    float *buf = nullptr;
    double *part = nullptr;
    void *state = nullptr;
    int rows = 0, cols = 0;
    int alloc(int m, int n, cudaStream_t s);
    void release(cudaStream_t s);
};
// alpha = argmin 1/2 |alpha - a|^2 + I(alpha >= 0) + u |W alpha|_1 by npg/admm.m
// (pmask: pixels of the reconstruction, alpha = 0 elsewhere; cmask: the
// coefficients of the masked transform, maskk; either NULL for all)
int wvlt_admm(WvltProx &ws, const float *a, int rows, int cols, const double *h, int lh, int levels, double u,
              double rel_tol, int max_itr, const float *init, float *alpha, int *iterations, cudaStream_t s,
              const unsigned char *pmask = nullptr, const unsigned char *cmask = nullptr);
// *d_out = |W x|_1 in FP64 (device), over the coefficients of cmask (NULL: all)
int wvlt_l1(WvltProx &ws, const float *x, int rows, int cols, const double *h, int lh, int levels, double *d_out,
            cudaStream_t s, const unsigned char *cmask = nullptr);
// cmask = the coefficients that the pixels of pmask reach (utils/wvltMask.m)
int wvlt_mask(WvltProx &ws, const unsigned char *pmask, int rows, int cols, const double *h, int lh, int levels,
              unsigned char *cmask, cudaStream_t s);

// launchers (projector.cu)
// the quad image of the forward pass (projector.cu): (half + 1) rows of
// 2 half + 1 float4, built in 32 x 32 tiles
__host__ __device__ inline size_t quad_elems(int n)
{
    const int half = (n - 1) / 2;
    return (size_t)(half + 1) * (size_t)(2 * half + 1);
}
__host__ __device__ inline int quad_tiles(int n)
{
    const int half = (n - 1) / 2;
    return ((2 * half + 1 + 31) / 32) * ((half + 1 + 31) / 32);
}
int launch_quad(const float *img, float4 *quad, int n, cudaStream_t s);
int launch_forward(const ctprj_plan *p, const float4 *quad, float *sino,
                   unsigned long long *counter, cudaStream_t s);
// fused forward projection + polychromatic epilogue; returns the number of
// per-block partials written to a.part
int launch_forward_bhc(const ctprj_plan *p, const float4 *quad,
                       const BhcArgs &a, int *nparts, cudaStream_t s);
// the fused likelihood of ctprj_bhc_forward (state saved) that also keeps the
// plain projection A x in proj (bhc.cu)
int bhc_forward_keep_projection(ctprj_bhc *m, const float *d_x, const double *d_Ie, const float *d_imea,
                                double *d_f, float *proj, cudaStream_t s);
int forward_blocks(const ctprj_plan *p);
int backward_max_span(const ctprj_plan *p, int *max_span);
FwdParams make_fwd_params(const ctprj_plan *p);
BwdParams make_bwd_params(const ctprj_plan *p);
// persistent batch launches (projector.cu)
int launch_quad_batch(const BatchArgs &a, cudaStream_t s);
int launch_forward_batch(const BatchArgs &a, int views, int ctas, cudaStream_t s);
int launch_backward_batch(const BatchArgs &a, int seg, int vb, int ctas, cudaStream_t s);
int batch_max_ctas(int kind, int param, int *per_sm);
int launch_backward_stream(const BatchArgs &a, int seg, int vb, int ctas, const int *ready,
                           int *status, unsigned long long timeout_ns, cudaStream_t s);
int launch_backward(const ctprj_plan *p, const float *sino, float *img, int fbp,
                    unsigned long long *counter, cudaStream_t s, float scale = 1.0f);

}  // namespace ctprj

// parprj.cu -- the double-precision masked parallel-beam operator (mParPrj)
// on the GPU.
//
// Same operator as prj/parPrj.c: for angle theta (degrees) and a masked pixel
// at column-major index m of an nr x nc image, x = m / nr - nc/2 and
// y = m % nr - nr/2, dist = x cos + y sin, and detector k (unit pitch, centred
// at max(nc, nr)/2) receives the overlap of its beam [k - bw/2, k + bw/2] with
// the pixel's trapezoid footprint.  The reference forms that footprint from the
// angle |trunc(fmod(theta, 90) - 45)| in whole degrees (prj/parPrj.c:111 passes
// a double to the integer abs()) with pi = 3.14159265; the view table below is
// built on the host the same way, and the overlap uses the reference's
// piecewise formula including its value when the beam is wider than the whole
// footprint (prj/parPrj.c:133-168).  Detectors with k + centre outside
// [0, nc) are skipped as in the reference (prj/parPrj.c:170), and also those
// beyond prjWidth, which the reference would write past its row.
//
//  forward   one block per (angle, pixel chunk); the chunk's contributions
//            accumulate in a shared-memory row (FP64 atomics), then the row is
//            added to the output view.
//  backward  one thread per masked pixel, gathering over angles and detectors
//            in the reference's order; no atomics.
#include <cmath>
#include <cstring>
#include <mutex>
#include <vector>

#include "ctprj_internal.h"
#include "../../include/parprj.h"

namespace ctprj {

struct ParView {
    double c, s, height, b1, b2, areaT, areaR, pad;
};

struct ParArgs {
    double bw;
    int nc, nr, np, W, xC, yC, pC;
    const ParView *view;
};

constexpr double kParPi = 3.14159265;   // prj/parPrj.c:29
constexpr double kParEps = 1e-8;        // prj/parPrj.h:8

static ParView par_view(double theta)
{
    ParView v;
    int whole = (int)(fmod(theta, 90) - 45);
    if (whole < 0) whole = -whole;
    const double tmp = whole * kParPi / 180;
    v.height = 1 / sin(tmp + kParPi / 4);
    v.b1 = sqrt(2.0) / 2 * sin(tmp);
    v.b2 = sqrt(2.0) / 2 * cos(tmp);
    v.areaT = 0.5 * v.height * (v.b2 - v.b1);
    v.areaR = v.height * v.b1 * 2;
    v.c = cos(theta * kParPi / 180);
    v.s = sin(theta * kParPi / 180);
    v.pad = 0;
    return v;
}

__device__ __forceinline__ double sq(double a) { return a * a; }

// overlap of the beam of detector k with the footprint centred at dist, by the
// zones of the beam's two edges (prj/parPrj.c:133-168)
__device__ __forceinline__ double par_overlap(const ParView &v, double dist, double k, double bw)
{
    const double hb = bw / 2, w = v.b2 - v.b1, H = v.height;
    const double ul = k - hb - dist, ur = k + hb - dist;
    const double aT = v.areaT, aR = v.areaR;
    if (ul <= -v.b2) {
        if (ur <= -v.b1) return aT * sq((ur + v.b2) / w);
        if (ur <= v.b1) return aT + H * (ur + v.b1);
        return aT * 2 + aR - aT * sq((v.b2 - ur) / w);
    }
    if (ul <= -v.b1) {
        const double rise = aT * (1 - sq((ul + v.b2) / w));
        if (ur <= -v.b1) return H / w * (k - dist + v.b2) * bw;
        if (ur <= v.b1) return rise + H * (ur + v.b1);
        if (ur <= v.b2) return rise + aR + aT * (1 - sq((v.b2 - ur) / w));
        return rise + aR + aT;
    }
    if (ul <= v.b1) {
        if (ur <= v.b1) return H * bw;
        if (ur <= v.b2) return H * (v.b1 - ul) + aT * (1 - sq((v.b2 - ur) / w));
        return H * (v.b1 - ul) + aT;
    }
    if (ur <= v.b2) return H / w * (dist + v.b2 - k) * bw;
    return 0.5 * H / w * sq(dist + v.b2 - k + hb);
}

constexpr int kParThreads = 256;

__global__ void __launch_bounds__(kParThreads)
k_par_forward(const ParArgs a, const double *__restrict__ x, const double *__restrict__ mask,
              long long npix, double *__restrict__ y)
{
    extern __shared__ double row[];
    const int it = blockIdx.x;
    for (int k = threadIdx.x; k < a.W; k += blockDim.x) row[k] = 0.0;
    __syncthreads();
    const ParView v = a.view[it];
    for (long long i = (long long)blockIdx.y * blockDim.x + threadIdx.x; i < npix;
         i += (long long)gridDim.y * blockDim.x) {
        const int m = (int)mask[i];
        const int px = m / a.nr - a.xC, py = m % a.nr - a.yC;
        const double dist = px * v.c + py * v.s;
        const double ub = floor(dist + v.b2 + a.bw / 2 - kParEps);
        const double lb = ceil(dist - v.b2 - a.bw / 2 + kParEps);
        const double xi = x[i];
        for (int k = (int)lb; k <= ub; ++k) {
            if (k < -a.pC || k + a.pC >= a.nc || k + a.pC >= a.W) continue;
            const double w = par_overlap(v, dist, (double)k, a.bw);
            if (w != 0.0) atomicAdd(&row[k + a.pC], w * xi);
        }
    }
    __syncthreads();
    double *out = y + (size_t)it * a.W;
    for (int k = threadIdx.x; k < a.W; k += blockDim.x)
        if (row[k] != 0.0) atomicAdd(&out[k], row[k]);
}

__global__ void __launch_bounds__(kParThreads)
k_par_backward(const ParArgs a, const double *__restrict__ y, const double *__restrict__ mask,
               long long npix, double *__restrict__ x)
{
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= npix) return;
    const int m = (int)mask[i];
    const int px = m / a.nr - a.xC, py = m % a.nr - a.yC;
    double acc = x[i];
    for (int it = 0; it < a.np; ++it) {
        const ParView &v = a.view[it];
        const double dist = px * v.c + py * v.s;
        const double ub = floor(dist + v.b2 + a.bw / 2 - kParEps);
        const double lb = ceil(dist - v.b2 - a.bw / 2 + kParEps);
        const double *rowp = y + (size_t)it * a.W;
        for (int k = (int)lb; k <= ub; ++k) {
            if (k < -a.pC || k + a.pC >= a.nc || k + a.pC >= a.W) continue;
            const double w = par_overlap(v, dist, (double)k, a.bw);
            if (w != 0.0) acc += rowp[k + a.pC] * w;
        }
    }
    x[i] = acc / a.bw;
}

__global__ void k_scale(double *__restrict__ v, long long n, double inv)
{
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x)
        v[i] /= inv;
}

static int par_validate(const ctprj_par_conf *c, long long npix)
{
    if (!c) return set_error(CTPRJ_EINVAL, "NULL configuration");
    if (c->nc < 1 || c->nr < 1 || c->np < 0 || c->prjWidth < 1 || npix < 0 || !(c->bw > 0))
        return set_error(CTPRJ_EINVAL, "invalid parPrj configuration");
    if ((long long)c->np * c->prjWidth >= (1LL << 31) || npix >= (1LL << 31))
        return set_error(CTPRJ_ERANGE, "parPrj sizes exceed 2^31");
    if ((size_t)c->prjWidth * sizeof(double) > 200 * 1024)
        return set_error(CTPRJ_ERANGE, "parPrj: prjWidth above %d", (int)(200 * 1024 / sizeof(double)));
    return CTPRJ_OK;
}

static ParArgs par_args(const ctprj_par_conf *c, const ParView *view)
{
    ParArgs a;
    a.bw = c->bw;
    a.nc = c->nc;
    a.nr = c->nr;
    a.np = c->np;
    a.W = c->prjWidth;
    a.xC = c->nc / 2;
    a.yC = c->nr / 2;
    a.pC = a.xC > a.yC ? a.xC : a.yC;
    a.view = view;
    return a;
}

// view table in stream-ordered device memory (released after the kernels)
static int par_table(const ctprj_par_conf *c, const double *theta, ParView **d_view, cudaStream_t s)
{
    std::vector<ParView> tab((size_t)(c->np > 0 ? c->np : 1));
    for (int it = 0; it < c->np; ++it) tab[it] = par_view(theta[it]);
    int st = cuda_error(cudaMallocAsync((void **)d_view, sizeof(ParView) * tab.size(), s),
                        "parPrj view table");
    if (st) return st;
    return cuda_error(cudaMemcpyAsync(*d_view, tab.data(), sizeof(ParView) * tab.size(),
                                      cudaMemcpyHostToDevice, s),
                      "parPrj view upload");
}

static int sm_count()
{
    int dev = 0, sms = 148;
    if (cudaGetDevice(&dev) == cudaSuccess)
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    return sms;
}

}  // namespace ctprj

using namespace ctprj;

extern "C" int ctprj_par_forward(const ctprj_par_conf *conf, const double *theta_host,
                                 const double *d_mask, long long npix, const double *d_x,
                                 double *d_y, void *stream)
{
    int st = par_validate(conf, npix);
    if (st) return st;
    if (conf->np > 0 && (!theta_host || !d_y)) return set_error(CTPRJ_EINVAL, "NULL buffer");
    if (npix > 0 && (!d_mask || !d_x)) return set_error(CTPRJ_EINVAL, "NULL buffer");
    cudaStream_t s = (cudaStream_t)stream;
    if (conf->np == 0) return CTPRJ_OK;
    ParView *d_view = nullptr;
    if ((st = par_table(conf, theta_host, &d_view, s))) return st;
    const ParArgs a = par_args(conf, d_view);
    const size_t smem = sizeof(double) * (size_t)conf->prjWidth;
    cudaFuncSetAttribute(k_par_forward, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    const long long per = (long long)kParThreads * 8;
    int chunks = (int)((npix + per - 1) / per);
    const int target = (4 * sm_count() + conf->np - 1) / conf->np;
    if (chunks > target) chunks = target;
    if (chunks < 1) chunks = 1;
    if (chunks > 65535) chunks = 65535;
    if (npix > 0) {
        k_par_forward<<<dim3(conf->np, chunks), kParThreads, smem, s>>>(a, d_x, d_mask, npix, d_y);
        if ((st = cuda_error(cudaGetLastError(), "parPrj forward"))) return st;
    }
    const long long ny = (long long)conf->np * conf->prjWidth;
    k_scale<<<4 * sm_count(), 256, 0, s>>>(d_y, ny, conf->bw);
    st = cuda_error(cudaGetLastError(), "parPrj scale");
    cudaFreeAsync(d_view, s);
    return st;
}

extern "C" int ctprj_par_backward(const ctprj_par_conf *conf, const double *theta_host,
                                  const double *d_mask, long long npix, const double *d_y,
                                  double *d_x, void *stream)
{
    int st = par_validate(conf, npix);
    if (st) return st;
    if (npix == 0) return CTPRJ_OK;
    if (!d_mask || !d_x || (conf->np > 0 && (!theta_host || !d_y)))
        return set_error(CTPRJ_EINVAL, "NULL buffer");
    cudaStream_t s = (cudaStream_t)stream;
    ParView *d_view = nullptr;
    if ((st = par_table(conf, theta_host, &d_view, s))) return st;
    const ParArgs a = par_args(conf, d_view);
    const int blocks = (int)((npix + kParThreads - 1) / kParThreads);
    k_par_backward<<<blocks, kParThreads, 0, s>>>(a, d_y, d_mask, npix, d_x);
    st = cuda_error(cudaGetLastError(), "parPrj backward");
    cudaFreeAsync(d_view, s);
    return st;
}

// ---------------------------------------------- prj/parPrj.h entry points

static std::mutex g_par_mu;
static double *g_img = nullptr, *g_prj = nullptr, *g_mask = nullptr;
static parConf g_opt;
static size_t g_tot = 0;
static bool g_conf_set = false;

extern "C" int parPrjConf(double *t_img, double *t_prj, double *t_maskIdx, parConf *t_opt,
                          size_t t_totPixels)
{
    std::lock_guard<std::mutex> lk(g_par_mu);
    g_img = t_img;
    g_prj = t_prj;
    g_mask = t_maskIdx;
    if (t_opt) g_opt = *t_opt;
    g_tot = t_totPixels;
    g_conf_set = t_opt != nullptr;
    return 0;
}

extern "C" int parPrjThread(void)
{
    std::lock_guard<std::mutex> lk(g_par_mu);
    if (!g_conf_set) return set_error(CTPRJ_ENOTSETUP, "parPrjConf() has not been called");
    const ctprj_par_conf c = {g_opt.bw, g_opt.nc, g_opt.nr, g_opt.np, g_opt.prjWidth};
    const long long npix = (long long)g_tot;
    int st = par_validate(&c, npix);
    if (st) return st;
    const size_t ny = (size_t)c.np * c.prjWidth;
    if ((npix > 0 && (!g_img || !g_mask)) || (ny > 0 && (!g_prj || !g_opt.theta)))
        return set_error(CTPRJ_EINVAL, "NULL buffer in the parPrj configuration");
    double *d_img = nullptr, *d_prj = nullptr, *d_mask = nullptr;
    cudaStream_t s = 0;
    if ((st = cuda_error(cudaMalloc((void **)&d_img, sizeof(double) * (npix ? npix : 1)), "parPrj buffers")) ||
        (st = cuda_error(cudaMalloc((void **)&d_prj, sizeof(double) * (ny ? ny : 1)), "parPrj buffers")) ||
        (st = cuda_error(cudaMalloc((void **)&d_mask, sizeof(double) * (npix ? npix : 1)), "parPrj buffers")))
        goto done;
    if ((npix && ((st = cuda_error(cudaMemcpy(d_img, g_img, sizeof(double) * npix, cudaMemcpyHostToDevice), "copy")) ||
                  (st = cuda_error(cudaMemcpy(d_mask, g_mask, sizeof(double) * npix, cudaMemcpyHostToDevice), "copy")))) ||
        (ny && (st = cuda_error(cudaMemcpy(d_prj, g_prj, sizeof(double) * ny, cudaMemcpyHostToDevice), "copy"))))
        goto done;
    if (g_opt.fwd) {
        if ((st = ctprj_par_forward(&c, g_opt.theta, d_mask, npix, d_img, d_prj, s))) goto done;
        if (ny) st = cuda_error(cudaMemcpy(g_prj, d_prj, sizeof(double) * ny, cudaMemcpyDeviceToHost), "copy back");
    } else {
        if ((st = ctprj_par_backward(&c, g_opt.theta, d_mask, npix, d_prj, d_img, s))) goto done;
        if (npix) st = cuda_error(cudaMemcpy(g_img, d_img, sizeof(double) * npix, cudaMemcpyDeviceToHost), "copy back");
    }
done:
    cudaFree(d_img);
    cudaFree(d_prj);
    cudaFree(d_mask);
    return st;
}

extern "C" int parPrjRun(void) { return parPrjThread(); }

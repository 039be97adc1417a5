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
//  forward   one thread per (angle, detector), gathering from a dense copy of
//            the masked image the pixels whose footprint reaches the detector.
//            Where the detector's band is closer to the rows than to the
//            columns (|sin| >= |cos|) they are taken column by column and row
//            by row -- increasing column-major index, the order in which the
//            reference sums a sorted mask -- otherwise row by row from a
//            row-major copy, so that the lanes of a warp (adjacent detectors)
//            always walk their bands in step.  No atomics: results repeat bit
//            for bit.
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
    double c, s, height, b1, b2, areaT, areaR;
    double inv_s, inv_c;   // 1 / s and 1 / c, 0 where zero
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
    v.inv_s = v.s != 0.0 ? 1.0 / v.s : 0.0;
    v.inv_c = v.c != 0.0 ? 1.0 / v.c : 0.0;
    return v;
}

__device__ __forceinline__ double sq(double a) { return a * a; }

// distance of pixel (px, py) from the central ray of angle v (prj/parPrj.c:123),
// one rounding order for both directions
__device__ __forceinline__ double par_dist(const ParView &v, int px, int py)
{
    return fma((double)py, v.s, (double)px * v.c);
}

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

// the masked pixel values in a dense nr x nc image, column-major (ximg) and
// row-major (ximgT), zero elsewhere.  A pixel listed twice in the mask holds
// the sum of its values; indices outside the image are not projected.
__global__ void k_par_scatter(const double *__restrict__ x, const double *__restrict__ mask,
                              long long npix, int nr, int nc, double *__restrict__ ximg,
                              double *__restrict__ ximgT)
{
    const long long nimg = (long long)nr * nc;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < npix;
         i += (long long)gridDim.x * blockDim.x) {
        const long long m = (long long)mask[i];
        if (m >= 0 && m < nimg) {
            atomicAdd(&ximg[m], x[i]);
            atomicAdd(&ximgT[(m % nr) * nc + m / nr], x[i]);
        }
    }
}

// y[it, kk] = (y[it, kk] + sum of w * x over the pixels that reach detector
// kk) / bw.  The rows a column can contribute are bracketed from
// |dist - k| <= b2 + bw/2 with a margin; each pixel then takes the reference's
// own detector range test (prj/parPrj.c:124-125) and weight.
__global__ void __launch_bounds__(kParThreads)
k_par_forward(const ParArgs a, const double *__restrict__ ximg, const double *__restrict__ ximgT,
              double *__restrict__ y)
{
    const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= (long long)a.np * a.W) return;
    const int it = (int)(e / a.W), kk = (int)(e % a.W);
    double acc = y[e];
    if (kk < a.nc) {   // detectors with k + centre >= nc are skipped (prj/parPrj.c:170)
        const ParView v = a.view[it];
        const double k = (double)(kk - a.pC);
        const double hw = v.b2 + a.bw / 2 + 1e-6;
        const double ylo = (double)-a.yC, yhi = (double)(a.nr - 1 - a.yC);
        const double xlo = (double)-a.xC, xhi = (double)(a.nc - 1 - a.xC);
        // the pixel's own range test and weight (prj/parPrj.c:124-125, :133-168)
        auto add = [&](int px, int py, double xv) {
            if (xv == 0.0) return;
            const double dist = par_dist(v, px, py);
            const double ub = floor(dist + v.b2 + a.bw / 2 - kParEps);
            const double lb = ceil(dist - v.b2 - a.bw / 2 + kParEps);
            if (k < lb || k > ub) return;
            const double w = par_overlap(v, dist, k, a.bw);
            if (w != 0.0) acc += w * xv;
        };
        if (fabs(v.s) < fabs(v.c)) {
            // the band is closer to the columns: row by row, a few columns each
            for (int ry = 0; ry < a.nr; ++ry) {
                const int py = ry - a.yC;
                const double ps = (double)py * v.s;
                double c0 = (k - hw - ps) * v.inv_c, c1 = (k + hw - ps) * v.inv_c;
                if (c0 > c1) { const double t = c0; c0 = c1; c1 = t; }
                const int px0 = (int)ceil(fmax(c0, xlo)), px1 = (int)floor(fmin(c1, xhi));
                const double *row = ximgT + (size_t)ry * a.nc + a.xC;
                for (int px = px0; px <= px1; ++px) add(px, py, row[px]);
            }
            y[e] = acc / a.bw;
            return;
        }
        for (int cx = 0; cx < a.nc; ++cx) {
            const int px = cx - a.xC;
            const double pc = (double)px * v.c;
            double r0, r1;
            if (v.inv_s != 0.0) {
                r0 = (k - hw - pc) * v.inv_s;
                r1 = (k + hw - pc) * v.inv_s;
                if (r0 > r1) { const double t = r0; r0 = r1; r1 = t; }
            } else if (fabs(pc - k) <= hw) {
                r0 = ylo;
                r1 = yhi;
            } else {
                continue;
            }
            const int py0 = (int)ceil(fmax(r0, ylo)), py1 = (int)floor(fmin(r1, yhi));
            const double *col = ximg + (size_t)cx * a.nr + a.yC;
            for (int py = py0; py <= py1; ++py) add(px, py, col[py]);
        }
    }
    y[e] = acc / a.bw;
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
        const double dist = par_dist(v, px, py);
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

static int par_validate(const ctprj_par_conf *c, long long npix)
{
    if (!c) return set_error(CTPRJ_EINVAL, "NULL configuration");
    if (c->nc < 1 || c->nr < 1 || c->np < 0 || c->prjWidth < 1 || npix < 0 || !(c->bw > 0))
        return set_error(CTPRJ_EINVAL, "invalid parPrj configuration");
    if ((long long)c->np * c->prjWidth >= (1LL << 31) || npix >= (1LL << 31) ||
        (long long)c->nc * c->nr >= (1LL << 31))
        return set_error(CTPRJ_ERANGE, "parPrj sizes exceed 2^31");
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
    double *d_img = nullptr;
    if ((st = par_table(conf, theta_host, &d_view, s))) return st;
    const ParArgs a = par_args(conf, d_view);
    const size_t img_elems = (size_t)conf->nc * (size_t)conf->nr, img_bytes = 2 * sizeof(double) * img_elems;
    if (!(st = cuda_error(cudaMallocAsync((void **)&d_img, img_bytes, s), "parPrj dense image")) &&
        !(st = cuda_error(cudaMemsetAsync(d_img, 0, img_bytes, s), "parPrj dense image"))) {
        if (npix > 0) {
            const long long blocks = (npix + kParThreads - 1) / kParThreads;
            k_par_scatter<<<(int)(blocks < 8 * sm_count() ? blocks : 8 * sm_count()), kParThreads, 0, s>>>(
                d_x, d_mask, npix, conf->nr, conf->nc, d_img, d_img + img_elems);
            st = cuda_error(cudaGetLastError(), "parPrj scatter");
        }
        if (!st) {
            const long long ny = (long long)conf->np * conf->prjWidth;
            k_par_forward<<<(int)((ny + kParThreads - 1) / kParThreads), kParThreads, 0, s>>>(
                a, d_img, d_img + img_elems, d_y);
            st = cuda_error(cudaGetLastError(), "parPrj forward");
        }
    }
    if (d_img) cudaFreeAsync(d_img, s);
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

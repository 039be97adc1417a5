// wavelet.cu -- the periodic orthogonal wavelet transform and the ADMM
// wavelet proximal map of the density step on the GPU.
//
// The transform is the reference's vendored Rice Wavelet Toolbox pair
// mdwt / midwt (rwt/mdwt_r.c, rwt/midwt_r.c): per level, on the top-left
// R x C block, every row and then every column is split into
//     lo[k] = sum_j h[j] x[(2k + j) mod N],   hi[k] = sum_j g[j] x[(2k + j) mod N],
// g[j] = (-1)^j h[lh-1-j], lowpass outputs first; the inverse is the exact
// adjoint (the filters are orthonormal).  Here one kernel launch does one
// level: a thread owns one quarter-block coordinate (k, l) and produces the
// four coefficients LL, LH, HL, HH there from the lh x lh input window
// (filtering along the row index of each window row first, as the reference
// does), or, inverting, the 2 x 2 output pixels from the lh/2 x lh/2 windows
// of the four quadrants.  Detail coefficients are final once their level is
// done and go straight to the coefficient array; the LL block goes to a
// ping-pong scratch buffer that the next level reads.
//
// The ADMM of npg/admm.m (the reference's 'wvltADMM' proximal map,
// bhc/beamhardenSpline.m:205-209) is fused into those passes: the inverse
// transform of s + nu ends in alpha = max((a + rho x) / (1 + rho), 0), and
// every final coefficient v of the forward transform of alpha updates
// s = soft(v - nu, u / rho), nu = nu + s - v in place, with the FP64 partial
// sums of |s - s_old|^2 and |s - v|^2.  A one-block kernel then advances the
// iteration's scalars (stopping rule, rho adaptation) on the device; s is
// double buffered by the parity of the device-side iteration counter, and the
// doubling / halving of nu that accompanies a rho change is applied as a
// factor when nu is next read.
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "ctprj_internal.h"
#include "../../include/ctprj_wavelet.h"

namespace ctprj {

constexpr int kWvThreadsX = 32, kWvThreadsY = 8, kWvThreads = kWvThreadsX * kWvThreadsY;

struct WFilter {
    float h[CTPRJ_WVLT_MAX_FILTER];   // scaling (lowpass) filter
    float g[CTPRJ_WVLT_MAX_FILTER];   // g[j] = (-1)^j h[lh-1-j]
    int lh;
};

struct AdmmState {
    double rho;       // penalty parameter of the coming iteration
    double nu_mul;    // factor on the stored nu for the coming iteration
    double tol;       // min(1e-3, rel_tol) * ||a||
    double dif, res;  // |s - s_old| and |s - Psit(alpha)| of the last iteration
    int iter;         // completed iterations
    int cnt;          // iterations since the last rho change
    int done;
    int max_itr;
    unsigned arrived; // blocks of the running fused iteration that have written their partials
};

enum { kEpiStore = 0, kEpiAdmm = 1, kEpiL1 = 2 };

struct AnaArgs {
    WFilter f;
    int R, C;                 // input block of this level
    const float *src;         // the block, row stride lds
    int lds;
    float *ll;                // LL destination (scratch) unless last
    int ldll;
    int last;                 // the LL is final: it belongs to the coefficient array
    float *y;                 // coefficient array (kEpiStore), row stride ldy
    int ldy;
    int epi;
    // kEpiAdmm
    const AdmmState *st;
    float *s0, *s1, *nu;
    double u;
    double *part;             // per-block partials of this level (2 per block)
    const unsigned char *cmask;   // coefficient mask (maskk): coefficients outside are zero; NULL: all
};

struct SynArgs {
    WFilter f;
    int R, C;                 // output block of this level
    const float *ll;          // LL (R/2 x C/2), row stride ldll, unless coarsest
    int ldll;
    int coarsest;             // the LL comes from the coefficient array
    const float *y0, *y1;     // coefficient array (ADMM: s buffers by parity), row stride ldy
    const float *nu;          // ADMM: + nu_mul * nu
    int ldy;
    const AdmmState *st;      // ADMM mode when non-null
    int final_pass;           // run even when st->done
    float *out;               // output block, row stride ldo
    int ldo;
    const float *a;           // ADMM: alpha = max((a + rho x) / (1 + rho), 0), stride ldo
    const unsigned char *pmask;   // ADMM: pixel mask, alpha = 0 outside; NULL: all pixels
};

// v mod n in [0, n): a long filter can reach several periods of a small block
__device__ __forceinline__ int wrap(int v, int n)
{
    const int r = v % n;
    return r < 0 ? r + n : r;
}

__device__ __forceinline__ void block_sum2(double a, double b, double *out)
{
    __shared__ double red[2][kWvThreads / 32];
    const int t = threadIdx.y * blockDim.x + threadIdx.x;
    for (int o = 16; o > 0; o >>= 1) {
        a += __shfl_down_sync(0xffffffffu, a, o);
        b += __shfl_down_sync(0xffffffffu, b, o);
    }
    if ((t & 31) == 0) {
        red[0][t >> 5] = a;
        red[1][t >> 5] = b;
    }
    __syncthreads();
    if (t == 0) {
        double x = 0.0, z = 0.0;
        for (int w = 0; w < kWvThreads / 32; ++w) {
            x += red[0][w];
            z += red[1][w];
        }
        out[0] = x;
        out[1] = z;
    }
}

// One analysis level.  Thread (k, l) of the (R/2) x (C/2) quarter grid.
__global__ void __launch_bounds__(kWvThreads) k_wvlt_analysis(const AnaArgs a)
{
    if (a.st && a.st->done) return;
    const int l = blockIdx.x * kWvThreadsX + threadIdx.x, k = blockIdx.y * kWvThreadsY + threadIdx.y;
    const int Rh = a.R >> 1, Ch = a.C >> 1;
    double p0 = 0.0, p1 = 0.0;
    if (k < Rh && l < Ch) {
        const int lh = a.f.lh;
        float ll = 0.0f, lhv = 0.0f, hl = 0.0f, hh = 0.0f;
        for (int i = 0; i < lh; ++i) {
            const float *row = a.src + (size_t)wrap(2 * k + i, a.R) * a.lds;
            float lo = 0.0f, hi = 0.0f;                 // along the row first
            for (int j = 0; j < lh; ++j) {
                const float v = row[wrap(2 * l + j, a.C)];
                lo = fmaf(a.f.h[j], v, lo);
                hi = fmaf(a.f.g[j], v, hi);
            }
            ll = fmaf(a.f.h[i], lo, ll);
            lhv = fmaf(a.f.h[i], hi, lhv);
            hl = fmaf(a.f.g[i], lo, hl);
            hh = fmaf(a.f.g[i], hi, hh);
        }
        // final coefficients: (row-lo, col-hi), (row-hi, col-lo), (row-hi,
        // col-hi), and the LL on the last level
        const float v[4] = {lhv, hl, hh, ll};
        const int pos[4] = {k * a.ldy + l + Ch, (k + Rh) * a.ldy + l, (k + Rh) * a.ldy + l + Ch, k * a.ldy + l};
        const int nfin = a.last ? 4 : 3;
        if (!a.last) a.ll[(size_t)k * a.ldll + l] = ll;
        const unsigned char *cm = a.cmask;
        if (a.epi == kEpiStore) {
            for (int q = 0; q < nfin; ++q) a.y[pos[q]] = (!cm || cm[pos[q]]) ? v[q] : 0.0f;
        } else if (a.epi == kEpiL1) {
            for (int q = 0; q < nfin; ++q)
                if (!cm || cm[pos[q]]) p0 += fabs((double)v[q]);
        } else {   // ADMM: s = soft(v - nu, u / rho), nu = nu + s - v
            const AdmmState *st = a.st;
            const int cur = st->iter & 1;
            const float *sold = cur ? a.s1 : a.s0;
            float *snew = cur ? a.s0 : a.s1;
            const float mul = (float)st->nu_mul, thr = (float)(a.u / st->rho);
            for (int q = 0; q < nfin; ++q) {
                const int p = pos[q];
                if (cm && !cm[p]) {   // not a coefficient of the masked transform
                    a.nu[p] = 0.0f;
                    snew[p] = 0.0f;
                    continue;
                }
                const float nue = mul * a.nu[p];
                const float w = v[q] - nue;
                const float sn = w > thr ? w - thr : (w < -thr ? w + thr : 0.0f);
                a.nu[p] = nue + sn - v[q];
                snew[p] = sn;
                const double d = (double)sn - (double)sold[p], r = (double)sn - (double)v[q];
                p0 = fma(d, d, p0);
                p1 = fma(r, r, p1);
            }
        }
    }
    if (a.epi == kEpiStore) return;   // uniform per launch: no partials
    double out[2];
    block_sum2(p0, p1, out);
    if (threadIdx.x == 0 && threadIdx.y == 0) {
        const size_t b = (size_t)blockIdx.y * gridDim.x + blockIdx.x;
        a.part[2 * b] = out[0];
        a.part[2 * b + 1] = out[1];
    }
}

// One synthesis level.  Thread (k, l) of the (R/2) x (C/2) quarter grid
// writes output pixels (2k + e, 2l + f), e, f in {0, 1}.
__global__ void __launch_bounds__(kWvThreads) k_wvlt_synthesis(const SynArgs a)
{
    const AdmmState *st = a.st;
    if (st && !a.final_pass && st->done) return;
    const int l = blockIdx.x * kWvThreadsX + threadIdx.x, k = blockIdx.y * kWvThreadsY + threadIdx.y;
    const int Rh = a.R >> 1, Ch = a.C >> 1;
    if (k >= Rh || l >= Ch) return;
    const float *Y = (st && (st->iter & 1)) ? a.y1 : a.y0;
    const float mul = st ? (float)st->nu_mul : 0.0f;
    auto coef = [&](int kk, int ll, int qr, int qc) -> float {
        if (qr == 0 && qc == 0 && !a.coarsest) return a.ll[(size_t)kk * a.ldll + ll];
        const int p = (kk + qr * Rh) * a.ldy + ll + qc * Ch;
        float v = Y[p];
        if (a.nu) v = fmaf(mul, a.nu[p], v);
        return v;
    };
    const int half = a.f.lh >> 1;
    float x[2][2] = {{0.0f, 0.0f}, {0.0f, 0.0f}};
    for (int q = 0; q < half; ++q) {
        const int lq = wrap(l - q, Ch);
        float ulo[2] = {0.0f, 0.0f}, uhi[2] = {0.0f, 0.0f};
        for (int p = 0; p < half; ++p) {   // along the row index first, as midwt
            const int kp = wrap(k - p, Rh);
            const float c00 = coef(kp, lq, 0, 0), c01 = coef(kp, lq, 0, 1);
            const float c10 = coef(kp, lq, 1, 0), c11 = coef(kp, lq, 1, 1);
#pragma unroll
            for (int e = 0; e < 2; ++e) {
                const float he = a.f.h[e + 2 * p], ge = a.f.g[e + 2 * p];
                ulo[e] = fmaf(he, c00, fmaf(ge, c10, ulo[e]));
                uhi[e] = fmaf(he, c01, fmaf(ge, c11, uhi[e]));
            }
        }
#pragma unroll
        for (int e = 0; e < 2; ++e)
#pragma unroll
            for (int f = 0; f < 2; ++f)
                x[e][f] = fmaf(a.f.h[f + 2 * q], ulo[e], fmaf(a.f.g[f + 2 * q], uhi[e], x[e][f]));
    }
    const float rho = st ? (float)st->rho : 0.0f;
#pragma unroll
    for (int e = 0; e < 2; ++e)
#pragma unroll
        for (int f = 0; f < 2; ++f) {
            const size_t o = (size_t)(2 * k + e) * a.ldo + 2 * l + f;
            float v = x[e][f];
            if (a.a) v = (a.pmask && !a.pmask[o]) ? 0.0f : fmaxf(fmaf(rho, v, a.a[o]) / (1.0f + rho), 0.0f);
            a.out[o] = v;
        }
}

// the iteration's scalars (npg/admm.m's loop tail) from the sums of
// |s - s_old|^2 and |s - Psit(alpha)|^2: the stopping rule, then the rho
// adaptation after more than 20 iterations without one
__device__ void admm_advance(AdmmState *st, double dif2, double res2)
{
    const double dif = sqrt(dif2), res = sqrt(res2);
    st->dif = dif;
    st->res = res;
    st->iter += 1;
    st->cnt += 1;
    st->nu_mul = 1.0;   // the stored nu is current again
    if (st->iter > st->max_itr || (dif <= st->tol && res <= st->tol)) {
        st->done = 1;
        return;
    }
    if (st->cnt > 20) {
        if (dif > 10.0 * res) {
            st->rho *= 0.5;
            st->nu_mul = 2.0;
            st->cnt = 0;
        } else if (dif < res / 10.0) {
            st->rho *= 2.0;
            st->nu_mul = 0.5;
            st->cnt = 0;
        }
    }
}

__global__ void __launch_bounds__(256) k_admm_scalars(AdmmState *st, const double *__restrict__ part, int nblocks)
{
    __shared__ double red[2][256];
    if (st->done) return;
    double s0 = 0.0, s1 = 0.0;
    for (int b = threadIdx.x; b < nblocks; b += 256) {
        s0 += part[2 * (size_t)b];
        s1 += part[2 * (size_t)b + 1];
    }
    red[0][threadIdx.x] = s0;
    red[1][threadIdx.x] = s1;
    __syncthreads();
    for (int h = 128; h > 0; h >>= 1) {
        if ((int)threadIdx.x < h) {
            red[0][threadIdx.x] += red[0][threadIdx.x + h];
            red[1][threadIdx.x] += red[1][threadIdx.x + h];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) admm_advance(st, red[0][0], red[1][0]);
}

__global__ void k_admm_start(AdmmState *st, double tol, int max_itr)
{
    st->rho = 1.0;
    st->nu_mul = 1.0;
    st->tol = tol;
    st->dif = st->res = 0.0;
    st->iter = 0;
    st->cnt = 0;
    st->done = 0;
    st->max_itr = max_itr;
    st->arrived = 0;
}

// ---- two-tap filters: one fused launch per ADMM iteration ----------------
// With a 2-tap filter every level reads only its own 2 x 2 input cells, so a
// 2^L x 2^L image tile holds every coefficient of all L levels that it
// touches and needs nothing from its neighbours.  One block per tile then
// does a whole iteration in shared memory: gather s + nu_mul nu from the
// tile's coefficient positions (Mallat order inside the tile), the inverse
// transform coarsest level first, alpha = max((a + rho x) / (1 + rho), 0),
// the forward transform finest level first, and the ADMM update written back
// to the same positions -- 20 bytes per pixel (s, nu, a in; s, nu out) and no
// alpha image.  Each level works in place: a thread reads its cells into
// registers, the block synchronises, then writes.  The arithmetic is the
// level kernels' operation for operation; only the FP64 partial sums are
// added in another order.  The last block to finish sums every tile's
// partials in a fixed order and advances the scalars.
constexpr int kHaarMaxLevels = 6;
constexpr int kHaarThreads = 256;

struct HaarArgs {
    float h0, h1, g0, g1;
    int rows, cols;
    const float *a;
    float *s0, *s1, *nu;
    float *alpha;             // the final pass writes alpha here
    AdmmState *st;
    double u;
    double *part;             // per-tile partials, 2 each
    int final_pass;
    const unsigned char *pmask, *cmask;   // pixel and coefficient masks, or NULL
};

// coefficient-array index of tile-layout cell (r, c) of tile (ti, tj)
template <int L>
__device__ __forceinline__ int haar_coef_index(int r, int c, int ti, int tj, int rows, int cols)
{
    const int m = r | c;   // its highest bit is that of max(r, c)
    int lev = L, Tl = 1, qr = 0, qc = 0;
    if (m) {
        const int b = 31 - __clz(m);
        Tl = 1 << b;
        lev = L - b;
        qr = r >= Tl;
        qc = c >= Tl;
    }
    const int grow = ti * Tl + (r - qr * Tl) + qr * (rows >> lev);
    const int gcol = tj * Tl + (c - qc * Tl) + qc * (cols >> lev);
    return grow * cols + gcol;
}

template <int L>
__global__ void __launch_bounds__(kHaarThreads) k_admm_haar(const HaarArgs a)
{
    constexpr int T = 1 << L, P = T + 1;
    constexpr int kItems = ((T / 2) * (T / 2) + kHaarThreads - 1) / kHaarThreads;
    extern __shared__ float sm[];
    float *W = sm;              // working tile, T x P
    float *Sv = sm + T * P;     // s_old, tile layout
    float *Nv = Sv + T * T;     // stored nu, tile layout
    __shared__ bool last;
    AdmmState *st = a.st;
    if (!a.final_pass && st->done) return;
    const int t = threadIdx.x, ti = blockIdx.y, tj = blockIdx.x;
    const int cur = st->iter & 1;
    const float *Sc = cur ? a.s1 : a.s0;
    float *Sn = cur ? a.s0 : a.s1;
    const float mul = (float)st->nu_mul, rho = (float)st->rho, thr = (float)(a.u / st->rho);
    const float h0 = a.h0, h1 = a.h1, g0 = a.g0, g1 = a.g1;
    for (int idx = t; idx < T * T; idx += kHaarThreads) {
        const int r = idx >> L, c = idx & (T - 1);
        const int gp = haar_coef_index<L>(r, c, ti, tj, a.rows, a.cols);
        const float sv = Sc[gp], nv = a.nu[gp];
        W[r * P + c] = fmaf(mul, nv, sv);
        Sv[idx] = sv;
        Nv[idx] = nv;
    }
    __syncthreads();
    // inverse transform, coarsest level first (unrolled: the block sides are
    // compile-time powers of two)
#pragma unroll
    for (int lev = L; lev >= 1; --lev) {
        const int Tl = T >> lev, n = Tl * Tl;
        float c00[kItems], c01[kItems], c10[kItems], c11[kItems];
#pragma unroll
        for (int it = 0; it < kItems; ++it) {
            const int q = t + it * kHaarThreads;
            if (q < n) {
                const int kk = q / Tl, ll = q % Tl;
                c00[it] = W[kk * P + ll];
                c01[it] = W[kk * P + ll + Tl];
                c10[it] = W[(kk + Tl) * P + ll];
                c11[it] = W[(kk + Tl) * P + ll + Tl];
            }
        }
        __syncthreads();
#pragma unroll
        for (int it = 0; it < kItems; ++it) {
            const int q = t + it * kHaarThreads;
            if (q < n) {
                const int kk = q / Tl, ll = q % Tl;
#pragma unroll
                for (int e = 0; e < 2; ++e) {
                    const float he = e ? h1 : h0, ge = e ? g1 : g0;
                    const float ulo = fmaf(he, c00[it], fmaf(ge, c10[it], 0.0f));
                    const float uhi = fmaf(he, c01[it], fmaf(ge, c11[it], 0.0f));
                    W[(2 * kk + e) * P + 2 * ll] = fmaf(h0, ulo, fmaf(g0, uhi, 0.0f));
                    W[(2 * kk + e) * P + 2 * ll + 1] = fmaf(h1, ulo, fmaf(g1, uhi, 0.0f));
                }
            }
        }
        __syncthreads();
    }
    // alpha = max((a + rho x) / (1 + rho), 0)
    for (int idx = t; idx < T * T; idx += kHaarThreads) {
        const int r = idx >> L, c = idx & (T - 1);
        const size_t gpix = (size_t)(ti * T + r) * a.cols + tj * T + c;
        const float v = (a.pmask && !a.pmask[gpix]) ? 0.0f
                                                    : fmaxf(fmaf(rho, W[r * P + c], a.a[gpix]) / (1.0f + rho), 0.0f);
        if (a.final_pass)
            a.alpha[gpix] = v;
        else
            W[r * P + c] = v;
    }
    if (a.final_pass) return;
    __syncthreads();
    // forward transform, finest level first
#pragma unroll
    for (int lev = 1; lev <= L; ++lev) {
        const int Tl = T >> lev, n = Tl * Tl;
        float x00[kItems], x01[kItems], x10[kItems], x11[kItems];
#pragma unroll
        for (int it = 0; it < kItems; ++it) {
            const int q = t + it * kHaarThreads;
            if (q < n) {
                const int kk = q / Tl, ll = q % Tl;
                x00[it] = W[2 * kk * P + 2 * ll];
                x01[it] = W[2 * kk * P + 2 * ll + 1];
                x10[it] = W[(2 * kk + 1) * P + 2 * ll];
                x11[it] = W[(2 * kk + 1) * P + 2 * ll + 1];
            }
        }
        __syncthreads();
#pragma unroll
        for (int it = 0; it < kItems; ++it) {
            const int q = t + it * kHaarThreads;
            if (q < n) {
                const int kk = q / Tl, ll = q % Tl;
                const float lo0 = fmaf(h1, x01[it], fmaf(h0, x00[it], 0.0f));
                const float hi0 = fmaf(g1, x01[it], fmaf(g0, x00[it], 0.0f));
                const float lo1 = fmaf(h1, x11[it], fmaf(h0, x10[it], 0.0f));
                const float hi1 = fmaf(g1, x11[it], fmaf(g0, x10[it], 0.0f));
                W[kk * P + ll] = fmaf(h1, lo1, fmaf(h0, lo0, 0.0f));
                W[kk * P + ll + Tl] = fmaf(h1, hi1, fmaf(h0, hi0, 0.0f));
                W[(kk + Tl) * P + ll] = fmaf(g1, lo1, fmaf(g0, lo0, 0.0f));
                W[(kk + Tl) * P + ll + Tl] = fmaf(g1, hi1, fmaf(g0, hi0, 0.0f));
            }
        }
        __syncthreads();
    }
    // s = soft(v - nu, u / rho), nu = nu + s - v at every coefficient of the tile
    double p0 = 0.0, p1 = 0.0;
    for (int idx = t; idx < T * T; idx += kHaarThreads) {
        const int r = idx >> L, c = idx & (T - 1);
        const int gp = haar_coef_index<L>(r, c, ti, tj, a.rows, a.cols);
        if (a.cmask && !a.cmask[gp]) {   // not a coefficient of the masked transform
            a.nu[gp] = 0.0f;
            Sn[gp] = 0.0f;
            continue;
        }
        const float v = W[r * P + c];
        const float nue = mul * Nv[idx];
        const float w = v - nue;
        const float sn = w > thr ? w - thr : (w < -thr ? w + thr : 0.0f);
        a.nu[gp] = nue + sn - v;
        Sn[gp] = sn;
        const double d = (double)sn - (double)Sv[idx], rr = (double)sn - (double)v;
        p0 = fma(d, d, p0);
        p1 = fma(rr, rr, p1);
    }
    double out[2];
    block_sum2(p0, p1, out);
    const unsigned nblocks = gridDim.x * gridDim.y;
    if (t == 0) {
        const size_t b = (size_t)blockIdx.y * gridDim.x + blockIdx.x;
        a.part[2 * b] = out[0];
        a.part[2 * b + 1] = out[1];
        __threadfence();
        last = atomicAdd(&st->arrived, 1u) == nblocks - 1;
    }
    __syncthreads();
    if (!last) return;
    // the last block: every tile's partials in a fixed order, then the scalars
    __threadfence();
    __shared__ double red[2][kHaarThreads];
    double q0 = 0.0, q1 = 0.0;
    for (unsigned b = t; b < nblocks; b += kHaarThreads) {
        q0 += __ldcg(a.part + 2 * (size_t)b);
        q1 += __ldcg(a.part + 2 * (size_t)b + 1);
    }
    red[0][t] = q0;
    red[1][t] = q1;
    __syncthreads();
    for (int h = kHaarThreads / 2; h > 0; h >>= 1) {
        if (t < h) {
            red[0][t] += red[0][t + h];
            red[1][t] += red[1][t + h];
        }
        __syncthreads();
    }
    if (t == 0) {
        admm_advance(st, red[0][0], red[1][0]);
        st->arrived = 0;
    }
}

template <int L>
int launch_admm_haar_t(const HaarArgs &a, cudaStream_t s)
{
    constexpr int T = 1 << L;
    const size_t smem = sizeof(float) * ((size_t)T * (T + 1) + 2 * (size_t)T * T);
    int st;
    if ((st = cuda_error(cudaFuncSetAttribute(k_admm_haar<L>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem),
                         "ADMM shared memory")))
        return st;
    const dim3 grid((unsigned)(a.cols / T), (unsigned)(a.rows / T));
    k_admm_haar<L><<<grid, kHaarThreads, smem, s>>>(a);
    return cuda_error(cudaGetLastError(), "ADMM iteration");
}

int launch_admm_haar(int levels, const HaarArgs &a, cudaStream_t s)
{
    switch (levels) {
    case 1: return launch_admm_haar_t<1>(a, s);
    case 2: return launch_admm_haar_t<2>(a, s);
    case 3: return launch_admm_haar_t<3>(a, s);
    case 4: return launch_admm_haar_t<4>(a, s);
    case 5: return launch_admm_haar_t<5>(a, s);
    case 6: return launch_admm_haar_t<6>(a, s);
    default: return set_error(CTPRJ_EINVAL, "fused ADMM: at most %d levels", kHaarMaxLevels);
    }
}

__global__ void __launch_bounds__(256) k_wvlt_sumsq(const float *__restrict__ x, long long n, double *__restrict__ part)
{
    __shared__ double red[8];
    double s = 0.0;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        s = fma((double)x[i], (double)x[i], s);
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int w = 0; w < 8; ++w) t += red[w];
        part[blockIdx.x] = t;
    }
}

__global__ void k_wvlt_sum(const double *__restrict__ part, int nrows, int stride, double *__restrict__ out)
{
    sum_partials(part, nrows, stride, 1, out);
}

namespace {

dim3 level_grid(int R, int C)
{
    return dim3((unsigned)(((C >> 1) + kWvThreadsX - 1) / kWvThreadsX), (unsigned)(((R >> 1) + kWvThreadsY - 1) / kWvThreadsY));
}

int check_args(const void *p, const void *q, int rows, int cols, const double *h, int lh, int levels, WFilter *f)
{
    if (!p || !q || !h) return set_error(CTPRJ_EINVAL, "NULL argument");
    if (lh < 2 || lh > CTPRJ_WVLT_MAX_FILTER || (lh & 1))
        return set_error(CTPRJ_EINVAL, "filter length %d: even, 2 .. %d", lh, CTPRJ_WVLT_MAX_FILTER);
    if (levels < 1 || levels > 30) return set_error(CTPRJ_EINVAL, "levels must be 1 .. 30");
    if (rows < 2 || cols < 2 || (long long)rows * cols >= (1LL << 31))
        return set_error(CTPRJ_EINVAL, "image of 2 x 2 to 2^31 pixels");
    if ((rows % (1 << levels)) || (cols % (1 << levels)))
        return set_error(CTPRJ_EINVAL, "rows and cols must be divisible by 2^levels");
    for (int j = 0; j < lh; ++j) {
        f->h[j] = (float)h[j];
        f->g[j] = (float)((j & 1) ? -h[lh - 1 - j] : h[lh - 1 - j]);
    }
    for (int j = lh; j < CTPRJ_WVLT_MAX_FILTER; ++j) f->h[j] = f->g[j] = 0.0f;
    f->lh = lh;
    return CTPRJ_OK;
}

// total analysis blocks over the levels (partials carry 2 doubles each)
int analysis_blocks(int rows, int cols, int levels)
{
    int total = 0;
    for (int lev = 0; lev < levels; ++lev) {
        const dim3 g = level_grid(rows >> lev, cols >> lev);
        total += (int)(g.x * g.y);
    }
    return total;
}

// forward transform of src into the coefficient array (kEpiStore), or its
// final coefficients into an epilogue (kEpiAdmm, kEpiL1)
int run_analysis(const WFilter &f, const float *src, int rows, int cols, int levels, float *scratch, int epi,
                 float *y, const AdmmState *st, float *s0, float *s1, float *nu, double u, double *part,
                 cudaStream_t s, const unsigned char *cmask = nullptr)
{
    const size_t quarter = (size_t)(rows / 2) * (cols / 2);
    const float *in = src;
    int lds = cols, pbase = 0;
    for (int lev = 0; lev < levels; ++lev) {
        const int R = rows >> lev, C = cols >> lev;
        AnaArgs a;
        a.f = f;
        a.R = R;
        a.C = C;
        a.src = in;
        a.lds = lds;
        a.last = lev == levels - 1;
        a.ll = scratch + (lev & 1) * quarter;
        a.ldll = C / 2;
        a.y = y;
        a.ldy = cols;
        a.epi = epi;
        a.st = st;
        a.s0 = s0;
        a.s1 = s1;
        a.nu = nu;
        a.u = u;
        a.part = part ? part + 2 * (size_t)pbase : nullptr;
        a.cmask = cmask;
        const dim3 g = level_grid(R, C);
        k_wvlt_analysis<<<g, dim3(kWvThreadsX, kWvThreadsY), 0, s>>>(a);
        pbase += (int)(g.x * g.y);
        in = a.ll;
        lds = a.ldll;
    }
    return cuda_error(cudaGetLastError(), "wavelet analysis");
}

// inverse transform of the coefficients (y0/y1 by parity, + nu) into out,
// with the ADMM epilogue when a is given
int run_synthesis(const WFilter &f, const float *y0, const float *y1, const float *nu, int rows, int cols,
                  int levels, float *scratch, const AdmmState *st, int final_pass, const float *a, float *out,
                  cudaStream_t s, const unsigned char *pmask = nullptr)
{
    const size_t quarter = (size_t)(rows / 2) * (cols / 2);
    const float *ll = nullptr;
    int ldll = 0;
    for (int lev = levels - 1; lev >= 0; --lev) {
        const int R = rows >> lev, C = cols >> lev;
        SynArgs g;
        g.f = f;
        g.R = R;
        g.C = C;
        g.coarsest = lev == levels - 1;
        g.ll = ll;
        g.ldll = ldll;
        g.y0 = y0;
        g.y1 = y1;
        g.nu = nu;
        g.ldy = cols;
        g.st = st;
        g.final_pass = final_pass;
        g.pmask = pmask;
        if (lev == 0) {
            g.out = out;
            g.ldo = cols;
            g.a = a;
        } else {
            g.out = scratch + (lev & 1) * quarter;
            g.ldo = C;
            g.a = nullptr;
        }
        k_wvlt_synthesis<<<level_grid(R, C), dim3(kWvThreadsX, kWvThreadsY), 0, s>>>(g);
        ll = g.out;
        ldll = C;
    }
    return cuda_error(cudaGetLastError(), "wavelet synthesis");
}

}  // namespace

// ---- the loop's use (bhc_loop.cu) ---------------------------------------
int WvltProx::alloc(int m, int n, cudaStream_t s)
{
    if (buf && rows == m && cols == n) return CTPRJ_OK;
    release(s);
    const size_t px = (size_t)m * n;
    int lmax = 0;   // the most levels these dimensions allow
    while (lmax < 30 && m % (2 << lmax) == 0 && n % (2 << lmax) == 0) ++lmax;
    const size_t nparts = 2 * (size_t)analysis_blocks(m, n, lmax > 0 ? lmax : 1) + 512;
    int st;
    if ((st = cuda_error(cudaMallocAsync((void **)&buf, sizeof(float) * (px / 2 + 3 * px), s), "wavelet buffers")) ||
        (st = cuda_error(cudaMallocAsync((void **)&part, sizeof(double) * nparts, s), "wavelet partials")) ||
        (st = cuda_error(cudaMallocAsync(&state, sizeof(AdmmState), s), "wavelet state"))) {
        release(s);
        return st;
    }
    rows = m;
    cols = n;
    return CTPRJ_OK;
}

void WvltProx::release(cudaStream_t s)
{
    if (buf) cudaFreeAsync(buf, s);
    if (part) cudaFreeAsync(part, s);
    if (state) cudaFreeAsync(state, s);
    buf = nullptr;
    part = nullptr;
    state = nullptr;
    rows = cols = 0;
}

int wvlt_admm(WvltProx &ws, const float *a, int rows, int cols, const double *h, int lh, int levels, double u,
              double rel_tol, int max_itr, const float *init, float *alpha, int *iterations, cudaStream_t s,
              const unsigned char *pmask, const unsigned char *cmask)
{
    WFilter f;
    int st;
    if ((st = check_args(a, alpha, rows, cols, h, lh, levels, &f))) return st;
    if ((st = ws.alloc(rows, cols, s))) return st;
    const size_t px = (size_t)rows * cols;
    float *scratch = ws.buf, *s0 = ws.buf + px / 2, *s1 = s0 + px, *nu = s1 + px;
    AdmmState *dst = (AdmmState *)ws.state;
    // scale = ||a|| (the reference works on a / scale; here on a, with the
    // tolerance scaled instead)
    const int sb = 256;
    k_wvlt_sumsq<<<sb, 256, 0, s>>>(a, (long long)px, ws.part);
    k_wvlt_sum<<<1, 256, 0, s>>>(ws.part, sb, 1, ws.part + sb);
    double ss = 0.0;
    if ((st = cuda_error(cudaMemcpyAsync(&ss, ws.part + sb, sizeof ss, cudaMemcpyDeviceToHost, s), "wavelet scale")) ||
        (st = cuda_error(cudaStreamSynchronize(s), "wavelet scale")))
        return st;
    const double scale = sqrt(ss);
    if (scale == 0.0) {
        if (iterations) *iterations = 0;
        return cuda_error(cudaMemsetAsync(alpha, 0, sizeof(float) * px, s), "wavelet result");
    }
    const double tol = fmin(1e-3, rel_tol) * scale;
    // s = Psit(init), nu = 0, rho = 1
    if ((st = run_analysis(f, init ? init : a, rows, cols, levels, scratch, kEpiStore, s0, nullptr, nullptr,
                           nullptr, nullptr, 0.0, nullptr, s, cmask)) ||
        (st = cuda_error(cudaMemsetAsync(nu, 0, sizeof(float) * px, s), "wavelet start")))
        return st;
    k_admm_start<<<1, 1, 0, s>>>(dst, tol, max_itr);
    const int nblocks = analysis_blocks(rows, cols, levels);
    // two-tap filters up to kHaarMaxLevels levels: the fused per-tile iteration
    // (CTPRJ_WVLT_KERNEL=levels keeps the level-by-level passes, for comparison)
    const char *kenv = getenv("CTPRJ_WVLT_KERNEL");
    const bool fused = lh == 2 && levels <= kHaarMaxLevels && !(kenv && !strcmp(kenv, "levels"));
    HaarArgs ha;
    ha.h0 = f.h[0];
    ha.h1 = f.h[1];
    ha.g0 = f.g[0];
    ha.g1 = f.g[1];
    ha.rows = rows;
    ha.cols = cols;
    ha.a = a;
    ha.s0 = s0;
    ha.s1 = s1;
    ha.nu = nu;
    ha.alpha = alpha;
    ha.st = dst;
    ha.u = u;
    ha.part = ws.part;
    ha.final_pass = 0;
    ha.pmask = pmask;
    ha.cmask = cmask;
    AdmmState h_st{};
    for (int it = 0; it <= max_itr + 1; ++it) {
        if (fused) {
            if ((st = launch_admm_haar(levels, ha, s))) return st;
        } else {
            if ((st = run_synthesis(f, s0, s1, nu, rows, cols, levels, scratch, dst, 0, a, alpha, s, pmask)) ||
                (st = run_analysis(f, alpha, rows, cols, levels, scratch, kEpiAdmm, nullptr, dst, s0, s1, nu, u,
                                   ws.part, s, cmask)))
                return st;
            k_admm_scalars<<<1, 256, 0, s>>>(dst, ws.part, nblocks);
        }
        if ((st = cuda_error(cudaGetLastError(), "ADMM iteration"))) return st;
        if ((it & 7) == 7) {
            if ((st = cuda_error(cudaMemcpyAsync(&h_st, dst, sizeof h_st, cudaMemcpyDeviceToHost, s), "ADMM state")) ||
                (st = cuda_error(cudaStreamSynchronize(s), "ADMM state")))
                return st;
            if (h_st.done) break;
        }
    }
    // alpha = max((a + rho Psi(s + nu)) / (1 + rho), 0) from the last s, nu
    ha.final_pass = 1;
    if ((st = fused ? launch_admm_haar(levels, ha, s)
                    : run_synthesis(f, s0, s1, nu, rows, cols, levels, scratch, dst, 1, a, alpha, s, pmask)) ||
        (st = cuda_error(cudaMemcpyAsync(&h_st, dst, sizeof h_st, cudaMemcpyDeviceToHost, s), "ADMM state")) ||
        (st = cuda_error(cudaStreamSynchronize(s), "ADMM state")))
        return st;
    if (!h_st.done) return set_error(CTPRJ_ECUDA, "ADMM did not reach its stopping rule");
    if (iterations) *iterations = h_st.iter;
    return CTPRJ_OK;
}

int wvlt_l1(WvltProx &ws, const float *x, int rows, int cols, const double *h, int lh, int levels, double *d_out,
            cudaStream_t s, const unsigned char *cmask)
{
    WFilter f;
    int st;
    if ((st = check_args(x, d_out, rows, cols, h, lh, levels, &f))) return st;
    if ((st = ws.alloc(rows, cols, s))) return st;
    if ((st = run_analysis(f, x, rows, cols, levels, ws.buf, kEpiL1, nullptr, nullptr, nullptr, nullptr, nullptr, 0.0,
                           ws.part, s, cmask)))
        return st;
    k_wvlt_sum<<<1, 256, 0, s>>>(ws.part, analysis_blocks(rows, cols, levels), 2, d_out);
    return cuda_error(cudaGetLastError(), "wavelet l1");
}

// coefficients that any pixel of the mask reaches (utils/wvltMask.m builds
// the same set as the union of Wt(e_i) != 0 over the mask's pixels e_i): the
// forward transform of the mask with the filters' magnitudes, whose sums of
// non-negative terms are positive exactly there
__global__ void k_mask_to_float(const unsigned char *__restrict__ m, long long n, float *__restrict__ out)
{
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        out[i] = m[i] ? 1.0f : 0.0f;
}
__global__ void k_float_to_mask(const float *__restrict__ v, long long n, unsigned char *__restrict__ out)
{
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        out[i] = v[i] > 0.0f ? 1 : 0;
}

int wvlt_mask(WvltProx &ws, const unsigned char *pmask, int rows, int cols, const double *h, int lh, int levels,
              unsigned char *cmask, cudaStream_t s)
{
    WFilter f;
    int st;
    if ((st = check_args(pmask, cmask, rows, cols, h, lh, levels, &f))) return st;
    for (int j = 0; j < lh; ++j) {
        f.h[j] = fabsf(f.h[j]);
        f.g[j] = fabsf(f.g[j]);
    }
    if ((st = ws.alloc(rows, cols, s))) return st;
    const size_t px = (size_t)rows * cols;
    float *scratch = ws.buf, *mimg = ws.buf + px / 2, *coef = mimg + px;
    k_mask_to_float<<<1024, 256, 0, s>>>(pmask, (long long)px, mimg);
    if ((st = run_analysis(f, mimg, rows, cols, levels, scratch, kEpiStore, coef, nullptr, nullptr, nullptr, nullptr,
                           0.0, nullptr, s)))
        return st;
    k_float_to_mask<<<1024, 256, 0, s>>>(coef, (long long)px, cmask);
    return cuda_error(cudaGetLastError(), "wavelet mask");
}

}  // namespace ctprj

using namespace ctprj;

extern "C" int ctprj_dwt(const float *d_x, int rows, int cols, const double *h, int lh, int levels, float *d_y,
                         void *stream)
{
    WFilter f;
    int st;
    if ((st = check_args(d_x, d_y, rows, cols, h, lh, levels, &f))) return st;
    cudaStream_t s = (cudaStream_t)stream;
    float *scratch = nullptr;
    if ((st = cuda_error(cudaMallocAsync((void **)&scratch, sizeof(float) * ((size_t)rows * cols / 2), s),
                         "wavelet scratch")))
        return st;
    st = run_analysis(f, d_x, rows, cols, levels, scratch, kEpiStore, d_y, nullptr, nullptr, nullptr, nullptr, 0.0,
                      nullptr, s);
    cudaFreeAsync(scratch, s);
    return st;
}

extern "C" int ctprj_idwt(const float *d_y, int rows, int cols, const double *h, int lh, int levels, float *d_x,
                          void *stream)
{
    WFilter f;
    int st;
    if ((st = check_args(d_y, d_x, rows, cols, h, lh, levels, &f))) return st;
    cudaStream_t s = (cudaStream_t)stream;
    float *scratch = nullptr;
    if ((st = cuda_error(cudaMallocAsync((void **)&scratch, sizeof(float) * ((size_t)rows * cols / 2), s),
                         "wavelet scratch")))
        return st;
    st = run_synthesis(f, d_y, d_y, nullptr, rows, cols, levels, scratch, nullptr, 0, nullptr, d_x, s);
    cudaFreeAsync(scratch, s);
    return st;
}

extern "C" int ctprj_wvlt_l1(const float *d_x, int rows, int cols, const double *h, int lh, int levels, double *d_l1,
                             void *stream)
{
    cudaStream_t s = (cudaStream_t)stream;
    WvltProx ws;
    int st = wvlt_l1(ws, d_x, rows, cols, h, lh, levels, d_l1, s);
    ws.release(s);
    return st;
}

extern "C" int ctprj_wvlt_admm(const float *d_a, int rows, int cols, const double *h, int lh, int levels, double u,
                               double rel_tol, int max_itr, const float *d_init, float *d_alpha, int *iterations,
                               void *stream)
{
    if (!(u >= 0.0)) return set_error(CTPRJ_EINVAL, "u must be non-negative");
    if (max_itr < 0) return set_error(CTPRJ_EINVAL, "negative iteration limit");
    cudaStream_t s = (cudaStream_t)stream;
    WvltProx ws;
    int st = wvlt_admm(ws, d_a, rows, cols, h, lh, levels, u, rel_tol, max_itr, d_init, d_alpha, iterations, s);
    ws.release(s);
    return st;
}

extern "C" int ctprj_wvlt_mask(const unsigned char *d_mask, int rows, int cols, const double *h, int lh, int levels,
                               unsigned char *d_maskk, void *stream)
{
    cudaStream_t s = (cudaStream_t)stream;
    WvltProx ws;
    int st = wvlt_mask(ws, d_mask, rows, cols, h, lh, levels, d_maskk, s);
    ws.release(s);
    return st;
}

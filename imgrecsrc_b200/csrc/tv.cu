// tv.cu -- the total-variation proximal map of the density step on the GPU.
//
// The reference's 'tviso' / 'tvl1' regularisation (bhc/beamhardenSpline.m:
// 199-224) makes the density step's proximal map a bounded TV denoising,
//     min_X ||X - Xobs||^2 + 2 lambda TV(X)   subject to  lb <= X <= ub,
// solved by Beck and Teboulle's fast gradient projection on the dual
// (utils/denoise_bound_mod.m, after A. Beck, M. Teboulle, IEEE TIP 18(11),
// 2009): dual variables P = (P1, P2) on the vertical and horizontal pixel
// differences (utils/Ltrans.m, adjoint utils/Lforward.m), each iteration
//     C = Xobs - lambda L(R),  D = clamp(C),  P = proj(R + L^T(D) / (8 lambda)),
//     R = P + (t_k - 1)/t_{k+1} (P - P_old),
// with the reference's stopping rule (five consecutive relative changes of D
// below epsilon, or max_iter iterations) and its restart (t reset to 1 when the
// dual objective |C|^2 - |C - D|^2 rises).
//
// Three kernels per iteration -- the primal pass (C, D and the FP64 partial
// sums the stopping rule needs), the dual pass, and a one-thread pass that
// advances the iteration's scalars -- keep every decision on the device; the
// host only checks the done flag every few iterations.  Buffers are double
// buffered by the parity of the device-side iteration counter, so launches
// after convergence change nothing.
#include <cmath>

#include "ctprj_internal.h"
#include "../../include/ctprj_tv.h"

namespace ctprj {

struct TvState {
    double tk;      // t of the coming iteration
    double fold;    // dual objective of the last iteration
    int count;      // consecutive relative changes below epsilon
    int iter;       // completed iterations
    int done;
    int pad;
};

struct TvArgs {
    const float *xobs;
    float *D[2], *P1[2], *P2[2];
    float *R1, *R2;
    int m, n;          // rows, columns
    float lam, lb, ub;
    int iso;
    TvState *st;
    double *part;      // per-block partials, 4 per block
};

constexpr int kTvThreads = 256;

__device__ __forceinline__ void block_sum4(double a[4], double *out)
{
    __shared__ double red[4][kTvThreads / 32];
#pragma unroll
    for (int k = 0; k < 4; ++k)
        for (int o = 16; o > 0; o >>= 1) a[k] += __shfl_down_sync(0xffffffffu, a[k], o);
    if ((threadIdx.x & 31) == 0)
#pragma unroll
        for (int k = 0; k < 4; ++k) red[k][threadIdx.x >> 5] = a[k];
    __syncthreads();
    if (threadIdx.x == 0)
        for (int k = 0; k < 4; ++k) {
            double t = 0.0;
            for (int w = 0; w < kTvThreads / 32; ++w) t += red[k][w];
            out[k] = t;
        }
}

// C = Xobs - lambda Lforward(R), D = clamp(C); partials of |D - D_old|^2,
// |D|^2, |C - D|^2, |C|^2
__global__ void __launch_bounds__(kTvThreads) k_tv_primal(const TvArgs a)
{
    if (a.st->done) return;
    const int cur = a.st->iter & 1;
    const float *Dold = cur ? a.D[1] : a.D[0];   // selects, not a local-memory index
    float *Dn = cur ? a.D[0] : a.D[1];
    const long long tot = (long long)a.m * a.n;
    double s[4] = {0.0, 0.0, 0.0, 0.0};
    for (long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x; idx < tot;
         idx += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(idx / a.n), j = (int)(idx % a.n);
        float L = 0.0f;
        if (i < a.m - 1) L += a.R1[idx];
        if (i > 0) L -= a.R1[idx - a.n];
        if (j < a.n - 1) L += a.R2[idx];
        if (j > 0) L -= a.R2[idx - 1];
        const float C = fmaf(-a.lam, L, a.xobs[idx]);
        const float Dv = fminf(fmaxf(C, a.lb), a.ub);
        Dn[idx] = Dv;
        const double dd = (double)Dv - (double)Dold[idx], cd = (double)C - (double)Dv;
        s[0] = fma(dd, dd, s[0]);
        s[1] = fma((double)Dv, (double)Dv, s[1]);
        s[2] = fma(cd, cd, s[2]);
        s[3] = fma((double)C, (double)C, s[3]);
    }
    double out[4];
    block_sum4(s, out);
    if (threadIdx.x == 0)
        for (int k = 0; k < 4; ++k) a.part[4 * blockIdx.x + k] = out[k];
}

// P = proj(R + Ltrans(D) / (8 lambda)); R = P + (t_k - 1)/t_{k+1} (P - P_old)
__global__ void __launch_bounds__(kTvThreads) k_tv_dual(const TvArgs a)
{
    if (a.st->done) return;
    const int cur = a.st->iter & 1;
    const float *Dn = cur ? a.D[0] : a.D[1];
    const float *Po1 = cur ? a.P1[1] : a.P1[0], *Po2 = cur ? a.P2[1] : a.P2[0];
    float *Pn1 = cur ? a.P1[0] : a.P1[1], *Pn2 = cur ? a.P2[0] : a.P2[1];
    const double tk = a.st->tk, tkp1 = 0.5 * (1.0 + sqrt(1.0 + 4.0 * tk * tk));
    const float c = (float)((tk - 1.0) / tkp1), inv8l = 1.0f / (8.0f * a.lam);
    const long long tot = (long long)a.m * a.n;
    for (long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x; idx < tot;
         idx += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(idx / a.n), j = (int)(idx % a.n);
        const bool h1 = i < a.m - 1, h2 = j < a.n - 1;
        const float d = Dn[idx];
        float p1 = h1 ? fmaf(d - Dn[idx + a.n], inv8l, a.R1[idx]) : 0.0f;
        float p2 = h2 ? fmaf(d - Dn[idx + 1], inv8l, a.R2[idx]) : 0.0f;
        if (a.iso) {
            const float A = sqrtf(fmaxf(fmaf(p1, p1, p2 * p2), 1.0f));
            p1 /= A;
            p2 /= A;
        } else {
            p1 = fminf(fmaxf(p1, -1.0f), 1.0f);
            p2 = fminf(fmaxf(p2, -1.0f), 1.0f);
        }
        Pn1[idx] = p1;
        Pn2[idx] = p2;
        a.R1[idx] = fmaf(c, p1 - Po1[idx], p1);
        a.R2[idx] = fmaf(c, p2 - Po2[idx], p2);
    }
}

// the iteration's scalars: stopping count, restart, t, done
__global__ void k_tv_scalars(const TvArgs a, int nblocks, int max_iter, double eps)
{
    TvState *st = a.st;
    if (threadIdx.x != 0 || st->done) return;
    double s[4] = {0.0, 0.0, 0.0, 0.0};
    for (int b = 0; b < nblocks; ++b)
        for (int k = 0; k < 4; ++k) s[k] += a.part[4 * b + k];
    const double re = sqrt(s[0]) / sqrt(s[1]);   // NaN for D = 0: not a small change
    st->count = re < eps ? st->count + 1 : 0;
    const double fval = s[3] - s[2];
    double tkp1 = 0.5 * (1.0 + sqrt(1.0 + 4.0 * st->tk * st->tk));
    if (fval > st->fold) tkp1 = 1.0;
    st->tk = tkp1;
    st->fold = fval;
    st->iter += 1;
    if (st->count >= 5 || st->iter >= max_iter) st->done = 1;
}

// per-block partials of the TV of x (utils/tlv.m)
__global__ void __launch_bounds__(kTvThreads)
k_tv_value(const float *__restrict__ x, int m, int n, int iso, double *__restrict__ part)
{
    const long long tot = (long long)m * n;
    double s[4] = {0.0, 0.0, 0.0, 0.0};
    for (long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x; idx < tot;
         idx += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(idx / n), j = (int)(idx % n);
        const double v = x[idx];
        const double q1 = i < m - 1 ? v - (double)x[idx + n] : 0.0;
        const double q2 = j < n - 1 ? v - (double)x[idx + 1] : 0.0;
        s[0] += iso ? sqrt(q1 * q1 + q2 * q2) : fabs(q1) + fabs(q2);
    }
    double out[4];
    block_sum4(s, out);
    if (threadIdx.x == 0) part[blockIdx.x] = out[0];
}

__global__ void k_tv_sum(const double *__restrict__ part, int nblocks, double *__restrict__ out)
{
    sum_partials(part, nblocks, 1, 1, out);
}

int tv_grid()
{
    int dev = 0, sms = 148;
    if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    return 2 * sms;
}

int TvWorkspace::alloc(int m, int n, cudaStream_t s)
{
    if (buf && rows == m && cols == n) return CTPRJ_OK;
    release(s);
    const size_t px = (size_t)m * n;
    blocks = tv_grid();
    int st;
    if ((st = cuda_error(cudaMallocAsync((void **)&buf, sizeof(float) * px * 8, s), "TV buffers")) ||
        (st = cuda_error(cudaMallocAsync((void **)&part, sizeof(double) * 4 * blocks + 8 * sizeof(double), s),
                         "TV partials")) ||
        (st = cuda_error(cudaMallocAsync((void **)&state, sizeof(TvState), s), "TV state"))) {
        release(s);
        return st;
    }
    rows = m;
    cols = n;
    return CTPRJ_OK;
}

void TvWorkspace::release(cudaStream_t s)
{
    if (buf) cudaFreeAsync(buf, s);
    if (part) cudaFreeAsync(part, s);
    if (state) cudaFreeAsync(state, s);
    buf = nullptr;
    part = nullptr;
    state = nullptr;
    rows = cols = 0;
}

int tv_denoise(TvWorkspace &ws, const float *xobs, int m, int n, double lambda, double lb, double ub,
               int iso, int max_iter, double eps, float *out, int *iterations, cudaStream_t s)
{
    int st;
    if ((st = ws.alloc(m, n, s))) return st;
    const size_t px = (size_t)m * n;
    TvArgs a;
    a.xobs = xobs;
    for (int k = 0; k < 2; ++k) {
        a.D[k] = ws.buf + px * k;
        a.P1[k] = ws.buf + px * (2 + k);
        a.P2[k] = ws.buf + px * (4 + k);
    }
    a.R1 = ws.buf + px * 6;
    a.R2 = ws.buf + px * 7;
    a.m = m;
    a.n = n;
    a.lam = (float)lambda;
    a.lb = (float)lb;
    a.ub = std::isinf(ub) ? INFINITY : (float)ub;
    a.iso = iso;
    a.st = (TvState *)ws.state;
    a.part = ws.part;
    // D = 0; P = proj(Ltrans(0)) = 0; R = P
    TvState init = {1.0, INFINITY, 0, 0, max_iter <= 0 ? 1 : 0, 0};
    if ((st = cuda_error(cudaMemsetAsync(a.D[0], 0, sizeof(float) * px, s), "TV init")) ||
        (st = cuda_error(cudaMemsetAsync(a.P1[0], 0, sizeof(float) * px, s), "TV init")) ||
        (st = cuda_error(cudaMemsetAsync(a.P2[0], 0, sizeof(float) * px, s), "TV init")) ||
        (st = cuda_error(cudaMemsetAsync(a.R1, 0, sizeof(float) * px * 2, s), "TV init")) ||
        (st = cuda_error(cudaMemcpyAsync(a.st, &init, sizeof init, cudaMemcpyHostToDevice, s), "TV init")))
        return st;
    TvState h = init;
    for (int it = 0; it < max_iter; ++it) {
        k_tv_primal<<<ws.blocks, kTvThreads, 0, s>>>(a);
        k_tv_dual<<<ws.blocks, kTvThreads, 0, s>>>(a);
        k_tv_scalars<<<1, 32, 0, s>>>(a, ws.blocks, max_iter, eps);
        if ((st = cuda_error(cudaGetLastError(), "TV iteration"))) return st;
        if ((it & 7) == 7 || it == max_iter - 1) {
            if ((st = cuda_error(cudaMemcpyAsync(&h, a.st, sizeof h, cudaMemcpyDeviceToHost, s), "TV state")) ||
                (st = cuda_error(cudaStreamSynchronize(s), "TV state")))
                return st;
            if (h.done) break;
        }
    }
    if ((st = cuda_error(cudaMemcpyAsync(&h, a.st, sizeof h, cudaMemcpyDeviceToHost, s), "TV state")) ||
        (st = cuda_error(cudaStreamSynchronize(s), "TV state")) ||
        (st = cuda_error(cudaMemcpyAsync(out, a.D[h.iter & 1], sizeof(float) * px, cudaMemcpyDeviceToDevice, s),
                         "TV result")))
        return st;
    if (iterations) *iterations = h.iter;
    return CTPRJ_OK;
}

int tv_value(TvWorkspace &ws, const float *x, int m, int n, int iso, double *d_out, cudaStream_t s)
{
    int st;
    if ((st = ws.alloc(m, n, s))) return st;
    k_tv_value<<<ws.blocks, kTvThreads, 0, s>>>(x, m, n, iso, ws.part);
    k_tv_sum<<<1, 256, 0, s>>>(ws.part, ws.blocks, d_out);
    return cuda_error(cudaGetLastError(), "TV value");
}

}  // namespace ctprj

using namespace ctprj;

extern "C" int ctprj_tv_denoise(const float *d_xobs, int rows, int cols, double lambda, double lb, double ub,
                                int tv_type, int max_iter, double epsilon, float *d_out, int *iterations,
                                void *stream)
{
    if (!d_xobs || !d_out) return set_error(CTPRJ_EINVAL, "NULL buffer");
    if (rows < 2 || cols < 2) return set_error(CTPRJ_EINVAL, "image of at least 2 x 2 pixels");
    if (!(lambda > 0.0)) return set_error(CTPRJ_EINVAL, "lambda must be positive");
    if (!(lb < ub)) return set_error(CTPRJ_EINVAL, "lower bound must be below the upper bound");
    if (tv_type != CTPRJ_TV_ISO && tv_type != CTPRJ_TV_L1) return set_error(CTPRJ_EINVAL, "unknown TV type");
    cudaStream_t s = (cudaStream_t)stream;
    TvWorkspace ws;
    int st = tv_denoise(ws, d_xobs, rows, cols, lambda, lb, ub, tv_type == CTPRJ_TV_ISO, max_iter, epsilon, d_out,
                        iterations, s);
    ws.release(s);
    return st;
}

extern "C" int ctprj_tv_value(const float *d_x, int rows, int cols, int tv_type, double *d_tv, void *stream)
{
    if (!d_x || !d_tv) return set_error(CTPRJ_EINVAL, "NULL buffer");
    if (rows < 1 || cols < 1) return set_error(CTPRJ_EINVAL, "empty image");
    if (tv_type != CTPRJ_TV_ISO && tv_type != CTPRJ_TV_L1) return set_error(CTPRJ_EINVAL, "unknown TV type");
    cudaStream_t s = (cudaStream_t)stream;
    TvWorkspace ws;
    int st = tv_value(ws, d_x, rows, cols, tv_type == CTPRJ_TV_ISO, d_tv, s);
    ws.release(s);
    return st;
}

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
// One fused kernel per iteration does the primal and the dual half on a
// 32 x 32 tile: it forms R = P + c (P - P_prev) on the tile and a one-pixel
// halo in shared memory, C = Xobs - lambda L(R) and D = clamp(C) on the tile
// plus its bottom row and right column, then the new P on the tile, with the
// FP64 partial sums the stopping rule needs.  Per pixel it reads Xobs, D_old,
// P and P_prev (float2 pairs of both components) and writes D and the new P:
// 36 bytes, no R image.  P is triple buffered (the new P cannot overwrite
// P_prev while neighbouring tiles still read its halo), D double buffered,
// both indexed by the device-side iteration counter.  The last block of each
// launch reduces the partials in a fixed order and advances the scalars
// (count, restart, t, the momentum coefficient, done), so every decision
// stays on the device; the host checks the done flag every eight
// iterations, and launches after convergence change nothing.
#include <cmath>

#include "ctprj_internal.h"
#include "../../include/ctprj_tv.h"

namespace ctprj {

struct TvState {
    double tk;          // t of the coming iteration
    double c;           // momentum coefficient of the R the coming iteration forms
    double fold;        // dual objective of the last iteration
    int count;          // consecutive relative changes below epsilon
    int iter;           // completed iterations
    int done;
    unsigned arrived;   // blocks of the running iteration that have written their partials
};

// ws.buf: D (2 images), then the dual buffers 0, 1, 2, each an image of
// float2 (P1, P2) pairs
__host__ __device__ inline float *tv_d(float *buf, size_t px, int k) { return buf + px * (size_t)k; }
__host__ __device__ inline float2 *tv_p(float *buf, size_t px, int b)
{
    return reinterpret_cast<float2 *>(buf + px * (size_t)(2 + 2 * b));
}

struct TvArgs {
    const float *xobs;
    float *buf;
    size_t px;
    int m, n;          // rows, columns
    float lam, lb, ub;
    int iso;
    int max_iter;
    double eps;
    TvState *st;
    double *part;      // per-block partials, 4 per block
};

constexpr int kTvTile = 32;               // tile of kTvTile x kTvTile pixels
constexpr int kTvThreads = 256;           // 32 x 8 threads
constexpr int kTvValueRows = 8;           // rows per block of k_tv_value

__device__ __forceinline__ void block_sum4(double a[4], double *out)
{
    __shared__ double red[4][kTvThreads / 32];
    const int t = threadIdx.y * blockDim.x + threadIdx.x;
#pragma unroll
    for (int k = 0; k < 4; ++k)
        for (int o = 16; o > 0; o >>= 1) a[k] += __shfl_down_sync(0xffffffffu, a[k], o);
    if ((t & 31) == 0)
#pragma unroll
        for (int k = 0; k < 4; ++k) red[k][t >> 5] = a[k];
    __syncthreads();
    if (t == 0)
        for (int k = 0; k < 4; ++k) {
            double v = 0.0;
            for (int w = 0; w < kTvThreads / 32; ++w) v += red[k][w];
            out[k] = v;
        }
}

// The iteration's scalars from the summed partials: stopping count, restart,
// t, momentum coefficient, done.
__device__ void tv_advance(TvState *st, const double s[4], int max_iter, double eps)
{
    const double re = sqrt(s[0]) / sqrt(s[1]);   // NaN for D = 0: not a small change
    st->count = re < eps ? st->count + 1 : 0;
    const double fval = s[3] - s[2];
    const double tk = st->tk, tkp1 = 0.5 * (1.0 + sqrt(1.0 + 4.0 * tk * tk));
    st->c = (tk - 1.0) / tkp1;                 // R = P + (t_k - 1) / t_{k+1} (P - P_old)
    st->tk = fval > st->fold ? 1.0 : tkp1;     // restart when the dual objective rises
    st->fold = fval;
    st->iter += 1;
    if (st->count >= 5 || st->iter >= max_iter) st->done = 1;
}

// One FGP iteration on a kTvTile x kTvTile tile.  Thread (tx, ty) of the
// 32 x 8 block owns column j0 + tx of rows ty, ty + 8, ty + 16, ty + 24, so
// every warp reads and writes whole rows; all global loads of the iteration
// (P, P_prev as float2 pairs, Xobs, D_old) are issued before the first
// barrier.  The last block to finish sums every block's partials in a fixed
// order and advances the scalars, so an iteration is one launch.
__global__ void __launch_bounds__(kTvThreads, 4) k_tv_iter(const TvArgs a)
{
    constexpr int T = kTvTile;
    __shared__ float R1s[T + 2][T + 1];   // rows i0-1 .. i0+T, cols j0 .. j0+T
    __shared__ float R2s[T + 1][T + 2];   // rows i0 .. i0+T, cols j0-1 .. j0+T
    __shared__ float Ds[T + 1][T + 1];    // rows i0 .. i0+T, cols j0 .. j0+T
    __shared__ bool last;
    TvState *st = a.st;
    if (st->done) return;
    const int it = st->iter;
    const float c = (float)st->c;
    const int m = a.m, n = a.n;
    const float2 *P = tv_p(a.buf, a.px, it % 3);          // P
    const float2 *Q = tv_p(a.buf, a.px, (it + 2) % 3);    // P_prev
    float2 *N = tv_p(a.buf, a.px, (it + 1) % 3);          // new P
    const float *Dold = tv_d(a.buf, a.px, it & 1);
    float *Dn = tv_d(a.buf, a.px, (it + 1) & 1);
    const int i0 = blockIdx.y * T, j0 = blockIdx.x * T;
    const int tx = threadIdx.x, ty = threadIdx.y, t = ty * 32 + tx;
    const int j = j0 + tx;
    // R = P + c (P - P_prev) on rows i0-1 .. i0+T.  R1 (vertical
    // differences) exists for rows < m-1, R2 for columns < n-1; elsewhere it
    // is 0, which makes L(R) one formula everywhere.  Every load reads a
    // clamped, valid address and is masked afterwards, so none waits behind a
    // bounds branch.
    const int jc = min(j, n - 1);
    float2 pv[5], qv[5];
#pragma unroll
    for (int k = 0; k < 5; ++k) {
        const int q = min(max(i0 - 1 + ty + 8 * k, 0), m - 1) * n + jc;   // m * n < 2^31
        pv[k] = P[q];
        qv[k] = Q[q];
    }
    // halo columns: j0 + T (R1 and R2, rows i0-1 .. i0+T) and j0 - 1 (R2)
    const int hr = t % (T + 2), hside = t / (T + 2);
    const int hI = i0 - 1 + hr, hJ = hside ? j0 - 1 : j0 + T;
    const int qh = min(max(hI, 0), m - 1) * n + min(max(hJ, 0), n - 1);
    const float2 hp = P[qh], hq = Q[qh];
    float xo[4], dol[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const int q = min(i0 + ty + 8 * k, m - 1) * n + jc;
        xo[k] = a.xobs[q];
        dol[k] = Dold[q];
    }
    // Xobs of the halo D: the bottom row (warp 0), the right column (warp 1)
    const int hi = ty == 0 ? i0 + T : i0 + tx, hj = ty == 0 ? j : j0 + T;
    const bool hin = ty < 2 && hi < m && hj < n;
    const float xh = a.xobs[min(hi, m - 1) * n + min(hj, n - 1)];
#pragma unroll
    for (int k = 0; k < 5; ++k) {
        const int r = ty + 8 * k, i = i0 - 1 + r;      // R1s row r, R2s row r - 1
        if (r < T + 2) {
            R1s[r][tx] = (i >= 0 && i < m - 1 && j < n) ? fmaf(c, pv[k].x - qv[k].x, pv[k].x) : 0.0f;
            if (r >= 1)
                R2s[r - 1][tx + 1] = (i < m && j < n - 1) ? fmaf(c, pv[k].y - qv[k].y, pv[k].y) : 0.0f;
        }
    }
    if (hside == 0 && hr < T + 2) {       // column j0 + T
        R1s[hr][T] = (hI >= 0 && hI < m - 1 && hJ < n) ? fmaf(c, hp.x - hq.x, hp.x) : 0.0f;
        if (hr >= 1) R2s[hr - 1][T + 1] = (hI < m && hJ < n - 1) ? fmaf(c, hp.y - hq.y, hp.y) : 0.0f;
    } else if (hside == 1 && hr >= 1) {   // column j0 - 1
        R2s[hr - 1][0] = (hI < m && hJ >= 0 && hJ < n - 1) ? fmaf(c, hp.y - hq.y, hp.y) : 0.0f;
    }
    __syncthreads();
    // C = Xobs - lambda L(R), D = clamp(C) on the tile (partials) and halo
    const float lam = a.lam, lb = a.lb, ub = a.ub;
    double s[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const int r = ty + 8 * k, i = i0 + r;
        if (i < m && j < n) {
            const float L = (R1s[r + 1][tx] - R1s[r][tx]) + (R2s[r][tx + 1] - R2s[r][tx]);
            const float C = fmaf(-lam, L, xo[k]);
            const float Dv = fminf(fmaxf(C, lb), ub);
            Ds[r][tx] = Dv;
            Dn[i * n + j] = Dv;
            const double dd = (double)Dv - (double)dol[k], cd = (double)C - (double)Dv;
            s[0] = fma(dd, dd, s[0]);
            s[1] = fma((double)Dv, (double)Dv, s[1]);
            s[2] = fma(cd, cd, s[2]);
            s[3] = fma((double)C, (double)C, s[3]);
        }
    }
    if (hin) {
        const int r = ty == 0 ? T : tx, cc = ty == 0 ? tx : T;
        const float L = (R1s[r + 1][cc] - R1s[r][cc]) + (R2s[r][cc + 1] - R2s[r][cc]);
        Ds[r][cc] = fminf(fmaxf(fmaf(-lam, L, xh), lb), ub);
    }
    __syncthreads();
    // P_new = proj(R + Ltrans(D) / (8 lambda)) on the tile
    const float inv8l = 1.0f / (8.0f * lam);
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const int r = ty + 8 * k, i = i0 + r;
        if (i < m && j < n) {
            const float d = Ds[r][tx];
            float p1 = i < m - 1 ? fmaf(d - Ds[r + 1][tx], inv8l, R1s[r + 1][tx]) : 0.0f;
            float p2 = j < n - 1 ? fmaf(d - Ds[r][tx + 1], inv8l, R2s[r][tx + 1]) : 0.0f;
            if (a.iso) {   // P / max(1, |P|): scaled only outside the unit ball
                const float q2 = fmaf(p1, p1, p2 * p2);
                if (q2 > 1.0f) {
                    const float r = rsqrtf(q2);
                    p1 *= r;
                    p2 *= r;
                }
            } else {
                p1 = fminf(fmaxf(p1, -1.0f), 1.0f);
                p2 = fminf(fmaxf(p2, -1.0f), 1.0f);
            }
            N[i * n + j] = make_float2(p1, p2);
        }
    }
    double out[4];
    block_sum4(s, out);
    const unsigned nblocks = gridDim.x * gridDim.y;
    if (t == 0) {
        const size_t b = (size_t)blockIdx.y * gridDim.x + blockIdx.x;
        for (int k = 0; k < 4; ++k) a.part[4 * b + k] = out[k];
        __threadfence();
        last = atomicAdd(&st->arrived, 1u) == nblocks - 1;
    }
    __syncthreads();
    if (!last) return;
    // the last block: sum the partials in a fixed order (thread t takes
    // blocks t, t + 256, ...; then a fixed tree), advance the scalars
    __threadfence();
    double v[4] = {0.0, 0.0, 0.0, 0.0};
    for (unsigned b = t; b < nblocks; b += kTvThreads)
#pragma unroll
        for (int k = 0; k < 4; ++k) v[k] += __ldcg(a.part + 4 * (size_t)b + k);
    __shared__ double red[4][kTvThreads];
#pragma unroll
    for (int k = 0; k < 4; ++k) red[k][t] = v[k];
    __syncthreads();
    for (int h = kTvThreads / 2; h > 0; h >>= 1) {
        if (t < h)
#pragma unroll
            for (int k = 0; k < 4; ++k) red[k][t] += red[k][t + h];
        __syncthreads();
    }
    if (t == 0) {
        const double tot[4] = {red[0][0], red[1][0], red[2][0], red[3][0]};
        tv_advance(st, tot, a.max_iter, a.eps);
        st->arrived = 0;
    }
}

__global__ void k_tv_start(TvState *st, int done)
{
    st->tk = 1.0;
    st->c = 0.0;
    st->fold = INFINITY;
    st->count = 0;
    st->iter = 0;
    st->done = done;
    st->arrived = 0;
}

// per-block partials of the TV of x (utils/tlv.m): block 32 x 8 over a
// 32-column, kTvValueRows-row strip
__global__ void __launch_bounds__(kTvThreads)
k_tv_value(const float *__restrict__ x, int m, int n, int iso, double *__restrict__ part)
{
    const int i = blockIdx.y * kTvValueRows + threadIdx.y, j = blockIdx.x * 32 + threadIdx.x;
    double s[4] = {0.0, 0.0, 0.0, 0.0};
    if (i < m && j < n) {
        const size_t q = (size_t)i * n + j;
        const double v = x[q];
        const double q1 = i < m - 1 ? v - (double)x[q + n] : 0.0;
        const double q2 = j < n - 1 ? v - (double)x[q + 1] : 0.0;
        s[0] = iso ? sqrt(q1 * q1 + q2 * q2) : fabs(q1) + fabs(q2);
    }
    double out[4];
    block_sum4(s, out);
    if (threadIdx.x == 0 && threadIdx.y == 0) part[(size_t)blockIdx.y * gridDim.x + blockIdx.x] = out[0];
}

__global__ void k_tv_sum(const double *__restrict__ part, int nblocks, double *__restrict__ out)
{
    sum_partials(part, nblocks, 1, 1, out);
}

int TvWorkspace::alloc(int m, int n, cudaStream_t s)
{
    if (buf && rows == m && cols == n) return CTPRJ_OK;
    release(s);
    const size_t px = (size_t)m * n;
    const size_t iter_blocks = (size_t)((n + kTvTile - 1) / kTvTile) * ((m + kTvTile - 1) / kTvTile);
    const size_t value_blocks = (size_t)((n + 31) / 32) * ((m + kTvValueRows - 1) / kTvValueRows);
    blocks = (int)(iter_blocks > value_blocks ? iter_blocks : value_blocks);
    int st;
    if ((st = cuda_error(cudaMallocAsync((void **)&buf, sizeof(float) * px * 8, s), "TV buffers")) ||
        (st = cuda_error(cudaMallocAsync((void **)&part, sizeof(double) * 4 * (size_t)blocks, s), "TV partials")) ||
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
    a.buf = ws.buf;
    a.px = px;
    a.m = m;
    a.n = n;
    a.lam = (float)lambda;
    a.lb = (float)lb;
    a.ub = std::isinf(ub) ? INFINITY : (float)ub;
    a.iso = iso;
    a.max_iter = max_iter;
    a.eps = eps;
    a.st = (TvState *)ws.state;
    a.part = ws.part;
    const dim3 grid((n + kTvTile - 1) / kTvTile, (m + kTvTile - 1) / kTvTile), block(32, kTvThreads / 32);
    // D = 0 and P = P_prev = 0 (denoise_bound_mod starts from D = 0, whose
    // projected dual is P = 0, R = P)
    if ((st = cuda_error(cudaMemsetAsync(tv_d(ws.buf, px, 0), 0, sizeof(float) * px, s), "TV start")) ||
        (st = cuda_error(cudaMemsetAsync(tv_p(ws.buf, px, 0), 0, sizeof(float2) * px, s), "TV start")) ||
        (st = cuda_error(cudaMemsetAsync(tv_p(ws.buf, px, 2), 0, sizeof(float2) * px, s), "TV start")))
        return st;
    k_tv_start<<<1, 1, 0, s>>>(a.st, max_iter <= 0 ? 1 : 0);
    TvState h{};
    for (int it = 0; it < max_iter; ++it) {
        k_tv_iter<<<grid, block, 0, s>>>(a);
        if ((st = cuda_error(cudaGetLastError(), "TV iteration"))) return st;
        if ((it & 7) == 7 && it != max_iter - 1) {
            if ((st = cuda_error(cudaMemcpyAsync(&h, a.st, sizeof h, cudaMemcpyDeviceToHost, s), "TV state")) ||
                (st = cuda_error(cudaStreamSynchronize(s), "TV state")))
                return st;
            if (h.done) break;
        }
    }
    if ((st = cuda_error(cudaMemcpyAsync(&h, a.st, sizeof h, cudaMemcpyDeviceToHost, s), "TV state")) ||
        (st = cuda_error(cudaStreamSynchronize(s), "TV state")) ||
        (st = cuda_error(cudaMemcpyAsync(out, tv_d(ws.buf, px, h.iter & 1), sizeof(float) * px,
                                         cudaMemcpyDeviceToDevice, s), "TV result")))
        return st;
    if (iterations) *iterations = h.iter;
    return CTPRJ_OK;
}

int tv_value(TvWorkspace &ws, const float *x, int m, int n, int iso, double *d_out, cudaStream_t s)
{
    int st;
    if ((st = ws.alloc(m, n, s))) return st;
    const dim3 grid((n + 31) / 32, (m + kTvValueRows - 1) / kTvValueRows), block(32, kTvValueRows);
    k_tv_value<<<grid, block, 0, s>>>(x, m, n, iso, ws.part);
    k_tv_sum<<<1, 256, 0, s>>>(ws.part, (int)(grid.x * grid.y), d_out);
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
    if ((long long)rows * cols >= (1LL << 31)) return set_error(CTPRJ_EINVAL, "image of 2^31 pixels or more");
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
    if ((long long)rows * cols >= (1LL << 31)) return set_error(CTPRJ_EINVAL, "image of 2^31 pixels or more");
    if (tv_type != CTPRJ_TV_ISO && tv_type != CTPRJ_TV_L1) return set_error(CTPRJ_EINVAL, "unknown TV type");
    cudaStream_t s = (cudaStream_t)stream;
    TvWorkspace ws;
    int st = tv_value(ws, d_x, rows, cols, tv_type == CTPRJ_TV_ISO, d_tv, s);
    ws.release(s);
    return st;
}

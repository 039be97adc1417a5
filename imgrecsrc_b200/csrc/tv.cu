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
#include <algorithm>
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

// cp.async copies of 8 or 4 bytes into shared memory; src_size 0 (a tile cell
// outside the image) writes zeros and reads nothing
__device__ __forceinline__ void cp_async8(void *smem, const void *gmem, bool valid)
{
    const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(sa), "l"(gmem), "r"(valid ? 8 : 0));
}
__device__ __forceinline__ void cp_async4(void *smem, const void *gmem, bool valid)
{
    const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;\n" ::"r"(sa), "l"(gmem), "r"(valid ? 4 : 0));
}
// 16 bytes, the first `bytes` of them read (the rest zero); both addresses 16-byte aligned
__device__ __forceinline__ void cp_async16(void *smem, const void *gmem, int bytes)
{
    const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(sa), "l"(gmem), "r"(bytes));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
__device__ __forceinline__ void cp_async_wait1() { asm volatile("cp.async.wait_group 1;\n" ::); }

// Shared-memory stage of one tile: P and P_prev on rows i0-1 .. i0+T and
// columns j0-2 .. j0+T+1 (float2 pairs; the extra column on each side keeps
// the 16-byte copies aligned), Xobs on rows i0 .. i0+T and columns
// j0 .. j0+T+3, D_old on the tile.  Cells outside the image are zero, which is
// what P, the difference operators and the clamped reads need there.
constexpr int kTvPR = kTvTile + 2, kTvPW = kTvTile + 4, kTvXR = kTvTile + 1, kTvXW = kTvTile + 4;
struct TvStage {
    float2 P[kTvPR][kTvPW];
    float2 Q[kTvPR][kTvPW];
    float X[kTvXR][kTvXW];
    float D[kTvTile][kTvTile];
};
struct TvSmem {
    TvStage st[2];
    float R1s[kTvTile + 2][kTvTile + 1];   // rows i0-1 .. i0+T, cols j0 .. j0+T
    float R2s[kTvTile + 1][kTvTile + 2];   // rows i0 .. i0+T, cols j0-1 .. j0+T
    float Ds[kTvTile + 1][kTvTile + 1];    // rows i0 .. i0+T, cols j0 .. j0+T
};

// 16-byte copies (two dual pairs or four floats) when a row starts 16-byte
// aligned (cols % 4 == 0), else 8- / 4-byte copies
template <bool VEC>
__device__ __forceinline__ void tv_stage_load(TvStage &S, const TvArgs &a, const float2 *P, const float2 *Q,
                                              const float *Dold, int i0, int j0, int t)
{
    constexpr int T = kTvTile;
    const int m = a.m, n = a.n;
    if (VEC) {
        for (int e = t; e < kTvPR * (kTvPW / 2); e += kTvThreads) {   // pairs of float2
            const int r = e / (kTvPW / 2), c = 2 * (e % (kTvPW / 2));
            const int i = i0 - 1 + r, j = j0 - 2 + c;
            const int cnt = (i >= 0 && i < m && j >= 0) ? max(0, min(2, n - j)) : 0;
            const int q = cnt ? i * n + j : 0;
            cp_async16(&S.P[r][c], P + q, 8 * cnt);
            cp_async16(&S.Q[r][c], Q + q, 8 * cnt);
        }
        for (int e = t; e < kTvXR * (kTvXW / 4); e += kTvThreads) {   // quads of floats
            const int r = e / (kTvXW / 4), c = 4 * (e % (kTvXW / 4));
            const int i = i0 + r, j = j0 + c;
            const int cnt = i < m ? max(0, min(4, n - j)) : 0;
            cp_async16(&S.X[r][c], a.xobs + (cnt ? i * n + j : 0), 4 * cnt);
        }
        for (int e = t; e < T * (T / 4); e += kTvThreads) {
            const int r = e / (T / 4), c = 4 * (e % (T / 4));
            const int i = i0 + r, j = j0 + c;
            const int cnt = i < m ? max(0, min(4, n - j)) : 0;
            cp_async16(&S.D[r][c], Dold + (cnt ? i * n + j : 0), 4 * cnt);
        }
        return;
    }
    for (int e = t; e < kTvPR * kTvPW; e += kTvThreads) {
        const int r = e / kTvPW, c = e % kTvPW;
        const int i = i0 - 1 + r, j = j0 - 2 + c;
        const bool v = i >= 0 && i < m && j >= 0 && j < n;
        const int q = v ? i * n + j : 0;
        cp_async8(&S.P[r][c], P + q, v);
        cp_async8(&S.Q[r][c], Q + q, v);
    }
    for (int e = t; e < kTvXR * kTvXW; e += kTvThreads) {
        const int r = e / kTvXW, c = e % kTvXW;
        const int i = i0 + r, j = j0 + c;
        const bool v = i < m && j < n;
        cp_async4(&S.X[r][c], a.xobs + (v ? i * n + j : 0), v);
    }
    for (int e = t; e < T * T; e += kTvThreads) {
        const int r = e / T, c = e % T;
        const int i = i0 + r, j = j0 + c;
        const bool v = i < m && j < n;
        cp_async4(&S.D[r][c], Dold + (v ? i * n + j : 0), v);
    }
}

// One FGP iteration.  Persistent blocks step through the kTvTile x kTvTile
// tiles; while a block computes one tile from a shared-memory stage, cp.async
// streams its next tile into the other stage, so the memory system stays
// busy across the compute phases.  Per tile: R = P + c (P - P_prev) on the
// tile and a one-pixel halo, C = Xobs - lambda L(R) and D = clamp(C) on the
// tile plus its bottom row and right column, then the new P on the tile.
// Thread (tx, ty) of the 32 x 8 block owns column tx of rows ty, ty + 8, ...
// The last block to finish sums every block's partials in a fixed order and
// advances the scalars, so an iteration is one launch.
template <bool VEC>
__global__ void __launch_bounds__(kTvThreads) k_tv_iter(const TvArgs a, int tiles_x, int ntiles)
{
    constexpr int T = kTvTile;
    extern __shared__ __align__(16) unsigned char tv_smem[];
    TvSmem &S = *reinterpret_cast<TvSmem *>(tv_smem);
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
    const int tx = threadIdx.x, ty = threadIdx.y, t = ty * 32 + tx;
    const float lam = a.lam, lb = a.lb, ub = a.ub, inv8l = 1.0f / (8.0f * lam);
    double s[4] = {0.0, 0.0, 0.0, 0.0};
    int tile = blockIdx.x, stage = 0;
    if (tile < ntiles) tv_stage_load<VEC>(S.st[0], a, P, Q, Dold, (tile / tiles_x) * T, (tile % tiles_x) * T, t);
    cp_async_commit();
    for (; tile < ntiles; tile += gridDim.x) {
        const int next = tile + gridDim.x;
        if (next < ntiles)
            tv_stage_load<VEC>(S.st[stage ^ 1], a, P, Q, Dold, (next / tiles_x) * T, (next % tiles_x) * T, t);
        cp_async_commit();
        cp_async_wait1();          // this tile's copies have landed (this thread's)
        __syncthreads();           // ... and every thread's
        const TvStage &G = S.st[stage];
        const int i0 = (tile / tiles_x) * T, j0 = (tile % tiles_x) * T;
        const int j = j0 + tx;
        // R on rows i0-1 .. i0+T (stage row r), columns j0-1 .. j0+T (stage
        // column cc + 1): R1 from column j0 + cc, R2 from column j0 - 1 + cc
        for (int e = t; e < (T + 2) * (T + 2); e += kTvThreads) {
            const int r = e / (T + 2), cc = e % (T + 2);
            const float2 p = G.P[r][cc + 1], q = G.Q[r][cc + 1];
            if (cc >= 1) S.R1s[r][cc - 1] = fmaf(c, p.x - q.x, p.x);
            if (r >= 1) S.R2s[r - 1][cc] = fmaf(c, p.y - q.y, p.y);
        }
        __syncthreads();
        // C = Xobs - lambda L(R), D = clamp(C) on the tile (partials) and its halo
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const int r = ty + 8 * k, i = i0 + r;
            if (i < m && j < n) {
                const float L = (S.R1s[r + 1][tx] - S.R1s[r][tx]) + (S.R2s[r][tx + 1] - S.R2s[r][tx]);
                const float C = fmaf(-lam, L, G.X[r][tx]);
                const float Dv = fminf(fmaxf(C, lb), ub);
                S.Ds[r][tx] = Dv;
                Dn[i * n + j] = Dv;
                const double dd = (double)Dv - (double)G.D[r][tx], cd = (double)C - (double)Dv;
                s[0] = fma(dd, dd, s[0]);
                s[1] = fma((double)Dv, (double)Dv, s[1]);
                s[2] = fma(cd, cd, s[2]);
                s[3] = fma((double)C, (double)C, s[3]);
            }
        }
        if (ty < 2) {   // the bottom row (warp 0) and the right column (warp 1)
            const int r = ty == 0 ? T : tx, cc = ty == 0 ? tx : T;
            if (i0 + r < m && j0 + cc < n) {
                const float L = (S.R1s[r + 1][cc] - S.R1s[r][cc]) + (S.R2s[r][cc + 1] - S.R2s[r][cc]);
                S.Ds[r][cc] = fminf(fmaxf(fmaf(-lam, L, G.X[r][cc]), lb), ub);
            }
        }
        __syncthreads();
        // P_new = proj(R + Ltrans(D) / (8 lambda)) on the tile
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const int r = ty + 8 * k, i = i0 + r;
            if (i < m && j < n) {
                const float d = S.Ds[r][tx];
                float p1 = i < m - 1 ? fmaf(d - S.Ds[r + 1][tx], inv8l, S.R1s[r + 1][tx]) : 0.0f;
                float p2 = j < n - 1 ? fmaf(d - S.Ds[r][tx + 1], inv8l, S.R2s[r][tx + 1]) : 0.0f;
                if (a.iso) {   // P / max(1, |P|): scaled only outside the unit ball
                    const float q2 = fmaf(p1, p1, p2 * p2);
                    if (q2 > 1.0f) {
                        const float rs = rsqrtf(q2);
                        p1 *= rs;
                        p2 *= rs;
                    }
                } else {
                    p1 = fminf(fmaxf(p1, -1.0f), 1.0f);
                    p2 = fminf(fmaxf(p2, -1.0f), 1.0f);
                }
                N[i * n + j] = make_float2(p1, p2);
            }
        }
        __syncthreads();           // the stage and the R / D tiles are free again
        stage ^= 1;
    }
    double out[4];
    block_sum4(s, out);
    const unsigned nblocks = gridDim.x;
    if (t == 0) {
        for (int k = 0; k < 4; ++k) a.part[4 * (size_t)blockIdx.x + k] = out[k];
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
    double(*red)[kTvThreads] = reinterpret_cast<double(*)[kTvThreads]>(tv_smem);   // the stages are free now
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
    const int tiles_x = (n + kTvTile - 1) / kTvTile, ntiles = tiles_x * ((m + kTvTile - 1) / kTvTile);
    const dim3 block(32, kTvThreads / 32);
    const size_t smem = sizeof(TvSmem);
    int dev = 0, sms = 148, per_sm = 1;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    // 16-byte aligned rows for the vector copies
    const bool vec = n % 4 == 0 && ((uintptr_t)xobs & 15) == 0;
    auto kern = vec ? k_tv_iter<true> : k_tv_iter<false>;
    if ((st = cuda_error(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem),
                         "TV shared memory")) ||
        (st = cuda_error(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kTvThreads, smem),
                         "TV occupancy")))
        return st;
    const int grid = std::min(ntiles, sms * std::max(per_sm, 1));   // persistent blocks
    // D = 0 and P = P_prev = 0 (denoise_bound_mod starts from D = 0, whose
    // projected dual is P = 0, R = P)
    if ((st = cuda_error(cudaMemsetAsync(tv_d(ws.buf, px, 0), 0, sizeof(float) * px, s), "TV start")) ||
        (st = cuda_error(cudaMemsetAsync(tv_p(ws.buf, px, 0), 0, sizeof(float2) * px, s), "TV start")) ||
        (st = cuda_error(cudaMemsetAsync(tv_p(ws.buf, px, 2), 0, sizeof(float2) * px, s), "TV start")))
        return st;
    k_tv_start<<<1, 1, 0, s>>>(a.st, max_iter <= 0 ? 1 : 0);
    TvState h{};
    for (int it = 0; it < max_iter; ++it) {
        kern<<<grid, block, smem, s>>>(a, tiles_x, ntiles);
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

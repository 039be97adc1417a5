// bhc_loop.cu -- the alternating beam-hardening reconstruction loop.
//
// The reference alternates an image step and a spectrum step
// (bhc/beamhardenSpline.m:340-570): the image step minimises the Poisson
// likelihood in the density with Nesterov's proximal gradient method (NPG,
// npg/NPG.m), the spectrum step updates the B-spline coefficients Ie >= 0 on
// poissLI's objective (bhc/poissLI.m:2-16).  This file runs that loop on the
// GPU:
//
//  density step   one NPG iteration: extrapolation, the fused forward and its
//                 adjoint at xbar, a majorisation line search on the fused
//                 forward, momentum restart (ctprj_bhc_reconstruct below);
//  spectrum step  Newton on Ie >= 0: gradient A^T (1 - m/Ir) and Hessian
//                 A^T diag(m / Ir^2) A (Gaussian model: A^T (Err / Ir) and the
//                 Gauss-Newton A^T diag(1 / Ir^2) A) reduced in FP64 from the rays x J basis
//                 matrix A of the current projections, the quadratic model
//                 minimised over Ie >= 0 by an active-set method in one warp
//                 (FP64 Cholesky, diagonal lifted until positive definite as
//                 bhc/ActiveSet.m:62-76 lifts the eigenvalues), then a line
//                 search shrinking the step by 0.8 (ActiveSet stepShrnk).
#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstring>
#include <vector>

#include "ctprj_internal.h"
#include "bhc_spline.cuh"
#include "../../include/ctprj_bhc_loop.h"

namespace ctprj {

constexpr int kMaxH = kMaxJ * (kMaxJ + 1) / 2;

// The basis matrix A (b_j(s_i), J <= 32 functions x nrays rays) of the
// spectrum step is stored in blocks of four rays: block c holds the 32 x 4
// values of rows j < 32 and rays 4c .. 4c + 3, row by row.  A warp's load of
// one row for 32 consecutive rays then reads eight whole 32-byte sectors, and
// the tensor-core fragments of four rays x eight rows are one contiguous
// 256-byte segment.  Rows J .. 31 are never read.
__host__ __device__ __forceinline__ size_t ie_index(int j, long long i)
{
    return ((size_t)(i >> 2) * 32 + j) * 4 + (size_t)(i & 3);
}
__host__ __device__ __forceinline__ size_t ie_elems(long long nrays) { return (size_t)((nrays + 3) >> 2) * 128; }

// The spectrum model at Ie from the basis matrix A, in two passes whose
// per-block partials share one layout,
// part[block * (1 + J + J(J+1)/2)] = {f, g (J), upper triangle of H}:
//  k_ie_rays  one thread per ray: Ir = A_i . Ie, the likelihood term into f,
//             r_i = df/dIr and sqrt(q_i) (q: the model curvature, >= 0 for
//             both noise models) into per-ray arrays;
//  k_ie_gh    g = sum_i A_i r_i and H = sum_i q_i A_i A_i^T = W^T W,
//             W = diag(sqrt q) A^T, on the FP64 tensor cores: a warp takes
//             four rays at a time, lane (group gr = lane / 4, t = lane % 4)
//             loading A[j][i] for ray i = 4c + t and rows j = gr, gr + 8,
//             gr + 16, gr + 24 -- exactly the operand fragments of the MMA
//             m8n8k4 (an 8 x 4 block of W^T and its 4 x 8 transpose share
//             them) -- so H accumulates as the 10 upper 8 x 8 tiles of a
//             32 x 32 matrix by mma.sync (the FP64 kind; tcgen05 has none).
//             Each warp walks a contiguous range of rays.
// One warp walks groups of 16 rays (four blocks of A, 4 KB contiguous): the
// group arrives in the warp's shared-memory slot by 16-byte cp.async (rows
// J .. 31 skipped), padded to 132 doubles per block so that the warp's 16
// (block, ray) columns fall in distinct bank pairs; lanes 2r and 2r + 1 then
// reduce rows 0..15 and 16..J-1 of ray r and add the halves by one shuffle.
// per_ray(i, Ir) runs in the even lane of each ray.
constexpr int kIeWarps = 8;
constexpr int kIeChunkStride = 132;

__device__ __forceinline__ void cp_async16(void *smem, const void *gmem)
{
    const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(sa), "l"(gmem) : "memory");
}

__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

template <class F>
__device__ __forceinline__ void ie_walk_rays(const double *__restrict__ A, long long nrays, int J,
                                             const double *Is, double *wbuf, F &&per_ray)
{
    const int lane = threadIdx.x & 31, h = lane & 1, r = lane >> 1;
    const long long nchunks = (nrays + 3) >> 2, ngroups = (nchunks + 3) >> 2;
    const long long nw = (long long)gridDim.x * kIeWarps;
    for (long long gi = (long long)blockIdx.x * kIeWarps + (threadIdx.x >> 5); gi < ngroups; gi += nw) {
        const long long c0 = gi * 4;
        const int nunits = (int)min(4LL, nchunks - c0) * 64;   // 16-byte units: block e / 64, row (e % 64) / 2
        const double *src = A + (size_t)c0 * 128;
        for (int e = lane; e < nunits; e += 32)
            if (((e & 63) >> 1) < J) cp_async16(wbuf + (e >> 6) * kIeChunkStride + (e & 63) * 2, src + (size_t)e * 2);
        cp_async_wait_all();
        __syncwarp();
        const double *col = wbuf + (r >> 2) * kIeChunkStride + (r & 3);
        const int j1 = min(J, 16 * h + 16);
        double Ir = 0.0;
        for (int j = 16 * h; j < j1; ++j) Ir = fma(col[4 * j], Is[j], Ir);
        Ir += __shfl_xor_sync(0xffffffffu, Ir, 1);
        const long long i = 4 * c0 + r;
        if (h == 0 && i < nrays) per_ray(i, Ir);
        __syncwarp();
    }
}

__device__ __forceinline__ void ie_block_sum(double f, double *red, double *out)
{
    for (int o = 16; o > 0; o >>= 1) f += __shfl_down_sync(0xffffffffu, f, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = f;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += red[w];
        *out = t;
    }
}

__global__ void __launch_bounds__(kIeWarps * 32)
k_ie_rays(const double *__restrict__ A, const float *__restrict__ m, long long nrays, int J,
          const double *__restrict__ Ie, int noise, int stride, double *__restrict__ rr,
          double *__restrict__ sq, double *__restrict__ part)
{
    __shared__ double Is[kMaxJ];
    __shared__ double red[kIeWarps];
    __shared__ __align__(16) double wb[kIeWarps][4 * kIeChunkStride];
    for (int j = threadIdx.x; j < J; j += blockDim.x) Is[j] = Ie[j];
    __syncthreads();
    double f = 0.0;
    ie_walk_rays(A, nrays, J, Is, wb[threadIdx.x >> 5], [&](long long i, double Ir) {
        const double mi = (double)m[i];
        const RayTerms t = ray_terms(noise, Ir, mi);
        f += t.f;
        rr[i] = t.r;
        sq[i] = sqrt(ray_curvature_model(noise, Ir, mi));
    });
    ie_block_sum(f, red, part + (size_t)blockIdx.x * stride);
}

constexpr int kGhWarps = 4;

__device__ __forceinline__ void dmma_acc(double &d0, double &d1, double a, double b)
{
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};\n"
                 : "+d"(d0), "+d"(d1)
                 : "d"(a), "d"(b));
}

__global__ void __launch_bounds__(kGhWarps * 32)
k_ie_gh(const double *__restrict__ A, long long nrays, int J, const double *__restrict__ rr,
        const double *__restrict__ sq, int stride, double *__restrict__ part)
{
    __shared__ double hred[kGhWarps][10][64];
    __shared__ double gred[kGhWarps][kMaxJ];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int gr = lane >> 2, tig = lane & 3;
    const int nb = (J + 7) >> 3;   // 8-row blocks in use
    // this warp's contiguous range of four-ray chunks
    const long long nchunks = (nrays + 3) >> 2;
    const long long wid = (long long)blockIdx.x * kGhWarps + warp, nw = (long long)gridDim.x * kGhWarps;
    const long long c0 = nchunks * wid / nw, c1 = nchunks * (wid + 1) / nw;
    double d[10][2];
#pragma unroll
    for (int t = 0; t < 10; ++t) d[t][0] = d[t][1] = 0.0;
    double g[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll 2
    for (long long c = c0; c < c1; ++c) {
        const long long i = 4 * c + tig;
        const bool in = i < nrays;
        const double si = in ? sq[i] : 0.0, ri = in ? rr[i] : 0.0;
        double w[4];
#pragma unroll
        for (int jb = 0; jb < 4; ++jb) {
            const int j = jb * 8 + gr;
            const double a = (in && j < J) ? __ldg(A + ie_index(j, i)) : 0.0;
            w[jb] = si * a;
            g[jb] = fma(a, ri, g[jb]);
        }
        int t = 0;
#pragma unroll
        for (int jr = 0; jr < 4; ++jr)
#pragma unroll
            for (int jc = jr; jc < 4; ++jc, ++t)
                if (jc < nb) dmma_acc(d[t][0], d[t][1], w[jr], w[jc]);
    }
    // the block: warp partials through shared memory, summed in a fixed order
    {
        int t = 0;
#pragma unroll
        for (int jr = 0; jr < 4; ++jr)
#pragma unroll
            for (int jc = jr; jc < 4; ++jc, ++t) {
                hred[warp][t][gr * 8 + 2 * tig] = d[t][0];
                hred[warp][t][gr * 8 + 2 * tig + 1] = d[t][1];
            }
    }
#pragma unroll
    for (int jb = 0; jb < 4; ++jb) {   // the four lanes of a group hold the same rows
        g[jb] += __shfl_xor_sync(0xffffffffu, g[jb], 1);
        g[jb] += __shfl_xor_sync(0xffffffffu, g[jb], 2);
    }
    if (tig == 0)
#pragma unroll
        for (int jb = 0; jb < 4; ++jb) gred[warp][jb * 8 + gr] = g[jb];
    __syncthreads();
    double *out = part + (size_t)blockIdx.x * stride;
    for (int j = threadIdx.x; j < J; j += blockDim.x) {
        double v = 0.0;
        for (int ww = 0; ww < kGhWarps; ++ww) v += gred[ww][j];
        out[1 + j] = v;
    }
    double *h = out + 1 + J;
    for (int e = threadIdx.x; e < 10 * 64; e += blockDim.x) {
        const int t = e >> 6, rc = e & 63;
        // tile t of the upper 4 x 4 tiles in row order: (0,0) (0,1) (0,2) (0,3) (1,1) ...
        const int jr = t < 4 ? 0 : t < 7 ? 1 : t < 9 ? 2 : 3;
        const int jc = jr + t - (jr == 0 ? 0 : jr == 1 ? 4 : jr == 2 ? 7 : 9);
        const int j = jr * 8 + (rc >> 3), k = jc * 8 + (rc & 7);
        if (j <= k && k < J) {
            double v = 0.0;
            for (int ww = 0; ww < kGhWarps; ++ww) v += hred[ww][t][rc];
            h[j * J - j * (j - 1) / 2 + (k - j)] = v;
        }
    }
}

// per-block partials of f alone (the line search's trial points), written to
// part[block * stride]
__global__ void __launch_bounds__(kIeWarps * 32)
k_ie_f(const double *__restrict__ A, const float *__restrict__ m, long long nrays, int J,
       const double *__restrict__ Ie, int noise, int stride, double *__restrict__ part)
{
    __shared__ double Is[kMaxJ];
    __shared__ double red[kIeWarps];
    __shared__ __align__(16) double wb[kIeWarps][4 * kIeChunkStride];
    for (int j = threadIdx.x; j < J; j += blockDim.x) Is[j] = Ie[j];
    __syncthreads();
    double f = 0.0;
    ie_walk_rays(A, nrays, J, Is, wb[threadIdx.x >> 5],
                 [&](long long i, double Ir) { f += ray_terms(noise, Ir, (double)m[i]).f; });
    ie_block_sum(f, red, part + (size_t)blockIdx.x * stride);
}

// out[c] = sum over blocks of part[b * stride + c] for c < ncols (fixed order, FP64)
__global__ void k_ie_sum(const double *__restrict__ part, int nblocks, int stride, int ncols,
                         double *__restrict__ out)
{
    sum_partials(part, nblocks, stride, ncols, out);
}

// the same sums for many columns: block (32 columns x 32 row groups), each
// thread four interleaved partial sums over its rows, then a fixed tree over
// the groups -- every column's order is fixed by the launch shape
__global__ void __launch_bounds__(1024) k_ie_sum_wide(const double *__restrict__ part, int nblocks, int stride,
                                                      int ncols, double *__restrict__ out)
{
    __shared__ double red[32][33];
    const int cl = threadIdx.x, grp = threadIdx.y, c = blockIdx.x * 32 + cl;
    double a0 = 0.0, a1 = 0.0, a2 = 0.0, a3 = 0.0;
    if (c < ncols) {
        auto P = [&](int b) { return part[(size_t)b * stride + c]; };
        int b = grp;
        for (; b + 96 < nblocks; b += 128) {
            a0 += P(b);
            a1 += P(b + 32);
            a2 += P(b + 64);
            a3 += P(b + 96);
        }
        if (b < nblocks) a0 += P(b);
        if (b + 32 < nblocks) a1 += P(b + 32);
        if (b + 64 < nblocks) a2 += P(b + 64);
    }
    red[grp][cl] = (a0 + a1) + (a2 + a3);
    __syncthreads();
    for (int h = 16; h > 0; h >>= 1) {
        if (grp < h) red[grp][cl] += red[grp + h][cl];
        __syncthreads();
    }
    if (grp == 0 && c < ncols) out[c] = red[0][cl];
}

// Cholesky factorisation, by one warp, of the Jacobi-scaled block
// H[F][F] / (dg_a dg_b) + lift I of the nf coefficients Fidx[0..nf) into L
// (lane r owns row r).  Fails (warp-uniformly) when a pivot is not above
// 1e-14 (1 + lift).
__device__ bool warp_cholesky(double (*L)[kMaxJ + 1], const double (*H)[kMaxJ + 1], const int *Fidx,
                              const double *dgs, int nf, double lift)
{
    const int r = threadIdx.x;
    if (r < nf) {
        const int jr = Fidx[r];
        for (int b = 0; b <= r; ++b) {
            const int jb = Fidx[b];
            L[r][b] = H[jr][jb] / (dgs[jr] * dgs[jb]) + (b == r ? lift : 0.0);
        }
    }
    bool ok = true;
    for (int k = 0; k < nf; ++k) {
        __syncwarp();
        const double d = L[k][k];
        if (!(d > 1e-14 * (1.0 + lift))) { ok = false; break; }
        const double lk = sqrt(d);
        __syncwarp();
        if (r == k) L[k][k] = lk;
        if (r > k && r < nf) L[r][k] /= lk;
        __syncwarp();
        if (r > k && r < nf) {
            const double lrk = L[r][k];
            for (int b = k + 1; b <= r; ++b) L[r][b] = fma(-lrk, L[b][k], L[r][b]);
        }
    }
    __syncwarp();
    return ok;
}

// The Newton direction of the spectrum step.  The quadratic model
//   q(y) = 1/2 y'Hy + c'y,   c = g - H Ie,
// is minimised over y >= 0 by a primal active-set method started at y = Ie
// (working set W: coefficients held at 0); dir = y - Ie, a feasible direction
// along which the line search needs no projection.  The reference's
// ActiveSet class (bhc/ActiveSet.m:52-181) also keeps the iterate feasible and
// moves the active set one constraint at a time; here the subproblem is solved
// to its optimum every Newton step, which is what makes the outer iteration
// converge in a few steps although H spans many decades.
// H is first made positive definite: its Jacobi-scaled form (unit diagonal) is
// factored with the diagonal lifted (0, then 1e-14, x10) until every pivot
// stays above 1e-14, and the lift is kept for the whole subproblem, so that the
// model is convex (bhc/ActiveSet.m:62-76 lifts the eigenvalues of the reduced
// Hessian the same way; the Gaussian model's Hessian can be indefinite).
// On each free set F, H_FF z_F = -c_F is solved through the same scaled
// factorisation.  A full step to z ends in a multiplier check (release the most
// negative lambda_j = (Hy + c)_j of W); a blocked step adds the blocking
// coefficient to W.
// One warp: lane t owns coefficient t; inside a factorisation lane r owns row
// r of the free block.  All branches that end loops are warp-uniform.
__global__ void __launch_bounds__(32)
k_ie_qp(const double *__restrict__ fgh, const double *__restrict__ Ie, int J, double *__restrict__ dir,
        int *__restrict__ qp_iters)
{
    __shared__ double H[kMaxJ][kMaxJ + 1];
    __shared__ double L[kMaxJ][kMaxJ + 1];
    __shared__ double rhs[kMaxJ], ys[kMaxJ], cs[kMaxJ], dgs[kMaxJ];
    __shared__ int Fidx[kMaxJ];
    const unsigned full = 0xffffffffu;
    const int t = threadIdx.x;
    const unsigned below = (1u << t) - 1u;
    const double *g = fgh + 1, *hp = fgh + 1 + J;
    if (t < J)
        for (int k = t; k < J; ++k) {
            const double v = hp[t * J - t * (t - 1) / 2 + (k - t)];   // packed upper triangle
            H[t][k] = v;
            H[k][t] = v;
        }
    __syncwarp();
    // a coefficient whose basis function vanishes on every ray has H_tt = 0
    // (and a zero row): it is left where it is
    const bool fixed = !(t < J) || !(H[t < J ? t : 0][t < J ? t : 0] > 0.0);
    const double ie = t < J ? Ie[t] : 0.0;
    const double dg = fixed ? 1.0 : sqrt(H[t][t]);
    dgs[t] = dg;
    // convexify: the smallest lift of the scaled diagonal that factors
    {
        const unsigned am = __ballot_sync(full, !fixed);
        if (!fixed) Fidx[__popc(am & below)] = t;
        __syncwarp();
        double lift = 0.0;
        bool ok = false;
        for (int attempt = 0; attempt < 40 && !ok; ++attempt) {
            ok = warp_cholesky(L, H, Fidx, dgs, __popc(am), lift);
            if (!ok) lift = lift == 0.0 ? 1e-14 : lift * 10.0;
        }
        if (!ok) {   // nothing sensible to do: no step
            if (t < J) dir[t] = 0.0;
            if (t == 0 && qp_iters) *qp_iters = -1;
            return;
        }
        if (!fixed) H[t][t] *= 1.0 + lift;
        __syncwarp();
    }
    double c = 0.0;
    if (t < J) {
        double hy = 0.0;
        for (int k = 0; k < J; ++k) hy = fma(H[t][k], Ie[k], hy);
        c = g[t] - hy;
    }
    double y = fixed ? ie : fmax(ie, 0.0);
    bool inW = !fixed && !(ie > 0.0);
    cs[t] = c;
    int it = 0;
    for (; it < 8 * J + 16; ++it) {
        const bool fr = !fixed && !inW;
        const unsigned fm = __ballot_sync(full, fr);
        const int nf = __popc(fm);
        if (fr) Fidx[__popc(fm & below)] = t;
        __syncwarp();
        double z = y;
        if (nf > 0) {
            // principal blocks of a positive definite matrix factor without a
            // lift; the retries only guard against rounding
            double lift = 0.0;
            bool ok = false;
            for (int attempt = 0; attempt < 40 && !ok; ++attempt) {
                ok = warp_cholesky(L, H, Fidx, dgs, nf, lift);
                if (!ok) lift = lift == 0.0 ? 1e-14 : lift * 10.0;
            }
            if (!ok) break;
            const int r = t;
            if (r < nf) rhs[r] = -cs[Fidx[r]] / dgs[Fidx[r]];
            for (int k = 0; k < nf; ++k) {   // L w = rhs
                __syncwarp();
                const double wk = rhs[k] / L[k][k];
                __syncwarp();
                if (r == k) rhs[k] = wk;
                if (r > k && r < nf) rhs[r] = fma(-L[r][k], wk, rhs[r]);
            }
            for (int k = nf - 1; k >= 0; --k) {   // L^T v = w
                __syncwarp();
                const double vk = rhs[k] / L[k][k];
                __syncwarp();
                if (r == k) rhs[k] = vk;
                if (r < k) rhs[r] = fma(-L[k][r], vk, rhs[r]);
            }
            __syncwarp();
            if (fr) z = rhs[__popc(fm & below)] / dg;
        }
        const double p = fr ? z - y : 0.0;
        // ratio test: the first coefficient to reach 0 along p
        double rv = (fr && p < 0.0) ? -y / p : INFINITY;
        int ri = t;
        for (int o = 16; o > 0; o >>= 1) {
            const double ov = __shfl_xor_sync(full, rv, o);
            const int oi = __shfl_xor_sync(full, ri, o);
            if (ov < rv || (ov == rv && oi < ri)) { rv = ov; ri = oi; }
        }
        if (rv >= 1.0) {
            if (fr) y = z;
            ys[t] = y;
            __syncwarp();
            double hy = 0.0;
            if (t < J)
                for (int k = 0; k < J; ++k) hy = fma(H[t][k], ys[k], hy);
            const double lam = hy + c;
            const bool cand = inW && lam < -1e-13 * (fabs(c) + fabs(hy));
            if (__ballot_sync(full, cand) == 0u) { ++it; break; }   // optimal
            double lv = cand ? lam : INFINITY;
            int li = t;
            for (int o = 16; o > 0; o >>= 1) {
                const double ov = __shfl_xor_sync(full, lv, o);
                const int oi = __shfl_xor_sync(full, li, o);
                if (ov < lv || (ov == lv && oi < li)) { lv = ov; li = oi; }
            }
            if (t == li) inW = false;
        } else {
            if (fr) y = fma(rv, p, y);
            if (t == ri) {
                y = 0.0;
                inW = true;
            }
        }
        __syncwarp();
    }
    if (t < J) dir[t] = y - ie;
    if (t == 0 && qp_iters) *qp_iters = it;
}

// Ie_trial = max(0, Ie + step * dir); out[J] = g . (Ie_trial - Ie)
__global__ void k_ie_trial(const double *__restrict__ Ie, const double *__restrict__ dir,
                           const double *__restrict__ fgh, int J, double step,
                           double *__restrict__ trial)
{
    if (threadIdx.x == 0) {
        double gd = 0.0;
        for (int j = 0; j < J; ++j) {
            const double v = fmax(0.0, Ie[j] + step * dir[j]);
            trial[j] = v;
            gd += fgh[1 + j] * (v - Ie[j]);
        }
        trial[J] = gd;
    }
}

// x_new = max(0, x - a g); per-block partials of g . (x_new - x) and |x_new - x|^2
__global__ void __launch_bounds__(256)
k_pg_step(const float *__restrict__ x, const float *__restrict__ g, long long n, float a,
          float *__restrict__ xn, double *__restrict__ part)
{
    __shared__ double red[2][8];
    double gd = 0.0, dd = 0.0;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        const float v = fmaxf(0.0f, x[i] - a * g[i]);
        xn[i] = v;
        const double d = (double)v - (double)x[i];
        gd = fma((double)g[i], d, gd);
        dd = fma(d, d, dd);
    }
    for (int o = 16; o > 0; o >>= 1) {
        gd += __shfl_down_sync(0xffffffffu, gd, o);
        dd += __shfl_down_sync(0xffffffffu, dd, o);
    }
    if ((threadIdx.x & 31) == 0) {
        red[0][threadIdx.x >> 5] = gd;
        red[1][threadIdx.x >> 5] = dd;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double a0 = 0.0, a1 = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) {
            a0 += red[0][w];
            a1 += red[1][w];
        }
        part[2 * blockIdx.x] = a0;
        part[2 * blockIdx.x + 1] = a1;
    }
}

// per-block partials of g . (xn - x) and |xn - x|^2 for a candidate xn that a
// proximal map other than the projection produced
__global__ void __launch_bounds__(256)
k_step_terms(const float *__restrict__ x, const float *__restrict__ g, const float *__restrict__ xn, long long n,
             double *__restrict__ part)
{
    __shared__ double red[2][8];
    double gd = 0.0, dd = 0.0;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        const double d = (double)xn[i] - (double)x[i];
        gd = fma((double)g[i], d, gd);
        dd = fma(d, d, dd);
    }
    for (int o = 16; o > 0; o >>= 1) {
        gd += __shfl_down_sync(0xffffffffu, gd, o);
        dd += __shfl_down_sync(0xffffffffu, dd, o);
    }
    if ((threadIdx.x & 31) == 0) {
        red[0][threadIdx.x >> 5] = gd;
        red[1][threadIdx.x >> 5] = dd;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double a0 = 0.0, a1 = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) {
            a0 += red[0][w];
            a1 += red[1][w];
        }
        part[2 * blockIdx.x] = a0;
        part[2 * blockIdx.x + 1] = a1;
    }
}

// x = 0 outside the reconstruction mask (the reference's density is the
// masked pixel vector, tomography/ConfigCT.m:122-135 with utils/maskFunc.m)
__global__ void __launch_bounds__(256)
k_mask_apply(float *__restrict__ x, const unsigned char *__restrict__ mask, long long n)
{
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        if (!mask[i]) x[i] = 0.0f;
}

// Nesterov extrapolation xbar = max(0, x + coef (x - xprev)); per-block
// partials of sum |xbar - x| (whether the step carries momentum)
__global__ void __launch_bounds__(256)
k_npg_extrapolate(const float *__restrict__ x, const float *__restrict__ xprev, long long n, float coef,
                  float *__restrict__ xbar, double *__restrict__ part)
{
    __shared__ double red[8];
    double mom = 0.0;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        const float xi = x[i];
        const float v = fmaxf(0.0f, fmaf(coef, xi - xprev[i], xi));
        xbar[i] = v;
        mom += fabs((double)v - (double)xi);
    }
    for (int o = 16; o > 0; o >>= 1) mom += __shfl_down_sync(0xffffffffu, mom, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = mom;
    __syncthreads();
    if (threadIdx.x == 0) {
        double a = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) a += red[w];
        part[2 * blockIdx.x] = a;
        part[2 * blockIdx.x + 1] = 0.0;
    }
}

// per-block partials of sum (a_i - b_i) c_i (b may be NULL), FP64
__global__ void __launch_bounds__(256)
k_vec_dot(const float *__restrict__ a, const float *__restrict__ b, const float *__restrict__ c, long long n,
          double *__restrict__ part)
{
    __shared__ double red[8];
    double acc = 0.0;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x)
        acc = fma((double)a[i] - (b ? (double)b[i] : 0.0), (double)c[i], acc);
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += red[w];
        part[blockIdx.x] = t;
    }
}

// per-block partials of |x - xp|^2 and |xp|^2 (the density's relative change)
__global__ void __launch_bounds__(256)
k_rel_change(const float *__restrict__ x, const float *__restrict__ xp, long long n, double *__restrict__ part)
{
    __shared__ double red[2][8];
    double dd = 0.0, pp = 0.0;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        const double a = (double)x[i], b = (double)xp[i];
        dd = fma(a - b, a - b, dd);
        pp = fma(b, b, pp);
    }
    for (int o = 16; o > 0; o >>= 1) {
        dd += __shfl_down_sync(0xffffffffu, dd, o);
        pp += __shfl_down_sync(0xffffffffu, pp, o);
    }
    if ((threadIdx.x & 31) == 0) {
        red[0][threadIdx.x >> 5] = dd;
        red[1][threadIdx.x >> 5] = pp;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double a0 = 0.0, a1 = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) {
            a0 += red[0][w];
            a1 += red[1][w];
        }
        part[2 * blockIdx.x] = a0;
        part[2 * blockIdx.x + 1] = a1;
    }
}

// out = x + alpha g
__global__ void __launch_bounds__(256)
k_axpy(const float *__restrict__ x, const float *__restrict__ g, float alpha, long long n, float *__restrict__ out)
{
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x)
        out[i] = fmaf(alpha, g[i], x[i]);
}

// basis matrix from the saved per-ray projections s (already scaled by Ts):
// A[ie_index(j, i)] = b_j(s_i), a thread per ray.  A block's 128 rays are 32
// whole four-ray blocks, 32 KB contiguous in A: the values are assembled in
// shared memory in A's own layout and written out as 16-byte stores, a warp
// covering 512 contiguous bytes (rows J .. 31 are skipped).
constexpr int kBasisThreads = 128;
__global__ void __launch_bounds__(kBasisThreads)
k_basis_from_s(const float *__restrict__ s, long long nrays, const double *__restrict__ tab_g, int J,
               double *__restrict__ A)
{
    __shared__ double tab[kMaxJ * kSplStride];
    __shared__ __align__(16) double stage[kBasisThreads * 32];
    for (int i = threadIdx.x; i < J * kSplStride; i += blockDim.x) tab[i] = tab_g[i];
    __syncthreads();
    const long long nchunks = (nrays + 3) >> 2;
    for (long long base = (long long)blockIdx.x * kBasisThreads; base < nrays;
         base += (long long)gridDim.x * kBasisThreads) {
        const long long i = base + threadIdx.x;
        double *col = stage + ((threadIdx.x >> 2) * 32) * 4 + (threadIdx.x & 3);   // row j at col[4 j]
        if (i < nrays) {
            const double si = (double)s[i];
            const double is2 = 1.0 / (si * si), as = fabs(si);
            double eL = exp(-tab[0] * si), eC = exp(-tab[1] * si);
            for (int j = 0; j < J; ++j) {
                const double *t = tab + j * kSplStride;
                const double eR = exp(-t[2] * si);
                double bj = ((eC - eR) * t[4] - (eL - eC) * t[3]) * is2;
                if (as < t[9]) bj = fma(fma(fma(t[8], si, t[7]), si, t[6]), si, t[5]);
                col[4 * j] = bj;
                eL = eC;
                eC = eR;
            }
        } else {
            for (int j = 0; j < J; ++j) col[4 * j] = 0.0;
        }
        __syncthreads();
        // 16-byte units e = (block, row, half): block e / 64, row (e / 2) % 32
        const long long c0 = base >> 2;
        const int nunits = (int)min((long long)kBasisThreads / 4, nchunks - c0) * 64;
        const double2 *src = reinterpret_cast<const double2 *>(stage);
        double2 *dst = reinterpret_cast<double2 *>(A + (size_t)c0 * 128);
        for (int e = threadIdx.x; e < nunits; e += kBasisThreads)
            if (((e >> 1) & 31) < J) dst[e] = src[e];
        __syncthreads();
    }
}

}  // namespace ctprj

using namespace ctprj;

namespace {

// device scratch of the spectrum step: the rays x J basis matrix and the
// reduction buffers
struct SpectrumWs {
    double *A = nullptr, *part = nullptr, *fgh = nullptr, *dir = nullptr, *trial = nullptr, *f1 = nullptr;
    double *rr = nullptr, *sq = nullptr;   // per-ray df/dIr and sqrt(curvature)
    int *qp_iters = nullptr;
    int blocks = 0;
    int alloc(int J, long long nr, int nblocks, cudaStream_t s)
    {
        const int w = 1 + J + J * (J + 1) / 2;
        blocks = nblocks;
        int st;
        if ((st = cuda_error(cudaMallocAsync((void **)&A, sizeof(double) * ie_elems(nr), s), "basis matrix")) ||
            (st = cuda_error(cudaMallocAsync((void **)&part, sizeof(double) * nblocks * w, s), "partials")) ||
            (st = cuda_error(cudaMallocAsync((void **)&fgh, sizeof(double) * w, s), "partials")) ||
            (st = cuda_error(cudaMallocAsync((void **)&dir, sizeof(double) * J, s), "partials")) ||
            (st = cuda_error(cudaMallocAsync((void **)&trial, sizeof(double) * (J + 1), s), "partials")) ||
            (st = cuda_error(cudaMallocAsync((void **)&f1, sizeof(double) * 2, s), "partials")) ||
            (st = cuda_error(cudaMallocAsync((void **)&qp_iters, sizeof(int), s), "partials")) ||
            (st = cuda_error(cudaMallocAsync((void **)&rr, sizeof(double) * nr, s), "ray weights")) ||
            (st = cuda_error(cudaMallocAsync((void **)&sq, sizeof(double) * nr, s), "ray weights")))
            release(s);
        return st;
    }
    void release(cudaStream_t s)
    {
        if (A) cudaFreeAsync(A, s);
        if (part) cudaFreeAsync(part, s);
        if (fgh) cudaFreeAsync(fgh, s);
        if (dir) cudaFreeAsync(dir, s);
        if (trial) cudaFreeAsync(trial, s);
        if (f1) cudaFreeAsync(f1, s);
        if (qp_iters) cudaFreeAsync(qp_iters, s);
        if (rr) cudaFreeAsync(rr, s);
        if (sq) cudaFreeAsync(sq, s);
        A = part = fgh = dir = trial = f1 = rr = sq = nullptr;
        qp_iters = nullptr;
    }
};

int sm_count(int dev)
{
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    return sms;
}

// blocks of the spectrum-model kernels: four per SM
int spectrum_grid(int dev) { return 4 * sm_count(dev); }

template <class T>
int fetch(T *h, const T *d, size_t n, cudaStream_t s)
{
    int st = cuda_error(cudaMemcpyAsync(h, d, sizeof(T) * n, cudaMemcpyDeviceToHost, s), "readback");
    if (st) return st;
    return cuda_error(cudaStreamSynchronize(s), "readback sync");
}

// Newton steps on Ie >= 0 over the saved projections m->d_s: model f, g, H
// (k_ie_rays, k_ie_gh), the QP direction (k_ie_qp), then a backtracking line search
// along the feasible direction, step x0.8 (bhc/ActiveSet.m stepShrnk), until
// f(Ie + a d) <= f + 1e-4 g.(a d).  Stops early when g.d >= -1e-14 |f| (the
// model predicts no decrease) or no step decreases f.  *f_out: f at the
// returned Ie.
int spectrum_steps(ctprj_bhc *m, const float *d_imea, double *d_Ie, int newton_steps, double *f_out,
                   SpectrumWs &ws, int *steps_done, cudaStream_t s)
{
    const int J = m->J, w = 1 + J + J * (J + 1) / 2;
    const long long nr = (long long)m->plan->g.np * m->plan->g.W;
    const int dev = m->plan->device;
    k_basis_from_s<<<6 * sm_count(dev), kBasisThreads, 0, s>>>(m->d_s, nr, m->d_tab, J, ws.A);
    int st = cuda_error(cudaGetLastError(), "basis matrix");
    double fcur = 0.0;
    int done = 0;
    for (int it = 0; it < newton_steps && !st; ++it) {
        k_ie_rays<<<ws.blocks, kIeWarps * 32, 0, s>>>(ws.A, d_imea, nr, J, d_Ie, m->noise, w, ws.rr, ws.sq, ws.part);
        k_ie_gh<<<ws.blocks, kGhWarps * 32, 0, s>>>(ws.A, nr, J, ws.rr, ws.sq, w, ws.part);
        k_ie_sum_wide<<<(w + 31) / 32, dim3(32, 32), 0, s>>>(ws.part, ws.blocks, w, w, ws.fgh);
        k_ie_qp<<<1, 32, 0, s>>>(ws.fgh, d_Ie, J, ws.dir, ws.qp_iters);
        if ((st = cuda_error(cudaGetLastError(), "spectrum Newton"))) break;
        if ((st = fetch(&fcur, ws.fgh, 1, s))) break;
        double step = 1.0;
        bool accepted = false, converged = false;
        for (int ls = 0; ls < 40; ++ls, step *= 0.8) {
            k_ie_trial<<<1, 32, 0, s>>>(d_Ie, ws.dir, ws.fgh, J, step, ws.trial);
            k_ie_f<<<ws.blocks, kIeWarps * 32, 0, s>>>(ws.A, d_imea, nr, J, ws.trial, m->noise, w, ws.part);
            k_ie_sum<<<1, 256, 0, s>>>(ws.part, ws.blocks, w, 1, ws.f1);
            double fn = 0.0, gd = 0.0;
            if ((st = cuda_error(cudaMemcpyAsync(&fn, ws.f1, sizeof(double), cudaMemcpyDeviceToHost, s), "readback")) ||
                (st = fetch(&gd, ws.trial + J, 1, s)))
                break;
            if (ls == 0 && !(gd < -1e-14 * fabs(fcur))) {
                converged = true;
                break;
            }
            if (fn <= fcur + 1e-4 * gd) {
                st = cuda_error(cudaMemcpyAsync(d_Ie, ws.trial, sizeof(double) * J, cudaMemcpyDeviceToDevice, s), "accept");
                fcur = fn;
                accepted = true;
                break;
            }
        }
        if (!accepted || converged) break;
        ++done;
    }
    if (f_out) *f_out = fcur;
    if (steps_done) *steps_done = done;
    return st;
}

}  // namespace

extern "C" int ctprj_bhc_spectrum_step(ctprj_bhc *m, const float *d_imea, double *d_Ie, int newton_steps,
                                       double *f_out, void *stream)
{
    if (!m || !d_imea || !d_Ie) return set_error(CTPRJ_EINVAL, "NULL argument");
    if (!m->saved) return set_error(CTPRJ_EINVAL, "the spectrum step needs a saved forward state");
    if (newton_steps < 1) return set_error(CTPRJ_EINVAL, "newton_steps must be >= 1");
    cudaStream_t s = (cudaStream_t)stream;
    SpectrumWs ws;
    int st = ws.alloc(m->J, (long long)m->plan->g.np * m->plan->g.W, spectrum_grid(m->plan->device), s);
    if (st) return st;
    st = spectrum_steps(m, d_imea, d_Ie, newton_steps, f_out, ws, nullptr, s);
    ws.release(s);
    return st;
}

namespace {

// the likelihood at (x, Ie), fused or from the plain projection; the per-ray
// state is saved (the spectrum step and the gradient read it) and the plain
// projection A x is left in sino either way
int likelihood(ctprj_bhc *m, const float *d_x, const double *d_Ie, const float *d_imea, double *d_f,
               bool unfused, float *sino, cudaStream_t s)
{
    if (!unfused) return bhc_forward_keep_projection(m, d_x, d_Ie, d_imea, d_f, sino, s);
    int st = ctprj_forward(m->plan, d_x, sino, s);
    if (st) return st;
    return ctprj_bhc_terms(m, sino, d_Ie, d_imea, d_f, 1, s);
}

struct LoopBufs {
    float *gx = nullptr, *xn = nullptr, *xbar = nullptr, *xprev = nullptr, *sino = nullptr;
    float *v = nullptr;   // input of the TV proximal map
    double *f = nullptr, *part = nullptr, *sum = nullptr;
    void release()
    {
        cudaFree(gx); cudaFree(xn); cudaFree(xbar); cudaFree(xprev); cudaFree(sino); cudaFree(v);
        cudaFree(f); cudaFree(part); cudaFree(sum);
    }
};

double reduce_fetch(const double *part, int nblocks, double *d_out, cudaStream_t s, int *st)
{
    k_ie_sum<<<1, 256, 0, s>>>(part, nblocks, 1, 1, d_out);
    double v = 0.0;
    if (!*st) *st = cuda_error(cudaGetLastError(), "reduction");
    if (!*st) *st = fetch(&v, d_out, 1, s);
    return v;
}

// The initial inverse step t of the density step, as the reference's
// stepSizeInit (npg/Methods.m:98-124):
//   hessian:  t = g'Hg / g'g at x (Hessian of the saved state at x);
//   BB:       t = |(g(x) - g(x - delta)) . delta| / |delta|^2 with delta along g.
// The reference's BB step, |delta| = 1e-5, is below the resolution of a
// single-precision image; here |delta| = 1e-3 |x| (1e-3 for x = 0).
// NaN becomes 1 and 0 becomes DBL_EPSILON, as there; a negative g'Hg (the
// exact Hessian of either model is indefinite far from the data, where the
// reference's NPG then stops with "a negative step size") is taken by its
// magnitude.
int initial_inverse_step(ctprj_bhc *m, const float *d_x, const double *d_Ie, const float *d_imea, int mode,
                         LoopBufs &b, int pgb, double *t_out, cudaStream_t s, const unsigned char *pmask,
                         bool unfused)
{
    const long long npx = (long long)m->plan->g.n * m->plan->g.n;
    int st = 0;
    if ((st = likelihood(m, d_x, d_Ie, d_imea, b.f, unfused, b.sino, s)) ||
        (st = ctprj_bhc_backward(m, nullptr, nullptr, nullptr, b.gx, nullptr, s)))
        return st;
    if (pmask) k_mask_apply<<<pgb, 256, 0, s>>>(b.gx, pmask, npx);
    k_vec_dot<<<pgb, 256, 0, s>>>(b.gx, nullptr, b.gx, npx, b.part);
    const double gg = reduce_fetch(b.part, pgb, b.sum, s, &st);
    if (st) return st;
    double t = NAN;
    if (mode == CTPRJ_STEP_HESSIAN) {
        if ((st = ctprj_bhc_hessian(m, d_Ie, d_imea, b.gx, nullptr, b.sum + 1, s))) return st;
        double gHg = 0.0;
        if ((st = fetch(&gHg, b.sum + 1, 1, s))) return st;
        t = fabs(gHg) / gg;   // the exact Hessian can curve down along g far from the data
    } else {
        k_vec_dot<<<pgb, 256, 0, s>>>(d_x, nullptr, d_x, npx, b.part);
        const double xx = reduce_fetch(b.part, pgb, b.sum, s, &st);
        if (st) return st;
        const double dn = xx > 0.0 ? 1e-3 * sqrt(xx) : 1e-3;
        const double scale = dn / sqrt(gg);   // delta = scale * g
        k_axpy<<<pgb, 256, 0, s>>>(d_x, b.gx, (float)(-scale), npx, b.xbar);
        if ((st = cuda_error(cudaGetLastError(), "BB step")) ||
            (st = likelihood(m, b.xbar, d_Ie, d_imea, b.f, unfused, b.sino, s)) ||
            (st = ctprj_bhc_backward(m, nullptr, nullptr, nullptr, b.xn, nullptr, s)))
            return st;
        if (pmask) k_mask_apply<<<pgb, 256, 0, s>>>(b.xn, pmask, npx);
        k_vec_dot<<<pgb, 256, 0, s>>>(b.gx, b.xn, b.gx, npx, b.part);
        const double dgd = reduce_fetch(b.part, pgb, b.sum, s, &st) * scale;
        if (st) return st;
        t = fabs(dgd) / (scale * scale * gg);
    }
    if (std::isnan(t)) t = 1.0;
    if (t == 0.0) t = DBL_EPSILON;
    *t_out = t;
    return CTPRJ_OK;
}

}  // namespace

// The density step follows the reference's NPG class (npg/NPG.m main, with
// the projection on x >= 0, the TV denoising of tv.cu or the wavelet ADMM of
// wavelet.cu as the proximal map), or its PG class (npg/PG.m: the same
// without extrapolation and restart):
//   theta' = (1 + sqrt(1 + 4 theta^2)) / 2,  xbar = max(0, x + (theta-1)/theta' (x - xprev));
//   f, grad at xbar;  candidate xn = max(0, xbar - grad / t), accepted when
//   f(xn) <= f(xbar) + grad.(xn - xbar) + t/2 |xn - xbar|^2 (utils/Utils.m
//   majorizationHolds); on failure t /= 0.5 (at most 20 times); in the first
//   preSteps iterations a success is retried with t *= 0.5 while it holds (at
//   most 17 times); after 4 consecutive first-try successes t *= 0.5 once (failure
//   of that try raises the count needed by 4);
//   if f(xn) exceeds the cost of the previous iteration: restart without
//   momentum (theta = 1) when xbar != x, else keep x when the majorisation
//   failed or f(xbar) < f(xn) (PG: keep x when the majorisation failed or the
//   cost rose).  With a TV map the candidate is TV.denoise(xbar - grad / t,
//   u / t) to tolerance admmTol * difAlpha (with the wavelet map admm(..., x)),
//   the cost carries u TV (u |Psit x|_1), and before
//   x is kept the step is retried with admmTol / 10 (down to 1e-6) or
//   maxInnerItr * 10 (up to 1000); those retries cannot change an exact
//   projection and are not taken for it.  The reference's reset of t to the
//   Hessian estimate after a failed majorisation is not taken.
// Then the spectrum step on the accepted density's projections, whose f
// becomes the cost the next density step compares against
// (bhc/beamhardenSpline.m:382-470).
extern "C" int ctprj_bhc_reconstruct(ctprj_bhc *m, float *d_x, double *d_Ie, const float *d_imea,
                                     const ctprj_bhc_loop_opts *opts, ctprj_bhc_loop_stats *stats,
                                     void *stream)
{
    if (!m || !d_x || !d_Ie || !d_imea || !opts) return set_error(CTPRJ_EINVAL, "NULL argument");
    if (opts->iterations < 0) return set_error(CTPRJ_EINVAL, "negative iteration count");
    const int prox = opts->proximal;
    if (prox != CTPRJ_PROX_NONNEG && prox != CTPRJ_PROX_TV_ISO && prox != CTPRJ_PROX_TV_L1 &&
        prox != CTPRJ_PROX_WVLT_ADMM)
        return set_error(CTPRJ_EINVAL, "unknown proximal map %d", prox);
    const bool tv = prox == CTPRJ_PROX_TV_ISO || prox == CTPRJ_PROX_TV_L1;
    const bool wv = prox == CTPRJ_PROX_WVLT_ADMM;
    const bool reg = tv || wv;   // a regulariser with an iterative proximal map
    if (reg && !(opts->u > 0.0)) return set_error(CTPRJ_EINVAL, "the regularised proximal maps need u > 0");
    if (reg && (long long)m->plan->g.n * m->plan->g.n >= (1LL << 31))
        return set_error(CTPRJ_EINVAL, "the regularised proximal maps need an image below 2^31 pixels");
    // the wavelet: Utils.getPsiPsit(daub, dwt_L) filter and levels, by default
    // daub = 2 (Haar) and dwt_L = 6 as the reference's BHC runs (bhc/doBHC.m:33)
    double wh[CTPRJ_WVLT_MAX_FILTER];
    const int wlh = opts->wvlt_filter_len > 0 ? opts->wvlt_filter_len : 2;
    const int wlev = opts->wvlt_levels > 0 ? opts->wvlt_levels : 6;
    if (wv) {
        if (wlh > CTPRJ_WVLT_MAX_FILTER || (wlh & 1))
            return set_error(CTPRJ_EINVAL, "wavelet filter length %d: even, at most %d", wlh, CTPRJ_WVLT_MAX_FILTER);
        for (int j = 0; j < wlh; ++j) wh[j] = opts->wvlt_filter_len > 0 ? opts->wvlt_filter[j] : M_SQRT1_2;
        if (wlev > 30 || m->plan->g.n % (1 << wlev))
            return set_error(CTPRJ_EINVAL, "image side %d not divisible by 2^%d wavelet levels", m->plan->g.n, wlev);
    }
    PlanDevice pd(m->plan->device);
    cudaStream_t s = (cudaStream_t)stream;
    const long long npx = (long long)m->plan->g.n * m->plan->g.n;
    const long long nr = (long long)m->plan->g.np * m->plan->g.W;
    const int dev = m->plan->device;
    const int pgb = 2 * sm_count(dev);
    LoopBufs b;
    SpectrumWs ws;
    TvWorkspace tvw;
    WvltProx wws;
    const int n = m->plan->g.n;
    const unsigned char *pmask = opts->mask;       // NULL: the whole image
    const unsigned char *cmask = opts->wvlt_mask;  // NULL: derived from pmask, or all coefficients
    unsigned char *own_cmask = nullptr;
    int st;
    if ((st = cuda_error(cudaMalloc((void **)&b.gx, sizeof(float) * npx), "loop buffers")) ||
        (st = cuda_error(cudaMalloc((void **)&b.xn, sizeof(float) * npx), "loop buffers")) ||
        (st = cuda_error(cudaMalloc((void **)&b.xbar, sizeof(float) * npx), "loop buffers")) ||
        (st = cuda_error(cudaMalloc((void **)&b.xprev, sizeof(float) * npx), "loop buffers")) ||
        (st = cuda_error(cudaMalloc((void **)&b.f, sizeof(double) * 2), "loop buffers")) ||
        (st = cuda_error(cudaMalloc((void **)&b.part, sizeof(double) * 2 * pgb), "loop buffers")) ||
        (st = cuda_error(cudaMalloc((void **)&b.sum, sizeof(double) * 4), "loop buffers")) ||
        (reg && (st = cuda_error(cudaMalloc((void **)&b.v, sizeof(float) * npx), "loop buffers"))) ||
        (tv && (st = tvw.alloc(n, n, s))) ||
        (wv && (st = wws.alloc(n, n, s))) ||
        (st = cuda_error(cudaMalloc((void **)&b.sino, sizeof(float) * nr), "loop buffers")) ||
        (!opts->skip_spectrum && (st = ws.alloc(m->J, nr, spectrum_grid(dev), s)))) {
        tvw.release(s);
        wws.release(s);
        cudaStreamSynchronize(s);
        b.release();
        return st;
    }
    const int newton = opts->spectrum_newton_steps > 0 ? opts->spectrum_newton_steps : 2;
    const bool pg = opts->density_method == CTPRJ_DENSITY_PG;
    double t = 1.0 / (opts->x_step > 0 ? opts->x_step : 1.0);   // inverse step size
    double theta = 0.0, cost = INFINITY;
    int p = 0, cumu = 0, cumu_tol = opts->cumu_tol > 0 ? opts->cumu_tol : 4, evals = 0, restarts = 0,
        newton_done = 0, conv = 0, converged = 0;
    const bool adaptive = !opts->no_adaptive_step, restart_on = !opts->no_restart;
    // opt.preSteps, which the BHC driver sets on its NPG / PG object
    // (bhc/beamhardenSpline.m:74, :304; the classes' own default is 10)
    const int pre_steps = opts->pre_steps > 0 ? opts->pre_steps : 2;
    const double shrink = 0.5;
    // the iterative proximal maps' state (npg/NPG.m:11,23-24 and Methods.m difAlpha = 1)
    const bool iso = prox == CTPRJ_PROX_TV_ISO;
    const int max_pass = reg ? 12 : 3;
    double admm_tol = opts->admm_tol > 0.0 ? opts->admm_tol : 1e-2, dif_alpha = 1.0, pen = 0.0;
    int max_inner = opts->max_inner > 0 ? opts->max_inner : 100, inner = 0, inner_total = 0, retries = 0;
    auto penalty_of = [&](const float *v, double *out) -> int {   // u TV(v) or u |Psit(v)|_1
        double tvv = 0.0;
        int e = tv ? tv_value(tvw, v, n, n, iso, b.sum + 3, s)
                   : wvlt_l1(wws, v, n, n, wh, wlh, wlev, b.sum + 3, s, cmask);
        if (!e) e = fetch(&tvv, b.sum + 3, 1, s);
        *out = opts->u * tvv;
        return e;
    };
    // a rejected regularised step is retried with a tighter inner tolerance or, when the
    // inner iteration ran out, more inner iterations (npg/NPG.m:117-128)
    auto retry = [&]() -> bool {
        if (inner < max_inner && admm_tol > 1e-6)
            admm_tol /= 10.0;
        else if (inner >= max_inner && max_inner < 1000)
            max_inner *= 10;
        else
            return false;
        ++retries;
        return true;
    };
    float ms_spec = 0.0f;
    cudaEvent_t e0, e1, es0, es1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventCreate(&es0);
    cudaEventCreate(&es1);
    // alpha = max(alpha, 0) before the NPG / PG object is built (bhc/beamhardenSpline.m:232,236)
    k_npg_extrapolate<<<pgb, 256, 0, s>>>(d_x, d_x, npx, 0.0f, d_x, b.part);
    if (pmask) k_mask_apply<<<pgb, 256, 0, s>>>(d_x, pmask, npx);
    st = cuda_error(cudaGetLastError(), "loop start");
    // the wavelet coefficients of the masked transform: given, or those the
    // mask's pixels reach (utils/wvltMask.m)
    if (!st && wv && pmask && !cmask) {
        if (!(st = cuda_error(cudaMalloc((void **)&own_cmask, (size_t)npx), "wavelet mask")) &&
            !(st = wvlt_mask(wws, pmask, n, n, wh, wlh, wlev, own_cmask, s)))
            cmask = own_cmask;
    }
    if (!st)
        st = cuda_error(cudaMemcpyAsync(b.xprev, d_x, sizeof(float) * npx, cudaMemcpyDeviceToDevice, s), "loop start");
    cudaEventRecord(e0, s);
    if (!st && opts->init_step != CTPRJ_STEP_FIXED) {
        st = initial_inverse_step(m, d_x, d_Ie, d_imea, opts->init_step, b, pgb, &t, s, opts->mask,
                                  opts->unfused != 0);
        evals += opts->init_step == CTPRJ_STEP_BB ? 2 : 1;
    }
    int done = 0;
    // b.sino holds A x for the current x: PG's next extrapolated point is x
    // itself, so its likelihood needs no new projection, only the terms at the
    // current spectrum (the same sums: the projection is deterministic)
    bool proj_at_x = false;
    for (int it = 0; it < opts->iterations && !st; ++it) {
        double nc = 0.0, obj = 0.0;
        bool moved = false, state_at_x = false;
        for (int pass = 0; pass < max_pass && !st; ++pass) {
            const bool last = pass == max_pass - 1;
            ++p;
            const double theta1 = (1.0 + sqrt(1.0 + 4.0 * theta * theta)) / 2.0;
            const float coef = pg ? 0.0f : (float)((theta - 1.0) / theta1);
            k_npg_extrapolate<<<pgb, 256, 0, s>>>(d_x, b.xprev, npx, coef, b.xbar, b.part);
            k_ie_sum<<<1, 256, 0, s>>>(b.part, pgb, 2, 1, b.sum + 1);
            double f0 = 0.0, mom = 0.0;
            if ((st = cuda_error(cudaGetLastError(), "extrapolation")) ||
                (st = (pg && proj_at_x) ? ctprj_bhc_terms(m, b.sino, d_Ie, d_imea, b.f, 1, s)
                                        : likelihood(m, b.xbar, d_Ie, d_imea, b.f, opts->unfused != 0, b.sino, s)) ||
                (st = ctprj_bhc_backward(m, nullptr, nullptr, nullptr, b.gx, nullptr, s)))
                break;
            proj_at_x = pg;   // xbar = x for PG
            if (pmask) k_mask_apply<<<pgb, 256, 0, s>>>(b.gx, pmask, npx);   // the masked gradient
            if ((st = cuda_error(cudaMemcpyAsync(&mom, b.sum + 1, sizeof(double), cudaMemcpyDeviceToHost, s), "readback")) ||
                (st = fetch(&f0, b.f, 1, s)))
                break;
            ++evals;
            int ppp = 0;
            bool good = true, inc = false, good_mm = true;
            if (adaptive && cumu >= cumu_tol) {   // adaptively grow the step
                t *= shrink;
                cumu = 0;
                inc = true;
            }
            while (true) {
                ++ppp;
                if (reg) {   // xn = proxmapping(xbar - g / t, u / t, admmTol difAlpha, maxInnerItr, x)
                    k_axpy<<<pgb, 256, 0, s>>>(b.xbar, b.gx, (float)(-1.0 / t), npx, b.v);
                    if ((st = cuda_error(cudaGetLastError(), "density step"))) break;
                    if (tv) {   // TV.denoise (utils/TV.m:56-80), which starts from D = 0
                        st = tv_denoise(tvw, b.v, n, n, opts->u / t, 0.0, INFINITY, iso, max_inner,
                                        admm_tol * dif_alpha, b.xn, &inner, s);
                        if (!st && pmask) k_mask_apply<<<pgb, 256, 0, s>>>(b.xn, pmask, npx);   // mask.a
                    } else {    // admm(Psi, Psit, ., init = x) (npg/admm.m)
                        st = wvlt_admm(wws, b.v, n, n, wh, wlh, wlev, opts->u / t, admm_tol * dif_alpha, max_inner,
                                       d_x, b.xn, &inner, s, pmask, cmask);
                    }
                    if (st) break;
                    inner_total += inner;
                    k_step_terms<<<pgb, 256, 0, s>>>(b.xbar, b.gx, b.xn, npx, b.part);
                } else {
                    k_pg_step<<<pgb, 256, 0, s>>>(b.xbar, b.gx, npx, (float)(1.0 / t), b.xn, b.part);
                }
                k_ie_sum<<<1, 256, 0, s>>>(b.part, pgb, 2, 2, b.sum);
                double gd_dd[2];
                if ((st = cuda_error(cudaGetLastError(), "density step")) ||
                    (st = likelihood(m, b.xn, d_Ie, d_imea, b.f + 1, opts->unfused != 0, b.sino, s)) ||
                    (st = cuda_error(cudaMemcpyAsync(gd_dd, b.sum, 2 * sizeof(double), cudaMemcpyDeviceToHost, s), "readback")) ||
                    (st = fetch(&nc, b.f + 1, 1, s)))
                    break;
                proj_at_x = false;   // b.sino now holds A xn
                ++evals;
                if (nc - f0 <= gd_dd[0] + 0.5 * t * gd_dd[1]) {
                    if (p <= pre_steps && ppp < 18 && good) {
                        t *= shrink;
                        continue;
                    }
                    break;
                }
                if (ppp <= 20) {
                    t /= shrink;
                    good = false;
                    if (inc) {
                        cumu_tol += 4;
                        inc = false;
                    }
                } else {
                    good_mm = false;
                    break;
                }
            }
            if (st) break;
            if (reg && (st = penalty_of(b.xn, &pen))) break;
            obj = nc + pen;
            moved = true;
            if (pg) {
                if (!good_mm || obj > cost) {
                    if (reg && !last && retry()) continue;
                    moved = false;                          // npg/PG.m: force convergence
                }
            } else if (obj > cost) {
                if (good_mm && mom != 0.0 && restart_on && !last) {   // restart without momentum
                    theta = 1.0;
                    ++restarts;
                    continue;
                }
                double pen_bar = 0.0;
                if (reg && good_mm && (st = penalty_of(b.xbar, &pen_bar))) break;
                if (!good_mm || f0 + pen_bar < obj) {
                    if (!good_mm) theta = 1.0;              // NPG's reset() (its t reset is not taken)
                    if (reg && !last && retry()) continue;
                    moved = false;                          // npg/NPG.m: force convergence
                }
            }
            if (!moved) obj = cost;   // keep x
            theta = theta1;
            st = cuda_error(cudaMemcpyAsync(b.xprev, d_x, sizeof(float) * npx, cudaMemcpyDeviceToDevice, s), "accept");
            if (!st && moved)
                st = cuda_error(cudaMemcpyAsync(d_x, b.xn, sizeof(float) * npx, cudaMemcpyDeviceToDevice, s), "accept");
            if (!st && reg) {   // difAlpha = relativeDif(x, x_new), the next inner tolerance's scale
                k_rel_change<<<pgb, 256, 0, s>>>(b.xprev, d_x, npx, b.part);
                k_ie_sum<<<1, 256, 0, s>>>(b.part, pgb, 2, 2, b.sum);
                double dq[2];
                if (!(st = cuda_error(cudaGetLastError(), "relative change")) && !(st = fetch(dq, b.sum, 2, s)))
                    dif_alpha = sqrt(dq[0]) / fmax(sqrt(dq[1]), 1e-10);
            }
            state_at_x = moved;   // the last likelihood evaluated (and saved) was at xn
            proj_at_x = moved;
            cumu = (ppp == 1 && adaptive) ? cumu + 1 : 0;
            break;
        }
        if (st) break;
        cost = obj;
        if (stats && it < CTPRJ_BHC_LOOP_MAX_TRACE) stats->x_step[it] = moved ? 1.0 / t : 0.0;
        if (!opts->skip_spectrum) {
            cudaEventRecord(es0, s);
            if (!state_at_x) {
                if ((st = likelihood(m, d_x, d_Ie, d_imea, b.f, opts->unfused != 0, b.sino, s))) break;
                proj_at_x = true;
                ++evals;
            }
            double fs = 0.0;
            int nd = 0;
            if ((st = spectrum_steps(m, d_imea, d_Ie, newton, &fs, ws, &nd, s))) break;
            newton_done += nd;
            cudaEventRecord(es1, s);
            cudaEventSynchronize(es1);
            float ms = 0.0f;
            cudaEventElapsedTime(&ms, es0, es1);
            ms_spec += ms;
            // alphaStep.cost = IeStep.cost + u fVal(3) (bhc/beamhardenSpline.m:460): the
            // penalty of the last density candidate, also when it was not accepted
            cost = fs + pen;
        }
        if (stats && it < CTPRJ_BHC_LOOP_MAX_TRACE) stats->cost[it] = cost;
        done = it + 1;
        // relativeDif(x_new, x) of the reference loop; xprev holds this
        // iteration's starting density
        k_rel_change<<<pgb, 256, 0, s>>>(d_x, b.xprev, npx, b.part);
        k_ie_sum<<<1, 256, 0, s>>>(b.part, pgb, 2, 2, b.sum);
        double dp[2];
        if ((st = cuda_error(cudaGetLastError(), "relative change")) || (st = fetch(dp, b.sum, 2, s))) break;
        const double change = sqrt(dp[0]) / fmax(sqrt(dp[1]), 1e-10);
        if (stats && it < CTPRJ_BHC_LOOP_MAX_TRACE) stats->x_change[it] = change;
        if (opts->thresh > 0.0 && it > 0 && change <= opts->thresh) ++conv;
        if (conv > 2 && done > opts->min_iterations) {
            converged = 1;
            break;
        }
    }
    cudaEventRecord(e1, s);
    cudaEventSynchronize(e1);
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaEventDestroy(es0);
    cudaEventDestroy(es1);
    if (stats) {
        stats->iterations = done;
        stats->final_cost = cost;
        stats->final_x_step = 1.0 / t;
        stats->ms = ms;
        stats->ms_spectrum = ms_spec;
        stats->evaluations = evals;
        stats->restarts = restarts;
        stats->newton_steps = newton_done;
        stats->converged = converged;
        stats->inner_iterations = inner_total;
        stats->prox_retries = retries;
        stats->penalty = pen;
    }
    ws.release(s);
    tvw.release(s);
    wws.release(s);
    cudaStreamSynchronize(s);
    cudaFree(own_cmask);
    b.release();
    return st;
}

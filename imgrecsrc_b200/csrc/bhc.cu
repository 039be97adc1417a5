// bhc.cu -- polychromatic beam-hardening model on a projector plan.
//
// Forward (bhc/poissLAlpha.m:1-13 with Phi = Ts A): for every ray i,
// s_i = Ts (A x)_i, BL_i = sum_j Ie_j b_j(s_i), the Poisson negative
// log-likelihood f = sum_i BL_i - m_i - m_i log(BL_i / m_i) reduced in FP64.
// The spline evaluation is fused into the forward projection kernel as a per-ray
// epilogue (projector.cu, kModeBhc); the sinogram itself is never written.
// Backward: df/dx = Ts A^T [(1 - m/BL) dBL/ds] (the plain backprojector with an
// output scale) and df/dIe_j = sum_i b_j(s_i) (1 - m_i/BL_i) (bhc/poissLI.m:2-6)
// accumulated in FP64 by k_bhc_spectrum.
#include <cmath>
#include <cstring>
#include <vector>

#include "ctprj_internal.h"
#include "bhc_spline.cuh"

namespace ctprj {

constexpr int kSpecThreads = 256;
constexpr int kTermThreads = 256;

__device__ __forceinline__ double block_sum_any(double v, double *red)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) red[warp] = v;
    __syncthreads();
    double t = 0.0;
    if (threadIdx.x == 0)
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += red[w];
    __syncthreads();
    return t;
}

// df/dIe_j = sum_i b_j(s_i) r_i, per-block partials part[block * J + j].
// The basis functions are taken kSpecChunk at a time, so that a thread keeps
// only that many FP64 accumulators in registers (two extra exponentials per
// chunk and ray restart the rolling product).  Two blocks of 256 threads per
// SM with 16 functions per chunk (114 registers): 0.28 ms at the 2048^2 fan
// workload with J = 30, against 0.48 ms for one block with 8 per chunk, 0.31
// for two with 8 and 0.41 for two with 32 (174 registers, one block resident).
#ifndef CTPRJ_SPEC_CHUNK
#define CTPRJ_SPEC_CHUNK 16
#endif
#ifndef CTPRJ_SPEC_BLOCKS_PER_SM
#define CTPRJ_SPEC_BLOCKS_PER_SM 2
#endif
constexpr int kSpecChunk = CTPRJ_SPEC_CHUNK;

__global__ void __launch_bounds__(kSpecThreads)
k_bhc_spectrum(const float *__restrict__ s, const double *__restrict__ r, long long nrays,
               const double *__restrict__ tab_g, int J, double *__restrict__ part)
{
    __shared__ double tab[kMaxJ * kSplStride];
    __shared__ double red[kSpecThreads / 32][kMaxJ];
    for (int i = threadIdx.x; i < J * kSplStride; i += blockDim.x) tab[i] = tab_g[i];
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int j0 = 0; j0 < J; j0 += kSpecChunk) {
        double acc[kSpecChunk];
#pragma unroll
        for (int q = 0; q < kSpecChunk; ++q) acc[q] = 0.0;
        const double *t0 = tab + j0 * kSplStride;
        for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < nrays;
             i += (long long)gridDim.x * blockDim.x) {
            const double si = (double)s[i], ri = r[i];
            const double is2 = 1.0 / (si * si), as = fabs(si);
            double eL = exp(-t0[0] * si), eC = exp(-t0[1] * si);
#pragma unroll
            for (int q = 0; q < kSpecChunk; ++q) {
                if (j0 + q < J) {
                    const double *t = t0 + q * kSplStride;
                    const double eR = exp(-t[2] * si);
                    double bj = ((eC - eR) * t[4] - (eL - eC) * t[3]) * is2;
                    if (as < t[9]) bj = fma(fma(fma(t[8], si, t[7]), si, t[6]), si, t[5]);
                    acc[q] = fma(bj, ri, acc[q]);
                    eL = eC;
                    eC = eR;
                }
            }
        }
#pragma unroll
        for (int q = 0; q < kSpecChunk; ++q) {
            double v = acc[q];
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
            if (lane == 0 && j0 + q < J) red[warp][j0 + q] = v;
        }
    }
    __syncthreads();
    if (threadIdx.x < J) {
        double t = 0.0;
        for (int w = 0; w < kSpecThreads / 32; ++w) t += red[w][threadIdx.x];
        part[(size_t)blockIdx.x * J + threadIdx.x] = t;
    }
}

// Unfused polychromatic terms over a sinogram from the plain projector (the
// same per-ray math as the fused epilogue), per-block partials of f.
__global__ void __launch_bounds__(kTermThreads)
k_bhc_terms(const float *__restrict__ sino, long long nrays, BhcArgs a)
{
    __shared__ double sm[kMaxJ * (kSplStride + 1)];
    __shared__ double red[kTermThreads / 32];
    for (int i = threadIdx.x; i < a.J * kSplStride; i += blockDim.x) sm[i] = a.tab[i];
    for (int i = threadIdx.x; i < a.J; i += blockDim.x) sm[kMaxJ * kSplStride + i] = a.Ie[i];
    __syncthreads();
    const double *tab = sm, *Ie = sm + kMaxJ * kSplStride;
    double f = 0.0;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < nrays;
         i += (long long)gridDim.x * blockDim.x) {
        const double s = a.Ts * (double)sino[i];
        const SplineEval e = b1_eval(s, tab, Ie, a.J);
        const double m = (double)a.imea[i];
        const RayTerms t = ray_terms(a.noise, e.BL, m);
        if (a.w_out) {
            a.w_out[i] = (float)(t.r * e.sBL);
            a.s_out[i] = (float)s;
            a.r_out[i] = t.r;
        }
        f += t.f;
    }
    const double t = block_sum_any(f, red);
    if (threadIdx.x == 0) a.part[blockIdx.x] = t;
}

// The rays x J basis matrix A[i][j] = b_j(Ts * sino_i) in FP64 (Spline.b1Iout
// with I empty, bhc/Spline.m:143, :168), materialised as the reference's
// spectrum step does (bhc/beamhardenSpline.m:447).
__global__ void __launch_bounds__(256)
k_bhc_basis(const float *__restrict__ sino, long long nrays, const double *__restrict__ tab_g,
            int J, double Ts, double *__restrict__ A)
{
    __shared__ double tab[kMaxJ * kSplStride];
    for (int i = threadIdx.x; i < J * kSplStride; i += blockDim.x) tab[i] = tab_g[i];
    __syncthreads();
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < nrays;
         i += (long long)gridDim.x * blockDim.x) {
        const double si = Ts * (double)sino[i];
        const double is2 = 1.0 / (si * si), as = fabs(si);
        double eL = exp(-tab[0] * si), eC = exp(-tab[1] * si);
        double *row = A + (size_t)i * J;
        for (int j = 0; j < J; ++j) {
            const double *t = tab + j * kSplStride;
            const double eR = exp(-t[2] * si);
            double bj = ((eC - eR) * t[4] - (eL - eC) * t[3]) * is2;
            if (as < t[9]) bj = fma(fma(fma(t[8], si, t[7]), si, t[6]), si, t[5]);
            row[j] = bj;
            eL = eC;
            eC = eR;
        }
    }
}

// out[c] = sum over b < nrows of part[b * ncols + c], in a fixed order (FP64)
__global__ void k_sum_columns(const double *__restrict__ part, int nrows, int ncols,
                              double *__restrict__ out)
{
    sum_partials(part, nrows, ncols, ncols, out);
}

static int spectrum_blocks()
{
    int dev = 0, sms = 148;
    if (cudaGetDevice(&dev) == cudaSuccess)
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    return sms;   // one block of 256 threads per SM
}

// blocks of the spectrum-gradient kernel
static int spectrum_grad_blocks() { return CTPRJ_SPEC_BLOCKS_PER_SM * spectrum_blocks(); }

// per basis function: a, b, c, 1/(a-b), 1/(b-c), Taylor B[4], thrB, Taylor D[4], thrD
// (bhc/Spline.m:154-181; threshold |EPS c0 / c3|^(1/3), EPS = 1e-6)
static std::vector<double> spline_table(const double *k, int J)
{
    std::vector<double> t((size_t)J * kSplStride);
    for (int j = 0; j < J; ++j) {
        const double a = k[j], b = k[j + 1], c = k[j + 2];
        double *e = &t[(size_t)j * kSplStride];
        e[0] = a; e[1] = b; e[2] = c;
        e[3] = 1.0 / (a - b);
        e[4] = 1.0 / (b - c);
        const double B[4] = {-a / 2 + c / 2,
                             (a * a * a - b * b * b) / (6 * (a - b)) - (b * b * b - c * c * c) / (6 * (b - c)),
                             -(pow(a, 4) - pow(b, 4)) / (24 * (a - b)) + (pow(b, 4) - pow(c, 4)) / (24 * (b - c)),
                             (pow(a, 5) - pow(b, 5)) / (120 * (a - b)) - (pow(b, 5) - pow(c, 5)) / (120 * (b - c))};
        const double D[4] = {B[1],
                             -(pow(a, 4) - pow(b, 4)) / (12 * (a - b)) + (pow(b, 4) - pow(c, 4)) / (12 * (b - c)),
                             (pow(a, 5) - pow(b, 5)) / (40 * (a - b)) - (pow(b, 5) - pow(c, 5)) / (40 * (b - c)),
                             -(pow(a, 6) - pow(b, 6)) / (180 * (a - b)) + (pow(b, 6) - pow(c, 6)) / (180 * (b - c))};
        for (int q = 0; q < 4; ++q) {
            e[5 + q] = B[q];
            e[10 + q] = D[q];
        }
        e[9] = cbrt(fabs(1e-6 * B[0] / B[3]));
        e[14] = cbrt(fabs(1e-6 * D[0] / D[3]));
    }
    return t;
}

// per basis function: the cubic Taylor coefficients of b_j'' about s = 0 and
// the |s| below which they are used (bhc/Spline.m:186-197, same 1e-6 rule)
static std::vector<double> spline_table2(const double *k, int J)
{
    std::vector<double> t((size_t)J * kSpl2Stride);
    for (int j = 0; j < J; ++j) {
        const double a = k[j], b = k[j + 1], c = k[j + 2];
        double *e = &t[(size_t)j * kSpl2Stride];
        e[0] = -((a + b) * (a * a + b * b)) / 12 + ((b + c) * (b * b + c * c)) / 12;
        e[1] = (pow(a, 4) + pow(a, 3) * b + a * a * b * b + a * pow(b, 3) + pow(b, 4)) / 20 -
               (pow(b, 4) + pow(b, 3) * c + b * b * c * c + b * pow(c, 3) + pow(c, 4)) / 20;
        e[2] = -((a + b) * (a * a + a * b + b * b) * (a * a - a * b + b * b)) / 60 +
               ((b + c) * (b * b + b * c + c * c) * (b * b - b * c + c * c)) / 60;
        e[3] = (pow(a, 6) + pow(a, 5) * b + pow(a, 4) * b * b + pow(a, 3) * pow(b, 3) + a * a * pow(b, 4) +
                a * pow(b, 5) + pow(b, 6)) / 252 -
               (pow(b, 6) + pow(b, 5) * c + pow(b, 4) * c * c + pow(b, 3) * pow(c, 3) + b * b * pow(c, 4) +
                b * pow(c, 5) + pow(c, 6)) / 252;
        e[4] = cbrt(fabs(1e-6 * e[0] / e[3]));
    }
    return t;
}

// Density Hessian weight per ray at the saved s: y = Ts (Phi v) in, h y out
// (the backprojection input), per-block partials of sum h y^2.
__global__ void __launch_bounds__(kTermThreads)
k_bhc_hess(const float *__restrict__ s_saved, float *__restrict__ y, long long nrays, BhcArgs a,
           const double *__restrict__ tab2_g)
{
    __shared__ double sm[kMaxJ * (kSplStride + kSpl2Stride + 1)];
    __shared__ double red[kTermThreads / 32];
    for (int i = threadIdx.x; i < a.J * kSplStride; i += blockDim.x) sm[i] = a.tab[i];
    for (int i = threadIdx.x; i < a.J * kSpl2Stride; i += blockDim.x) sm[kMaxJ * kSplStride + i] = tab2_g[i];
    for (int i = threadIdx.x; i < a.J; i += blockDim.x) sm[kMaxJ * (kSplStride + kSpl2Stride) + i] = a.Ie[i];
    __syncthreads();
    const double *tab = sm, *tab2 = sm + kMaxJ * kSplStride, *Ie = sm + kMaxJ * (kSplStride + kSpl2Stride);
    double q = 0.0;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < nrays;
         i += (long long)gridDim.x * blockDim.x) {
        const SplineEval2 e = b1_eval2((double)s_saved[i], tab, tab2, Ie, a.J);
        const double m = (double)a.imea[i];
        const double h = ray_curvature(a.noise, e.BL, m) * e.sBL * e.sBL + ray_terms(a.noise, e.BL, m).r * e.ssBL;
        const double yi = a.Ts * (double)y[i];
        y[i] = (float)(h * yi);
        q = fma(h * yi, yi, q);
    }
    q = block_sum_any(q, red);
    if (threadIdx.x == 0) a.part[blockIdx.x] = q;
}

}  // namespace ctprj

using namespace ctprj;

extern "C" void ctprj_bhc_destroy(ctprj_bhc *m);

static int ensure_parts(ctprj_bhc *m, int need)
{
    if (m->part_cap >= need) return CTPRJ_OK;
    cudaFree(m->d_part);
    m->d_part = nullptr;
    m->part_cap = 0;
    int st = cuda_error(cudaMalloc((void **)&m->d_part, sizeof(double) * (size_t)need),
                        "partials allocation");
    if (!st) m->part_cap = need;
    return st;
}

extern "C" int ctprj_bhc_create(ctprj_plan *plan, int J, const double *kappa_nodes, double Ts,
                                ctprj_bhc **out)
{
    if (!plan || !kappa_nodes || !out) return set_error(CTPRJ_EINVAL, "NULL argument");
    *out = nullptr;
    if (J < 1 || J > kMaxJ) return set_error(CTPRJ_ERANGE, "J must be in [1, %d] (J=%d)", kMaxJ, J);
    if (!(Ts > 0) || !std::isfinite(Ts)) return set_error(CTPRJ_EINVAL, "Ts must be positive");
    for (int j = 0; j < J + 2; ++j)
        if (!(kappa_nodes[j] > 0) || (j > 0 && !(kappa_nodes[j] > kappa_nodes[j - 1])))
            return set_error(CTPRJ_EINVAL, "kappa nodes must be positive and increasing");
    PlanDevice pd(plan->device);
    ctprj_bhc *m = new (std::nothrow) ctprj_bhc();
    if (!m) return set_error(CTPRJ_ENOMEM, "host allocation failed");
    memset(m, 0, sizeof *m);
    m->plan = plan;
    m->J = J;
    m->Ts = Ts;
    const std::vector<double> tab = spline_table(kappa_nodes, J);
    const std::vector<double> tab2 = spline_table2(kappa_nodes, J);
    const size_t nr = (size_t)plan->g.np * plan->g.W;
    int st;
    if ((st = cuda_error(cudaMalloc((void **)&m->d_tab, sizeof(double) * tab.size()), "spline table")) ||
        (st = cuda_error(cudaMemcpy(m->d_tab, tab.data(), sizeof(double) * tab.size(),
                                    cudaMemcpyHostToDevice), "spline upload")) ||
        (st = cuda_error(cudaMalloc((void **)&m->d_tab2, sizeof(double) * tab2.size()), "spline table")) ||
        (st = cuda_error(cudaMemcpy(m->d_tab2, tab2.data(), sizeof(double) * tab2.size(),
                                    cudaMemcpyHostToDevice), "spline upload")) ||
        (st = cuda_error(cudaMalloc((void **)&m->d_s, sizeof(float) * nr), "ray state")) ||
        (st = cuda_error(cudaMalloc((void **)&m->d_r, sizeof(double) * nr), "ray state")) ||
        (st = cuda_error(cudaMalloc((void **)&m->d_w, sizeof(float) * nr), "ray state"))) {
        cudaFree(m->d_tab); cudaFree(m->d_tab2); cudaFree(m->d_s); cudaFree(m->d_r); cudaFree(m->d_w);
        delete m;
        return st;
    }
    // partials for every reduction this model launches, sized once
    int need = forward_blocks(plan);
    if (need < 4 * spectrum_blocks()) need = 4 * spectrum_blocks();
    if (need < spectrum_grad_blocks() * J) need = spectrum_grad_blocks() * J;
    if ((st = ensure_parts(m, need))) {
        ctprj_bhc_destroy(m);
        return st;
    }
    *out = m;
    return CTPRJ_OK;
}

extern "C" void ctprj_bhc_destroy(ctprj_bhc *m)
{
    if (!m) return;
    PlanDevice pd(m->plan->device);
    cudaFree(m->d_tab);
    cudaFree(m->d_tab2);
    cudaFree(m->d_s);
    cudaFree(m->d_r);
    cudaFree(m->d_w);
    cudaFree(m->d_part);
    cudaFree(m->d_hsino);
    delete m;
}

static BhcArgs bhc_args(ctprj_bhc *m, const double *d_Ie, const float *d_imea, int keep)
{
    BhcArgs a;
    a.tab = m->d_tab;
    a.Ie = d_Ie;
    a.J = m->J;
    a.Ts = m->Ts;
    a.imea = d_imea;
    a.s_out = keep ? m->d_s : nullptr;
    a.r_out = keep ? m->d_r : nullptr;
    a.w_out = keep ? m->d_w : nullptr;
    a.part = m->d_part;
    a.noise = m->noise;
    a.proj_out = nullptr;
    return a;
}

extern "C" int ctprj_bhc_forward(ctprj_bhc *m, const float *d_x, const double *d_Ie,
                                 const float *d_imea, double *d_f, int save, void *stream)
{
    if (!m || !d_x || !d_Ie || !d_imea || !d_f) return set_error(CTPRJ_EINVAL, "NULL argument");
    PlanDevice pd(m->plan->device);
    cudaStream_t s = (cudaStream_t)stream;
    int st;
    if ((st = ensure_parts(m, forward_blocks(m->plan)))) return st;
    if ((st = launch_quad(d_x, m->plan->d_quad, m->plan->g.n, s))) return st;
    int nparts = 0;
    if ((st = launch_forward_bhc(m->plan, m->plan->d_quad, bhc_args(m, d_Ie, d_imea, save),
                                 &nparts, s)))
        return st;
    k_sum_columns<<<1, 256, 0, s>>>(m->d_part, nparts, 1, d_f);
    m->saved = save ? 1 : 0;
    return cuda_error(cudaGetLastError(), "likelihood reduction");
}

int ctprj::bhc_forward_keep_projection(ctprj_bhc *m, const float *d_x, const double *d_Ie, const float *d_imea,
                                       double *d_f, float *proj, cudaStream_t s)
{
    int st;
    if ((st = ensure_parts(m, forward_blocks(m->plan)))) return st;
    if ((st = launch_quad(d_x, m->plan->d_quad, m->plan->g.n, s))) return st;
    BhcArgs a = bhc_args(m, d_Ie, d_imea, 1);
    a.proj_out = proj;
    int nparts = 0;
    if ((st = launch_forward_bhc(m->plan, m->plan->d_quad, a, &nparts, s))) return st;
    k_sum_columns<<<1, 256, 0, s>>>(m->d_part, nparts, 1, d_f);
    m->saved = 1;
    return cuda_error(cudaGetLastError(), "likelihood reduction");
}

extern "C" int ctprj_bhc_terms(ctprj_bhc *m, const float *d_sino, const double *d_Ie,
                               const float *d_imea, double *d_f, int save, void *stream)
{
    if (!m || !d_sino || !d_Ie || !d_imea || !d_f) return set_error(CTPRJ_EINVAL, "NULL argument");
    PlanDevice pd(m->plan->device);
    cudaStream_t s = (cudaStream_t)stream;
    const long long nr = (long long)m->plan->g.np * m->plan->g.W;
    const int blocks = 4 * spectrum_blocks();
    int st;
    if ((st = ensure_parts(m, blocks))) return st;
    k_bhc_terms<<<blocks, kTermThreads, 0, s>>>(d_sino, nr, bhc_args(m, d_Ie, d_imea, save));
    k_sum_columns<<<1, 256, 0, s>>>(m->d_part, blocks, 1, d_f);
    m->saved = save ? 1 : 0;
    return cuda_error(cudaGetLastError(), "polychromatic terms");
}

extern "C" int ctprj_bhc_backward(ctprj_bhc *m, const float *d_x, const double *d_Ie,
                                  const float *d_imea, float *d_gx, double *d_gIe, void *stream)
{
    if (!m) return set_error(CTPRJ_EINVAL, "NULL model");
    PlanDevice pd(m->plan->device);
    cudaStream_t s = (cudaStream_t)stream;
    int st;
    if (!m->saved) {
        // nothing kept by the forward pass: recompute the fused forward
        if (!d_x || !d_Ie || !d_imea)
            return set_error(CTPRJ_EINVAL, "no saved forward state and no inputs to recompute it");
        if ((st = ensure_parts(m, forward_blocks(m->plan)))) return st;
        if ((st = launch_quad(d_x, m->plan->d_quad, m->plan->g.n, s))) return st;
        if ((st = launch_forward_bhc(m->plan, m->plan->d_quad, bhc_args(m, d_Ie, d_imea, 1),
                                     nullptr, s)))
            return st;
    }
    if (d_gIe) {
        const int blocks = spectrum_grad_blocks();
        if ((st = ensure_parts(m, blocks * m->J))) return st;
        const long long nr = (long long)m->plan->g.np * m->plan->g.W;
        k_bhc_spectrum<<<blocks, kSpecThreads, 0, s>>>(m->d_s, m->d_r, nr, m->d_tab, m->J, m->d_part);
        k_sum_columns<<<1, 256, 0, s>>>(m->d_part, blocks, m->J, d_gIe);
        if ((st = cuda_error(cudaGetLastError(), "spectrum gradient"))) return st;
    }
    if (d_gx) {
        if ((st = launch_backward(m->plan, m->d_w, d_gx, 0, nullptr, s, (float)m->Ts))) return st;
    }
    m->saved = 1;
    return CTPRJ_OK;
}

extern "C" int ctprj_bhc_basis(ctprj_bhc *m, const float *d_sino, double *d_A, void *stream)
{
    if (!m || !d_sino || !d_A) return set_error(CTPRJ_EINVAL, "NULL argument");
    PlanDevice pd(m->plan->device);
    const long long nr = (long long)m->plan->g.np * m->plan->g.W;
    k_bhc_basis<<<4 * spectrum_blocks(), 256, 0, (cudaStream_t)stream>>>(d_sino, nr, m->d_tab, m->J,
                                                                         m->Ts, d_A);
    return cuda_error(cudaGetLastError(), "basis matrix");
}

extern "C" int ctprj_bhc_set_noise(ctprj_bhc *m, int noise)
{
    if (!m) return set_error(CTPRJ_EINVAL, "NULL model");
    if (noise != CTPRJ_NOISE_POISSON && noise != CTPRJ_NOISE_GAUSSIAN)
        return set_error(CTPRJ_EINVAL, "unknown noise model %d", noise);
    m->noise = noise;
    m->saved = 0;   // the saved weights belong to the other model
    return CTPRJ_OK;
}

extern "C" int ctprj_bhc_hessian(ctprj_bhc *m, const double *d_Ie, const float *d_imea, const float *d_v,
                                 float *d_Hv, double *d_vHv, void *stream)
{
    if (!m || !d_Ie || !d_imea || !d_v) return set_error(CTPRJ_EINVAL, "NULL argument");
    if (!d_Hv && !d_vHv) return set_error(CTPRJ_EINVAL, "nothing requested");
    if (!m->saved) return set_error(CTPRJ_EINVAL, "the Hessian needs a saved forward state");
    PlanDevice pd(m->plan->device);
    cudaStream_t s = (cudaStream_t)stream;
    const long long nr = (long long)m->plan->g.np * m->plan->g.W;
    int st;
    if (!m->d_hsino &&
        (st = cuda_error(cudaMalloc((void **)&m->d_hsino, sizeof(float) * nr), "Hessian scratch")))
        return st;
    const int blocks = 4 * spectrum_blocks();
    if ((st = ensure_parts(m, blocks))) return st;
    if ((st = ctprj_forward(m->plan, d_v, m->d_hsino, s))) return st;
    k_bhc_hess<<<blocks, kTermThreads, 0, s>>>(m->d_s, m->d_hsino, nr, bhc_args(m, d_Ie, d_imea, 0),
                                                m->d_tab2);
    if (d_vHv) k_sum_columns<<<1, 256, 0, s>>>(m->d_part, blocks, 1, d_vHv);
    if ((st = cuda_error(cudaGetLastError(), "Hessian weights"))) return st;
    if (d_Hv) return launch_backward(m->plan, m->d_hsino, d_Hv, 0, nullptr, s, (float)m->Ts);
    return CTPRJ_OK;
}

extern "C" int ctprj_bhc_state(ctprj_bhc *m, const float **d_s, const double **d_r, const float **d_w)
{
    if (!m) return set_error(CTPRJ_EINVAL, "NULL model");
    if (d_s) *d_s = m->d_s;
    if (d_r) *d_r = m->d_r;
    if (d_w) *d_w = m->d_w;
    return m->saved ? CTPRJ_OK : set_error(CTPRJ_EINVAL, "no forward state saved");
}

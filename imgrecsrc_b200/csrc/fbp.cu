// fbp.cu -- filtered backprojection (cmd & FBP_BIT of gpuPrj).
//
// The reference (prj/cpuPrj.c:718-784, prj/utils.h:94-151) pre-weights each
// fan-beam detector by d / sqrt(d^2 + t^2), filters every view with a
// Hann-windowed ramp by FFTs of length 2 prjWidth (zero padded), and
// backprojects with the FBP distance weights.  Its filter is a fixed linear map:
// a circular convolution whose kernel h = IDFT(Re DFT(ramp) * hann) / 2W is real
// and even.  For outputs and inputs inside one view row (|m - n| < prjWidth) the
// wrap-around never reaches the padding, so the filter is the symmetric
// Toeplitz product out[m] = sum_n x[n] h[|m - n|].  The plan derives h once, in
// FP64 on the host, from the reference's own taps (its ramp values are formed in
// float arithmetic, prj/utils.h:117-121).  Rows of up to 4096 detectors are
// filtered by FFTs of the next power of two >= 2 prjWidth - 1, two views per
// complex transform (k_fbp_fft: 0.050 ms at 1440 views x 2048 detectors, where
// the Toeplitz product takes 0.348); longer rows by the register-tiled Toeplitz
// product (k_fbp_filter).
#include <cmath>
#include <vector>

#include "ctprj_internal.h"

namespace ctprj {


// taps h[0..W-1] of the reference's ramp filter for a row of W detectors
static std::vector<double> ramp_taps(int W)
{
    const int N = 2 * W;
    std::vector<double> ramp(N, 0.0), ct(N), reH(N), h(W);
    for (int i = 1; i < N; ++i) {
        if (i % 2 == 0) continue;
        const int m = i < N / 2 ? i : N - i;
        volatile float r = -1.0f / kRefPiF;
        r = r / kRefPiF;
        r = r / (float)m;
        r = r / (float)m;
        ramp[i] = r;
    }
    ramp[0] = 0.25;
    for (int i = 0; i < N; ++i) ct[i] = cos(2.0 * M_PI * (double)i / (double)N);
    for (int i = 0; i < N; ++i) {
        double acc = 0.0;
        for (int m = 0; m < N; ++m)
            if (ramp[m] != 0.0) acc += ramp[m] * ct[(long long)i * m % N];
        // Hann window, argument formed in float as 2*PI*i/N (prj/utils.h:108)
        volatile float arg = 2.0f * kRefPiF;
        arg = arg * (float)i;
        arg = arg / (float)N;
        reH[i] = acc * (0.5 + 0.5 * cos((double)arg));
    }
    for (int k = 0; k < W; ++k) {
        double acc = 0.0;
        for (int i = 0; i < N; ++i) acc += reH[i] * ct[(long long)i * k % N];
        h[k] = acc / N;
    }
    return h;
}

// The filter as a register-tiled Toeplitz product.  A block of kFT threads
// owns kFO = kFT * kFR consecutive outputs of kFV view rows; thread t the kFR
// consecutive outputs mt = m0 + kFR t .. mt + kFR - 1 of every row, in
// kFV * kFR accumulators.  Inputs go through shared memory in chunks of kFN,
// with the taps of the chunk's lag window; for input n the thread needs the
// kFR taps h[|mt + r - n|], r < kFR, which slide by one element per input, so
// it keeps them in registers and loads one new tap per input: kFV + 1 shared
// loads (kFV of them broadcasts) per kFV * kFR FMAs.  The lag window is stored
// with one pad per 32 taps, so that lanes kFR apart read distinct banks.
constexpr int kFT = 128, kFR = 8, kFV = 4, kFN = 256;
constexpr int kFO = kFT * kFR;
constexpr int kFH = kFO + kFN;   // lag window length (one spare)

__device__ __forceinline__ int skew(int i) { return i + (i >> 5); }

__global__ void __launch_bounds__(kFT)
k_fbp_filter(const float *__restrict__ sino, float *__restrict__ out, const float *__restrict__ taps,
             const float *__restrict__ colw, int W, int np)
{
    __shared__ float xs[kFV][kFN];
    __shared__ float hs[kFH + kFH / 32 + 1];
    const int m0 = blockIdx.x * kFO, v0 = blockIdx.y * kFV;
    const int lane0 = threadIdx.x * kFR;   // mt - m0
    float acc[kFV][kFR];
#pragma unroll
    for (int v = 0; v < kFV; ++v)
#pragma unroll
        for (int r = 0; r < kFR; ++r) acc[v][r] = 0.0f;
    for (int n0 = 0; n0 < W; n0 += kFN) {
        __syncthreads();
        for (int e = threadIdx.x; e < kFV * kFN; e += kFT) {
            const int v = e / kFN, i = e % kFN, n = n0 + i;
            xs[v][i] = (v0 + v < np && n < W) ? sino[(size_t)(v0 + v) * W + n] * (colw ? colw[n] : 1.0f) : 0.0f;
        }
        // hs[j] = h[|lag_lo + j|], lag_lo = m0 - (n0 + kFN - 1): the lag of
        // output mt + r and input n0 + i is at j = lane0 + r + kFN - 1 - i
        const int lag_lo = m0 - (n0 + kFN - 1);
        for (int j = threadIdx.x; j < kFH; j += kFT) {
            const int lag = abs(lag_lo + j);
            hs[skew(j)] = lag < W ? taps[lag] : 0.0f;
        }
        __syncthreads();
        float w[kFR];
#pragma unroll
        for (int r = 0; r < kFR; ++r) w[r] = hs[skew(lane0 + r + kFN - 1)];
        for (int i0 = 0; i0 < kFN; i0 += kFR) {
#pragma unroll
            for (int q = 0; q < kFR; ++q) {
                const int i = i0 + q;
                float xv[kFV];
#pragma unroll
                for (int v = 0; v < kFV; ++v) xv[v] = xs[v][i];
#pragma unroll
                for (int v = 0; v < kFV; ++v)
#pragma unroll
                    for (int r = 0; r < kFR; ++r) acc[v][r] = fmaf(xv[v], w[r], acc[v][r]);
                // the taps of input i + 1 are those of input i shifted by one
#pragma unroll
                for (int r = kFR - 1; r > 0; --r) w[r] = w[r - 1];
                const int jn = lane0 + kFN - 2 - i;
                w[0] = jn >= 0 ? hs[skew(jn)] : 0.0f;
            }
        }
    }
#pragma unroll
    for (int v = 0; v < kFV; ++v) {
        if (v0 + v >= np) break;
#pragma unroll
        for (int r = 0; r < kFR; ++r) {
            const int m = m0 + lane0 + r;
            if (m < W) out[(size_t)(v0 + v) * W + m] = acc[v][r];
        }
    }
}

// The same filter by FFTs.  Zero-padded to a power of two N >= 2W - 1, the
// circular convolution of a row with the even kernel h'[k] = h'[N - k] = h[k]
// (k < W, zero between) equals the Toeplitz product for every output m < W,
// since |m - n| < W never wraps onto a nonzero tap.  The kernel is real, so two
// view rows go through one complex transform as its real and imaginary parts
// and come back filtered in the same parts.  A block takes two views: the rows
// (pre-weighted) are transformed in place by radix-2 decimation in frequency,
// which leaves the spectrum in bit-reversed order, multiplied by the real
// response H = DFT(h') / N stored in that order, and transformed back by
// decimation in time, which takes bit-reversed input and returns the natural
// order: no permutation pass.  Twiddles from FP64, one table per stage.
#ifndef CTPRJ_FBP_FFT_THREADS
#define CTPRJ_FBP_FFT_THREADS 256
#endif
constexpr int kFftThreads = CTPRJ_FBP_FFT_THREADS;
// CTPRJ_FBP_TOEPLITZ = 1 keeps every plan on the Toeplitz kernel
#ifndef CTPRJ_FBP_TOEPLITZ
#define CTPRJ_FBP_TOEPLITZ 0
#endif
constexpr bool kFbpToeplitz = CTPRJ_FBP_TOEPLITZ != 0;
constexpr int kFftMaxLog = 13;   // N <= 8192: rows of up to 4096 detectors

__device__ __forceinline__ float2 cmulf(float2 a, float2 b)
{
    return make_float2(fmaf(a.x, b.x, -a.y * b.y), fmaf(a.x, b.y, a.y * b.x));
}

// Shared-memory slot of element i: its low four bits XOR (r | r << 2), r = bits
// 4-5 of i.  Every access pattern below (linear passes, and the radix-2 and
// paired stages at every span) then puts the 16 lanes of a half-warp on 16
// distinct 8-byte slots: no bank conflicts (4-way at the three smallest spans
// without it).
__device__ __forceinline__ int swz(int i)
{
    const int r = (i >> 4) & 3;
    return i ^ (r | (r << 2));
}

// Twiddles of stage s (half-span h = 2^s) at tw[h - 1 + pos] = exp(-2 pi i pos / 2h),
// pos < h: consecutive lanes read consecutive entries at every stage.
template <bool CONJ>
__device__ __forceinline__ float2 twiddle(const float2 *tw, int h, int pos)
{
    const float2 w = __ldg(tw + h - 1 + pos);
    return CONJ ? make_float2(w.x, -w.y) : w;
}

// one radix-2 butterfly j < N/2 of stage s, forward (decimation in time) or
// decimation in frequency
template <bool CONJ>
__device__ __forceinline__ void dit2(float2 *z, const float2 *tw, int j, int s)
{
    const int h = 1 << s, pos = j & (h - 1), i0 = swz(((j >> s) << (s + 1)) + pos), i1 = swz(((j >> s) << (s + 1)) + pos + h);
    const float2 a = z[i0], t = cmulf(twiddle<CONJ>(tw, h, pos), z[i1]);
    z[i0] = make_float2(a.x + t.x, a.y + t.y);
    z[i1] = make_float2(a.x - t.x, a.y - t.y);
}
template <bool CONJ>
__device__ __forceinline__ void dif2(float2 *z, const float2 *tw, int j, int s)
{
    const int h = 1 << s, pos = j & (h - 1), i0 = swz(((j >> s) << (s + 1)) + pos), i1 = swz(((j >> s) << (s + 1)) + pos + h);
    const float2 a = z[i0], b = z[i1], w = twiddle<CONJ>(tw, h, pos);
    z[i0] = make_float2(a.x + b.x, a.y + b.y);
    z[i1] = cmulf(make_float2(a.x - b.x, a.y - b.y), w);
}
// stages s and s + 1 on the four elements base + pos + {0, h, 2h, 3h}, j < N/4
// (base = (j / h) 4h, pos = j mod h): DIT stage s on (0, 1), (2, 3), then stage
// s + 1 on (0, 2), (1, 3); DIF the same pairs in the opposite order
template <bool CONJ>
__device__ __forceinline__ void dit4(float2 *z, const float2 *tw, int j, int s)
{
    const int h = 1 << s, pos = j & (h - 1), b = ((j >> s) << (s + 2)) + pos;
    const int k0 = swz(b), k1 = swz(b + h), k2 = swz(b + 2 * h), k3 = swz(b + 3 * h);
    float2 e0 = z[k0], e1 = z[k1], e2 = z[k2], e3 = z[k3];
    const float2 w1 = twiddle<CONJ>(tw, h, pos);
    float2 t = cmulf(w1, e1);
    e1 = make_float2(e0.x - t.x, e0.y - t.y);
    e0 = make_float2(e0.x + t.x, e0.y + t.y);
    t = cmulf(w1, e3);
    e3 = make_float2(e2.x - t.x, e2.y - t.y);
    e2 = make_float2(e2.x + t.x, e2.y + t.y);
    const float2 wa = twiddle<CONJ>(tw, 2 * h, pos), wb = twiddle<CONJ>(tw, 2 * h, pos + h);
    t = cmulf(wa, e2);
    z[k2] = make_float2(e0.x - t.x, e0.y - t.y);
    z[k0] = make_float2(e0.x + t.x, e0.y + t.y);
    t = cmulf(wb, e3);
    z[k3] = make_float2(e1.x - t.x, e1.y - t.y);
    z[k1] = make_float2(e1.x + t.x, e1.y + t.y);
}
template <bool CONJ>
__device__ __forceinline__ void dif4(float2 *z, const float2 *tw, int j, int s)
{
    const int h = 1 << s, pos = j & (h - 1), b = ((j >> s) << (s + 2)) + pos;
    const int k0 = swz(b), k1 = swz(b + h), k2 = swz(b + 2 * h), k3 = swz(b + 3 * h);
    const float2 e0 = z[k0], e1 = z[k1], e2 = z[k2], e3 = z[k3];
    const float2 wa = twiddle<CONJ>(tw, 2 * h, pos), wb = twiddle<CONJ>(tw, 2 * h, pos + h);
    const float2 f0 = make_float2(e0.x + e2.x, e0.y + e2.y);
    const float2 f2 = cmulf(make_float2(e0.x - e2.x, e0.y - e2.y), wa);
    const float2 f1 = make_float2(e1.x + e3.x, e1.y + e3.y);
    const float2 f3 = cmulf(make_float2(e1.x - e3.x, e1.y - e3.y), wb);
    const float2 w1 = twiddle<CONJ>(tw, h, pos);
    z[k0] = make_float2(f0.x + f1.x, f0.y + f1.y);
    z[k1] = cmulf(make_float2(f0.x - f1.x, f0.y - f1.y), w1);
    z[k2] = make_float2(f2.x + f3.x, f2.y + f3.y);
    z[k3] = cmulf(make_float2(f2.x - f3.x, f2.y - f3.y), w1);
}

__global__ void __launch_bounds__(kFftThreads)
k_fbp_fft(const float *__restrict__ sino, float *__restrict__ out, const float *__restrict__ colw,
          const float2 *__restrict__ tw, const float *__restrict__ H, int W, int np, int logN)
{
    extern __shared__ float2 z[];
    const int N = 1 << logN, va = 2 * blockIdx.x, vb = va + 1;
    const bool hasb = vb < np;
    for (int n = threadIdx.x; n < N; n += blockDim.x) {
        float2 v = make_float2(0.0f, 0.0f);
        if (n < W) {
            const float c = colw ? colw[n] : 1.0f;
            v.x = sino[(size_t)va * W + n] * c;
            if (hasb) v.y = sino[(size_t)vb * W + n] * c;
        }
        z[swz(n)] = v;
    }
    __syncthreads();
    // forward: decimation in frequency, stages s = logN - 1 .. 0 (half-span 2^s),
    // natural order in, bit-reversed out; two stages at a time where they pair
    // up (a thread's four elements base + pos + {0, h, 2h, 3h} are closed under
    // stages s + 1 and s, so the arithmetic is the radix-2 one with half the
    // barriers)
    for (int st = logN - 2; st >= (logN & 1); st -= 2) {
        for (int j = threadIdx.x; j < N / 4; j += blockDim.x) dif4<false>(z, tw, j, st);
        __syncthreads();
    }
    if (logN & 1) {
        for (int j = threadIdx.x; j < N / 2; j += blockDim.x) dif2<false>(z, tw, j, 0);
        __syncthreads();
    }
    // the response, stored in the same bit-reversed order
    for (int k = threadIdx.x; k < N; k += blockDim.x) {
        const float hk = __ldg(H + k);
        const int q = swz(k);
        z[q] = make_float2(z[q].x * hk, z[q].y * hk);
    }
    __syncthreads();
    // inverse: decimation in time with conjugate twiddles, stages 0 .. logN - 1,
    // bit-reversed order in, natural order out
    int s0 = 0;
    if (logN & 1) {
        for (int j = threadIdx.x; j < N / 2; j += blockDim.x) dit2<true>(z, tw, j, 0);
        __syncthreads();
        s0 = 1;
    }
    for (int st = s0; st < logN; st += 2) {
        for (int j = threadIdx.x; j < N / 4; j += blockDim.x) dit4<true>(z, tw, j, st);
        __syncthreads();
    }
    for (int m = threadIdx.x; m < W; m += blockDim.x) {
        const float2 v = z[swz(m)];
        out[(size_t)va * W + m] = v.x;
        if (hasb) out[(size_t)vb * W + m] = v.y;
    }
}

// log2 of the transform length for rows of W detectors, or 0 when the rows are
// too long for one block's shared memory (the Toeplitz kernel then runs)
static int fft_log(int W)
{
    int l = 1;
    while ((1 << l) < 2 * W - 1) ++l;
    return l <= kFftMaxLog ? l : 0;
}

// H = DFT_N(h') / N, real and even: h[0] + 2 sum_{0<j<W} h[j] cos(2 pi j k / N)
static std::vector<double> fft_response(const std::vector<double> &h, int logN)
{
    const int N = 1 << logN, W = (int)h.size();
    std::vector<double> ct(N), H(N);
    for (int i = 0; i < N; ++i) ct[i] = cos(2.0 * M_PI * (double)i / (double)N);
    for (int k = 0; k < N; ++k) {
        double acc = h[0];
        for (int j = 1; j < W; ++j) acc += 2.0 * h[j] * ct[(long long)j * k % N];
        H[k] = acc / N;
    }
    return H;
}

}  // namespace ctprj

using namespace ctprj;

int ctprj_fbp_device(ctprj_plan *plan, const float *d_sino, float *d_img, cudaStream_t s)
{
    const Geo &g = plan->g;
    int st;
    if (!plan->d_ramp) {
        std::vector<double> h = ramp_taps(g.W);
        const int lg = kFbpToeplitz ? 0 : fft_log(g.W);
        const size_t nfft = lg ? (size_t)1 << lg : 0;
        // taps, pre-weights, then (FFT path) N/2 twiddles as float pairs and the
        // N-point response
        std::vector<float> buf(2 * (size_t)g.W + 3 * nfft);
        for (int k = 0; k < g.W; ++k) buf[k] = (float)h[k];
        // fan-beam cosine pre-weight d / sqrt(d^2 + t^2) (prj/cpuPrj.c:737-751)
        for (int k = 0; k < g.W; ++k) {
            const double t = (double)(k - g.pC) * g.dSize;
            buf[g.W + k] = g.fan ? (float)(g.d / sqrt(g.d * g.d + t * t)) : 1.0f;
        }
        if (lg) {
            // per stage s (half-span h = 2^s) the h twiddles exp(-2 pi i pos / 2h)
            // at float pairs h - 1 + pos: N - 1 pairs in all
            float *tw = buf.data() + 2 * (size_t)g.W, *Hf = tw + 2 * nfft;
            for (size_t h = 1; h < nfft; h <<= 1)
                for (size_t pos = 0; pos < h; ++pos) {
                    const double a = -M_PI * (double)pos / (double)h;
                    tw[2 * (h - 1 + pos)] = (float)cos(a);
                    tw[2 * (h - 1 + pos) + 1] = (float)sin(a);
                }
            // in the bit-reversed order the forward transform leaves its output in
            const std::vector<double> H = fft_response(h, lg);
            for (size_t k = 0; k < nfft; ++k) {
                size_t r = 0;
                for (int bit = 0; bit < lg; ++bit) r |= ((k >> bit) & 1) << (lg - 1 - bit);
                Hf[r] = (float)H[k];
            }
        }
        plan->fbp_log = lg;
        if ((st = cuda_error(cudaMalloc((void **)&plan->d_ramp, sizeof(float) * buf.size()),
                             "FBP taps")) ||
            (st = cuda_error(cudaMalloc((void **)&plan->d_fsino, sizeof(float) * (size_t)g.W * g.np),
                             "FBP scratch")) ||
            (st = cuda_error(cudaMemcpy(plan->d_ramp, buf.data(), sizeof(float) * buf.size(),
                                        cudaMemcpyHostToDevice),
                             "FBP taps upload"))) {
            cudaFree(plan->d_ramp);
            cudaFree(plan->d_fsino);
            plan->d_ramp = plan->d_fsino = nullptr;
            return st;
        }
    }
    const float *colw = g.fan ? plan->d_ramp + g.W : nullptr;
    if (plan->fbp_log) {
        const int lg = plan->fbp_log;
        const size_t nfft = (size_t)1 << lg, smem = sizeof(float2) * nfft;
        const float *tw = plan->d_ramp + 2 * (size_t)g.W;
        if (smem > 48 * 1024 &&
            (st = cuda_error(cudaFuncSetAttribute(k_fbp_fft, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                  (int)smem),
                             "FBP transform shared memory")))
            return st;
        k_fbp_fft<<<(g.np + 1) / 2, kFftThreads, smem, s>>>(d_sino, plan->d_fsino, colw,
                                                             reinterpret_cast<const float2 *>(tw),
                                                             tw + 2 * nfft, g.W, g.np, lg);
    } else {
        dim3 grid((g.W + kFO - 1) / kFO, (g.np + kFV - 1) / kFV);
        k_fbp_filter<<<grid, kFT, 0, s>>>(d_sino, plan->d_fsino, plan->d_ramp, colw, g.W, g.np);
    }
    if ((st = cuda_error(cudaGetLastError(), "FBP filter launch"))) return st;
    return launch_backward(plan, plan->d_fsino, d_img, 1, nullptr, s);
}

extern "C" int ctprj_fbp(ctprj_plan *plan, const float *d_sino, float *d_img, void *stream)
{
    if (!plan || !d_sino || !d_img) return set_error(CTPRJ_EINVAL, "NULL plan or buffer");
    int prev = -1;
    cudaGetDevice(&prev);
    if (prev != plan->device) cudaSetDevice(plan->device);
    int st = ctprj_fbp_device(plan, d_sino, d_img, (cudaStream_t)stream);
    if (prev >= 0 && prev != plan->device) cudaSetDevice(prev);
    return st;
}

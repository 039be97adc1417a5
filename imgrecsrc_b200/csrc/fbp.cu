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
// float arithmetic, prj/utils.h:117-121); the device applies it directly as a
// register-tiled product (k_fbp_filter).
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

}  // namespace ctprj

using namespace ctprj;

int ctprj_fbp_device(ctprj_plan *plan, const float *d_sino, float *d_img, cudaStream_t s)
{
    const Geo &g = plan->g;
    int st;
    if (!plan->d_ramp) {
        std::vector<double> h = ramp_taps(g.W);
        std::vector<float> buf(2 * (size_t)g.W);
        for (int k = 0; k < g.W; ++k) buf[k] = (float)h[k];
        // fan-beam cosine pre-weight d / sqrt(d^2 + t^2) (prj/cpuPrj.c:737-751)
        for (int k = 0; k < g.W; ++k) {
            const double t = (double)(k - g.pC) * g.dSize;
            buf[g.W + k] = g.fan ? (float)(g.d / sqrt(g.d * g.d + t * t)) : 1.0f;
        }
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
    dim3 grid((g.W + kFO - 1) / kFO, (g.np + kFV - 1) / kFV);
    k_fbp_filter<<<grid, kFT, 0, s>>>(d_sino, plan->d_fsino, plan->d_ramp,
                                       g.fan ? plan->d_ramp + g.W : nullptr, g.W, g.np);
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

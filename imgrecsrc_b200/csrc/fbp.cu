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
// float arithmetic, prj/utils.h:117-121); the device applies it directly, one
// block per view row with the row and the taps staged in shared memory.
#include <cmath>
#include <vector>

#include "ctprj_internal.h"

namespace ctprj {

constexpr int kFiltThreads = 256;
constexpr int kFiltChunk = 4096;   // row / tap elements staged per pass

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

__global__ void __launch_bounds__(kFiltThreads)
k_fbp_filter(const float *__restrict__ sino, float *__restrict__ out, const float *__restrict__ taps,
             const float *__restrict__ colw, int W, int np)
{
    __shared__ float xs[kFiltChunk];
    __shared__ float hs[2 * kFiltChunk];
    const int v = blockIdx.y;
    if (v >= np) return;
    const float *row = sino + (size_t)v * W;
    const int m0 = blockIdx.x * kFiltThreads;
    const int m = m0 + threadIdx.x;
    float acc = 0.0f;
    // outputs m0..m0+255 need taps |m - n| for n in the staged input chunk
    for (int n0 = 0; n0 < W; n0 += kFiltChunk) {
        const int nlen = min(kFiltChunk, W - n0);
        __syncthreads();
        for (int i = threadIdx.x; i < nlen; i += kFiltThreads)
            xs[i] = row[n0 + i] * (colw ? colw[n0 + i] : 1.0f);
        // tap window: lags from (m0 - (n0 + nlen - 1)) to (m0 + 255 - n0)
        const int lag_lo = m0 - (n0 + nlen - 1);
        const int nl = nlen + kFiltThreads - 1;
        for (int i = threadIdx.x; i < nl; i += kFiltThreads) {
            const int lag = abs(lag_lo + i);
            hs[i] = lag < W ? taps[lag] : 0.0f;
        }
        __syncthreads();
        if (m < W) {
            // lag for input n0 + i is m - n0 - i = (m - m0) + (nlen - 1 - i) + lag_lo
            const int base = (m - m0) + nlen - 1;
            for (int i = 0; i < nlen; ++i) acc = fmaf(xs[i], hs[base - i], acc);
        }
    }
    if (m < W) out[(size_t)v * W + m] = acc;
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
    dim3 grid((g.W + kFiltThreads - 1) / kFiltThreads, g.np);
    k_fbp_filter<<<grid, kFiltThreads, 0, s>>>(d_sino, plan->d_fsino, plan->d_ramp,
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

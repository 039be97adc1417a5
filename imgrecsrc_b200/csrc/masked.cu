// masked.cu -- the projector in MATLAB's data layout with the reconstruction
// mask applied on the device (include/ctprj_masked.h).
//
// MATLAB stores the n x n image column-major: element (row r, column c) at
// r + c n.  The gateway (prj/mPrj.c:82-84) copies it into the projector's
// row-major image with the same rows and columns, img[r n + c], and copies the
// backprojection back the same way (:134-136); the sinogram passes in the
// projector's own order.  ConfigCT's mask (utils/maskFunc.m) holds column-major
// linear indices m, i.e. the pixel (m mod n, m div n).  Each entry point is a
// scatter or cast kernel, the plan's projection, and a gather or cast kernel
// that applies the scale in double precision.
#include "ctprj_internal.h"
#include "../../include/ctprj_masked.h"

namespace ctprj {

// img (row-major, n x n, zeroed by the caller) at the masked pixels = (float)s
__global__ void __launch_bounds__(256)
k_mask_scatter(const double *__restrict__ s, const int *__restrict__ mask, long long npix, int n,
               float *__restrict__ img)
{
    const long long nn = (long long)n * n;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < npix;
         i += (long long)gridDim.x * blockDim.x) {
        const long long m = mask ? (long long)mask[i] : i;
        if (m < 0 || m >= nn) continue;
        img[(m % n) * n + m / n] = (float)s[i];
    }
}

// s[i] = scale * img at the i-th masked pixel
__global__ void __launch_bounds__(256)
k_mask_gather(const float *__restrict__ img, const int *__restrict__ mask, long long npix, int n,
              double scale, double *__restrict__ s)
{
    const long long nn = (long long)n * n;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < npix;
         i += (long long)gridDim.x * blockDim.x) {
        const long long m = mask ? (long long)mask[i] : i;
        if (m < 0 || m >= nn) continue;
        s[i] = scale * (double)img[(m % n) * n + m / n];
    }
}

__global__ void __launch_bounds__(256)
k_to_double(const float *__restrict__ src, long long n, double scale, double *__restrict__ dst)
{
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x)
        dst[i] = scale * (double)src[i];
}

__global__ void __launch_bounds__(256)
k_to_float(const double *__restrict__ src, long long n, float *__restrict__ dst)
{
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x)
        dst[i] = (float)src[i];
}

}  // namespace ctprj

using namespace ctprj;

namespace {

int grid_for(long long n)
{
    const long long b = (n + 255) / 256;
    return (int)(b < 4096 ? (b > 0 ? b : 1) : 4096);
}

// the plan's layout scratch: one single-precision image and one sinogram
int ensure_scratch(ctprj_plan *p)
{
    int st = CTPRJ_OK;
    if (!p->d_mimg)
        st = cuda_error(cudaMalloc((void **)&p->d_mimg, sizeof(float) * (size_t)p->g.n * p->g.n),
                        "layout scratch");
    if (!st && !p->d_msino)
        st = cuda_error(cudaMalloc((void **)&p->d_msino, sizeof(float) * (size_t)p->g.np * p->g.W),
                        "layout scratch");
    return st;
}

int check_args(ctprj_plan *plan, const int *d_mask, long long npix, const void *a, const void *b)
{
    if (!plan || !a || !b) return set_error(CTPRJ_EINVAL, "NULL plan or buffer");
    const long long nn = (long long)plan->g.n * plan->g.n;
    if (d_mask ? (npix < 0 || npix > nn) : npix != nn)
        return set_error(CTPRJ_EINVAL, "npix %lld: at most n*n with a mask, n*n = %lld without", npix, nn);
    return CTPRJ_OK;
}

}  // namespace

extern "C" int ctprj_masked_forward(ctprj_plan *plan, const int *d_mask, long long npix, const double *d_s,
                                    double scale, double *d_y, void *stream)
{
    int st = check_args(plan, d_mask, npix, d_s, d_y);
    if (st) return st;
    PlanDevice pd(plan->device);
    cudaStream_t s = (cudaStream_t)stream;
    const long long nn = (long long)plan->g.n * plan->g.n, ns = (long long)plan->g.np * plan->g.W;
    if ((st = ensure_scratch(plan)) ||
        (st = cuda_error(cudaMemsetAsync(plan->d_mimg, 0, sizeof(float) * nn, s), "image clear")))
        return st;
    k_mask_scatter<<<grid_for(npix), 256, 0, s>>>(d_s, d_mask, npix, plan->g.n, plan->d_mimg);
    if ((st = cuda_error(cudaGetLastError(), "mask scatter")) ||
        (st = ctprj_forward(plan, plan->d_mimg, plan->d_msino, s)))
        return st;
    k_to_double<<<grid_for(ns), 256, 0, s>>>(plan->d_msino, ns, scale, d_y);
    return cuda_error(cudaGetLastError(), "sinogram cast");
}

static int masked_back(ctprj_plan *plan, const int *d_mask, long long npix, const double *d_y, double scale,
                       double *d_s, void *stream, bool fbp)
{
    int st = check_args(plan, d_mask, npix, d_y, d_s);
    if (st) return st;
    PlanDevice pd(plan->device);
    cudaStream_t s = (cudaStream_t)stream;
    const long long ns = (long long)plan->g.np * plan->g.W;
    if ((st = ensure_scratch(plan))) return st;
    k_to_float<<<grid_for(ns), 256, 0, s>>>(d_y, ns, plan->d_msino);
    if ((st = cuda_error(cudaGetLastError(), "sinogram cast")) ||
        (st = fbp ? ctprj_fbp(plan, plan->d_msino, plan->d_mimg, s)
                  : ctprj_backward(plan, plan->d_msino, plan->d_mimg, s)))
        return st;
    k_mask_gather<<<grid_for(npix), 256, 0, s>>>(plan->d_mimg, d_mask, npix, plan->g.n, scale, d_s);
    return cuda_error(cudaGetLastError(), "mask gather");
}

extern "C" int ctprj_masked_backward(ctprj_plan *plan, const int *d_mask, long long npix, const double *d_y,
                                     double scale, double *d_s, void *stream)
{
    return masked_back(plan, d_mask, npix, d_y, scale, d_s, stream, false);
}

extern "C" int ctprj_masked_fbp(ctprj_plan *plan, const int *d_mask, long long npix, const double *d_y,
                                double scale, double *d_s, void *stream)
{
    return masked_back(plan, d_mask, npix, d_y, scale, d_s, stream, true);
}

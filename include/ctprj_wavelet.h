/*
 * ctprj_wavelet.h -- the wavelet regulariser of the density step on the GPU.
 *
 * The reference's default proximal map for its NPG / PG density step
 * (opt.proximal = 'wvltADMM', bhc/beamhardenSpline.m:36, :205-209) solves
 *
 *     alpha = argmin 1/2 ||alpha - a||^2 + I(alpha >= 0) + u ||Psit(alpha)||_1
 *
 * by ADMM (npg/admm.m), where Psi / Psit are the inverse / forward periodic
 * orthogonal wavelet transforms of the vendored Rice Wavelet Toolbox
 * (midwt / mdwt, rwt/midwt_r.c, rwt/mdwt_r.c) with a Daubechies scaling
 * filter h (rwt/daubcqf.m) and L levels (utils/Utils.m:445-469; the BHC
 * examples use the 2-tap filter, L = 6, bhc/doBHC.m:33).
 *
 * Images are rows x cols floats, row-major, element (r, c) at r * cols + c,
 * and the transforms treat element (r, c) as the reference treats the MATLAB
 * matrix element x(r, c): the same filters along both axes, lowpass outputs
 * first, level by level on the top-left block.  Because the two axes are
 * treated alike, a column-major MATLAB array passed as it lies with rows and
 * columns swapped gives the transposed layout of the same coefficients, that
 * is, MATLAB's own coefficient array.  rows and cols must be divisible by
 * 2^levels; h is the scaling filter (lh even, 2 <= lh <= 20) in host memory.
 * Arithmetic is FP32 per coefficient with FP64 norms; calls are enqueued on
 * `stream`.
 */
#ifndef CTPRJ_WAVELET_H
#define CTPRJ_WAVELET_H

#include "ctprj.h"

#ifdef __cplusplus
extern "C" {
#endif

#define CTPRJ_WVLT_MAX_FILTER 20

/* d_y = mdwt(d_x, h, levels) (rwt/mdwt.m; rwt/mdwt_r.c MDWT).  d_y may not
 * alias d_x. */
int ctprj_dwt(const float *d_x, int rows, int cols, const double *h, int lh, int levels, float *d_y,
              void *stream);

/* d_x = midwt(d_y, h, levels) (rwt/midwt.m; rwt/midwt_r.c MIDWT), the
 * inverse (and adjoint) of ctprj_dwt.  d_x may not alias d_y. */
int ctprj_idwt(const float *d_y, int rows, int cols, const double *h, int lh, int levels, float *d_x,
               void *stream);

/* *d_l1 = pNorm(Psit(x), 1), the 'wvltADMM' penalty
 * (bhc/beamhardenSpline.m:208), in FP64, written to device memory. */
int ctprj_wvlt_l1(const float *d_x, int rows, int cols, const double *h, int lh, int levels, double *d_l1,
                  void *stream);

/* [alpha, iter] = admm(Psi, Psit, a, u, rel_tol, max_itr, false, init)
 * (npg/admm.m): the same start (s = Psit(init), nu = 0, rho = 1), steps,
 * stopping rule (change of s and residual both <= min(1e-3, rel_tol) in the
 * units of a / ||a||, or more than max_itr iterations) and rho adaptation.
 * d_init may be NULL (init = a).  d_alpha (rows*cols floats) may not alias
 * d_a or d_init.  *iterations (may be NULL) receives iter.  Synchronises
 * `stream` once at the start and every eight iterations. */
int ctprj_wvlt_admm(const float *d_a, int rows, int cols, const double *h, int lh, int levels, double u,
                    double rel_tol, int max_itr, const float *d_init, float *d_alpha, int *iterations,
                    void *stream);

/* d_maskk = wvltMask(d_mask, levels, daub) (utils/wvltMask.m): 1 at every
 * coefficient of the rows x cols transform that a pixel with d_mask != 0
 * reaches, else 0 (uint8 images, row-major like the transforms). */
int ctprj_wvlt_mask(const unsigned char *d_mask, int rows, int cols, const double *h, int lh, int levels,
                    unsigned char *d_maskk, void *stream);

#ifdef __cplusplus
}
#endif

#endif /* CTPRJ_WAVELET_H */

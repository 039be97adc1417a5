/*
 * ctprj_tv.h -- the total-variation proximal map on the GPU.
 *
 * The reference's 'tviso' and 'tvl1' regularisers (bhc/beamhardenSpline.m:
 * 214-223) make the density step's proximal map a bounded TV denoising,
 *
 *     D = argmin_X ||X - Xobs||_F^2 + 2 lambda TV(X)   subject to  lb <= X <= ub,
 *
 * computed by utils/TV.m:56-80 (TV.denoise) through utils/denoise_bound_mod.m:
 * Beck and Teboulle's fast gradient projection on the dual, with the
 * difference operators of utils/Ltrans.m / utils/Lforward.m and the TV of
 * utils/tlv.m.  These entry points run that iteration on device buffers:
 * the same dual start (zero), step 1/(8 lambda), momentum, restart (t = 1
 * when the dual objective rises) and stopping rule (five consecutive
 * relative changes ||D - D_old|| / ||D|| below `epsilon`, or `max_iter`
 * iterations).  Arithmetic is FP32 per pixel with FP64 sums for the stopping
 * rule and restart test.
 *
 * Images are `rows` x `cols` floats, row-major: element (i, j) at
 * i * cols + j.  The reference's images are column-major MATLAB arrays; since
 * the iteration treats the two axes alike, passing a column-major image with
 * rows and cols swapped gives the same D up to FP32 rounding.  All calls are
 * enqueued on `stream`; ctprj_tv_denoise synchronises it every eight
 * iterations to read the stopping flag.
 */
#ifndef CTPRJ_TV_H
#define CTPRJ_TV_H

#include "ctprj.h"

#ifdef __cplusplus
extern "C" {
#endif

#define CTPRJ_TV_ISO 0   /* isotropic: sum sqrt(dx^2 + dy^2) (pars.tv = 'iso') */
#define CTPRJ_TV_L1 1    /* anisotropic: sum |dx| + |dy| (pars.tv = 'l1') */

/* [D, iter] = denoise_bound_mod(Xobs, lambda, lb, ub, pars) with
 * pars.MAXITER = max_iter, pars.epsilon = epsilon, pars.tv = tv_type
 * (utils/denoise_bound_mod.m:1; TV.denoise, utils/TV.m:56, passes
 * lb = 0, ub = inf).  ub may be +INFINITY.  d_out (rows*cols floats) may not
 * alias d_xobs.  *iterations (may be NULL) receives iter.  Needs rows, cols
 * >= 2, rows * cols < 2^31, lambda > 0, lb < ub. */
int ctprj_tv_denoise(const float *d_xobs, int rows, int cols, double lambda, double lb, double ub,
                     int tv_type, int max_iter, double epsilon, float *d_out, int *iterations,
                     void *stream);

/* *d_tv = tlv(X, tv_type) (utils/tlv.m), in FP64, written to device memory. */
int ctprj_tv_value(const float *d_x, int rows, int cols, int tv_type, double *d_tv, void *stream);

#ifdef __cplusplus
}
#endif

#endif /* CTPRJ_TV_H */

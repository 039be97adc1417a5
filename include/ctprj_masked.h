/*
 * ctprj_masked.h -- the projector in MATLAB's data layout, masked, on the GPU.
 *
 * The reference wraps its projector for MATLAB in two layers of host copies:
 * the MEX gateway transposes the column-major image and casts it to single
 * precision on the way in and back out (prj/mPrj.c:82-84, 134-136), and
 * ConfigCT scatters the reconstruction's masked pixel vector into a zero image
 * before every forward call and gathers it back after every backward call
 * (tomography/ConfigCT.m:122-135 with utils/maskFunc.m).  These entry points
 * take the MATLAB-side arrays in device memory and do the scatter, gather,
 * transposes, casts and the Ts scaling in kernels around ctprj_forward /
 * ctprj_backward / ctprj_fbp:
 *
 *   forward:   d_y = scale * gpuPrj(maskFunc(d_s, mask, [n n]), 0, 'forward')
 *   backward:  d_s = scale * maskFunc(gpuPrj(d_y, 0, 'backward'), mask)
 *   fbp:       d_s = scale * maskFunc(gpuPrj(d_y, 0, 'FBP'), mask)
 *
 * (ConfigCT's Phi and Phit use scale = Ts, its FBP scale = 1/Ts.)  d_mask
 * holds npix distinct 0-based column-major pixel indices (MATLAB's
 * find(mask ~= 0) - 1) as int32; NULL means every pixel in column-major order
 * (npix = n*n), the gateway's own 'forward' / 'backward' / 'FBP'.  Indices
 * outside [0, n*n) are ignored.  d_s: npix doubles; d_y: np*prjWidth doubles
 * in the gateway's order (view-major, prjWidth per view).  The image and
 * sinogram in between are single precision, as in the gateway.  Enqueued on
 * `stream`; the plan's scratch (one image, one sinogram, allocated on first
 * use) serialises calls on one plan.
 *
 * No reference counterpart as a single call: each replaces a MATLAB-side
 * maskFunc plus a gateway call.
 */
#ifndef CTPRJ_MASKED_H
#define CTPRJ_MASKED_H

#include "ctprj.h"

#ifdef __cplusplus
extern "C" {
#endif

int ctprj_masked_forward(ctprj_plan *plan, const int *d_mask, long long npix, const double *d_s,
                         double scale, double *d_y, void *stream);
int ctprj_masked_backward(ctprj_plan *plan, const int *d_mask, long long npix, const double *d_y,
                          double scale, double *d_s, void *stream);
int ctprj_masked_fbp(ctprj_plan *plan, const int *d_mask, long long npix, const double *d_y,
                     double scale, double *d_s, void *stream);

#ifdef __cplusplus
}
#endif

#endif /* CTPRJ_MASKED_H */

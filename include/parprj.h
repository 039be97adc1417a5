/*
 * parprj.h -- double-precision masked parallel-beam operator on the GPU.
 *
 * Drop-in for prj/parPrj.h (the operator behind the mParPrj MEX function,
 * prj/mParPrj.c): forward y = A x / bw and backward x = A^T y / bw over an
 * explicit list of view angles (degrees) and a list of image pixels (0-based
 * column-major indices of an nr x nc image), with the reference's footprint
 * rule (prj/parPrj.c:105-183).  FP64 throughout; computed by CUDA kernels.
 */
#ifndef CTPRJ_PARPRJ_H
#define CTPRJ_PARPRJ_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* prj/parPrj.h:9-16, field for field. */
typedef struct {
    double bw;      /* X-ray beam width */
    int nc, nr;     /* number of columns and rows of the image */
    int np;         /* number of angles in theta */
    int prjWidth;   /* detectors per projection */
    double *theta;  /* angles in degrees */
    int fwd;        /* 1: forward projection, 0: backprojection */
} parConf;

/* Replaces prj/parPrj.c:38-46 (parPrjConf): records the host buffers and the
 * configuration for the next parPrjThread()/parPrjRun().  Forward: t_img holds
 * one value per mask entry and t_prj (np*prjWidth) receives the projection;
 * backward: t_prj is read and t_img (totPixels) receives the result.  As in the
 * reference the output is accumulated onto what the buffer holds and then
 * divided by bw.  Returns 0. */
int parPrjConf(double *t_img, double *t_prj, double *t_maskIdx, parConf *t_opt,
               size_t t_totPixels);

/* Replace prj/parPrj.c:48-79 (parPrjThread, parPrjRun): run the configured
 * operator on the GPU (copies in, kernels, copies out; returns when done).
 * Return 0 or a CTPRJ_* status of include/ctprj.h. */
int parPrjThread(void);
int parPrjRun(void);

/* Device-pointer form.  d_theta: np angles (degrees); d_mask: npix 0-based
 * column-major indices (as doubles, as MATLAB passes them).  Forward:
 * d_y[np*prjWidth] = (d_y + A d_x) / bw; backward: d_x[npix] = (d_x + A^T d_y) / bw. */
typedef struct {
    double bw;
    int nc, nr, np, prjWidth;
} ctprj_par_conf;

int ctprj_par_forward(const ctprj_par_conf *conf, const double *theta_host, const double *d_mask,
                      long long npix, const double *d_x, double *d_y, void *stream);
int ctprj_par_backward(const ctprj_par_conf *conf, const double *theta_host, const double *d_mask,
                       long long npix, const double *d_y, double *d_x, void *stream);

#ifdef __cplusplus
}
#endif

#endif /* CTPRJ_PARPRJ_H */

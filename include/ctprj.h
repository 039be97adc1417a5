/*
 * ctprj.h -- C ABI of the B200 X-ray CT projection engine (imgrecsrc_b200).
 *
 * Drop-in for the projector of anindyabijoydas/imgRecSrc (prj/prj.h:59-70,
 * prj/gpuPrj.cu, prj/parPrj.h): the parallel- and fan-beam forward projector,
 * its matched backprojector, FBP, and the double-precision masked
 * parallel-beam operator behind mParPrj.  All compute runs in hand-written
 * sm_100a CUDA kernels; there is no CPU fallback.  Plain C types only.
 *
 * Conventions (identical to the reference, prj/cpuPrj.c):
 *   image  float[n][n] row-major; pixel (x, y), x, y in [-(n-1)/2, (n-1)/2],
 *          at img[(y + n/2) * n + x + n/2]
 *   sino   float[np][prjWidth] view-major; detector k at
 *          t = (k - prjWidth/2) * dSize on a flat virtual detector through the
 *          isocentre; view i at angle i * 2 * pi / prjFull
 *   d > 0  fan beam with the source at distance d (pixels) from the isocentre;
 *          d <= 0 parallel beam
 *   Outputs are divided by effectiveRate; the beam width is
 *   dSize * effectiveRate.  For even n the image's row 0 and column 0, and for
 *   even prjWidth the sinogram's detector 0, are written as zero.
 *
 * Every entry point returns a status (CTPRJ_OK = 0); none exits the process or
 * resets the device (the reference calls exit() and cudaDeviceReset(),
 * prj/gpuPrj.cu:60-68, :849).
 */
#ifndef CTPRJ_H
#define CTPRJ_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

enum {
    CTPRJ_OK = 0,
    CTPRJ_EINVAL = 1,     /* invalid geometry, argument or NULL pointer */
    CTPRJ_ENOTSETUP = 2,  /* gpuPrj() before a successful setup() */
    CTPRJ_ENOMEM = 3,     /* device or host allocation failed */
    CTPRJ_ECUDA = 4,      /* a CUDA call failed; see ctprj_last_error() */
    CTPRJ_ERANGE = 5,     /* size beyond the limits of this entry point */
    CTPRJ_ETIMEOUT = 6    /* a bounded device-side wait gave up */
};

/* Command bits of gpuPrj()/cpuPrj(), prj/prj.h:29-32. */
#define RENEW_MEM (1)
#define FWD_BIT (1 << 1)
#define BWD_BIT (1 << 2)
#define FBP_BIT (1 << 3)

/* prj/prj.h:42-57, field for field. */
struct prjConf {
    int n;                /* rows and columns of the image */
    int prjWidth;         /* detectors per projection */
    int np;               /* projections computed (views 0 .. np-1) */
    int prjFull;          /* projections in 360 degrees; a multiple of 4 */
    float dSize;          /* detector pitch at the isocentre, pixels */
    float effectiveRate;  /* active fraction of the detector pitch */
    float d;              /* source to isocentre distance, pixels; <= 0: parallel */
    char cmd;
    unsigned int imgSize;
    unsigned int sinoSize;
};

/* ------------------------------------------------------------------------
 * Reference-compatible entry points (host buffers, process-global config).
 * ---------------------------------------------------------------------- */

/* Replaces setup() of prj/gpuPrj.cu:794-865 (declared prj/prj.h:62).  Validates
 * the geometry and builds the device plan and buffers on the current device.
 * Errors are reported by the next gpuPrj() and by ctprj_last_error(). */
void setup(int n, int prjWidth, int np, int prjFull, float dSize,
           float effectiveRate, float d);

/* Replaces showSetup() of prj/gpuPrj.cu:867-875 (prj/prj.h:63). */
void showSetup(void);

/* Replaces gpuPrj() of prj/gpuPrj.cu:887-1047 (prj/prj.h:65).  cmd & FWD_BIT:
 * sino (np*prjWidth) = A img (n*n); cmd & BWD_BIT: img = A^T sino; cmd &
 * FBP_BIT: img = filtered backprojection of sino.  Host pointers; the copies
 * and the kernels run on the default stream and the call returns when img or
 * sino holds the result. */
int gpuPrj(float *img, float *sino, char cmd);

/* prj/gpuPrj.cu:41: the configuration the MEX gateway reads
 * (prj/mPrj.c:28, :72-76). */
extern struct prjConf *pConf;

/* ------------------------------------------------------------------------
 * Plan API: device pointers, caller's stream, no host synchronisation.
 * One plan may be used by one stream at a time (it owns scratch memory).
 * ---------------------------------------------------------------------- */

typedef struct ctprj_geometry {
    int n, prjWidth, np, prjFull;
    float dSize, effectiveRate, d;
} ctprj_geometry;

typedef struct ctprj_plan ctprj_plan;

/* Validates geom and allocates the plan's tables and scratch on `device`
 * (-1: the current device). */
int ctprj_plan_create(const ctprj_geometry *geom, int device, ctprj_plan **plan);
void ctprj_plan_destroy(ctprj_plan *plan);

/* Forward projection, the GPU counterpart of rayDrivePar/rayDriveFan
 * (prj/gpuPrj.cu:419-792): d_sino[np*prjWidth] = A d_img[n*n]. */
int ctprj_forward(ctprj_plan *plan, const float *d_img, float *d_sino, void *stream);

/* Backprojection, the counterpart of pixelDrivePar/pixelDriveFan
 * (prj/gpuPrj.cu:71-417): d_img[n*n] = A^T d_sino[np*prjWidth]. */
int ctprj_backward(ctprj_plan *plan, const float *d_sino, float *d_img, void *stream);

/* Filtered backprojection, the counterpart of cpuPrj/gpuPrj with FBP_BIT
 * (prj/cpuPrj.c:718-784, prj/utils.h:94-151): fan-beam cosine pre-weight,
 * Hann-windowed ramp filter per view, FBP-weighted backprojection.
 * d_img[n*n] from d_sino[np*prjWidth]; d_sino is not modified. */
int ctprj_fbp(ctprj_plan *plan, const float *d_sino, float *d_img, void *stream);

/* Exact number of nonzero operator entries the forward and the backward pass
 * visit (ray-pixel updates per call), counted on the device. */
int ctprj_count_updates(ctprj_plan *plan, long long *fwd, long long *bwd, void *stream);

/* ------------------------------------------------------------------------
 * Polychromatic beam-hardening model (bhc/Spline.m b1Iout, bhc/poissLAlpha.m,
 * bhc/poissLI.m; Gaussian variant below) on a plan.  Per ray i: s_i = Ts (A x)_i, the degree-1
 * B-spline spectrum model BL_i = sum_j Ie_j b_j(s_i) over J basis functions
 * on the J + 2 mass-attenuation nodes kappa (bhc/Spline.m:122-203), and the
 * Poisson negative log-likelihood of the measured intensity m_i (counts / I0):
 *   f = sum_i BL_i - m_i - m_i log(BL_i / m_i)   (0 log 0 := 0),
 * with gradients df/dx = Ts A^T [(1 - m/BL) dBL/ds] and
 * df/dIe_j = sum_i b_j(s_i) (1 - m_i/BL_i).  Spline arithmetic and every
 * reduction are FP64; projections FP32.  One model per stream at a time.
 * ---------------------------------------------------------------------- */

typedef struct ctprj_bhc ctprj_bhc;

/* J in [1, 32]; kappa_nodes: J + 2 increasing positive nodes (cm^2/g);
 * Ts > 0: pixel size (cm).  Allocates per-ray state (2 floats and 1 double per ray). */
int ctprj_bhc_create(ctprj_plan *plan, int J, const double *kappa_nodes, double Ts,
                     ctprj_bhc **model);
void ctprj_bhc_destroy(ctprj_bhc *model);

/* Fused forward: projection and per-ray spline epilogue in one kernel; the
 * likelihood f is reduced in FP64 into d_f (1 double, device).  d_x: n*n
 * float; d_Ie: J doubles; d_imea: np*prjWidth floats.  save != 0 keeps the
 * per-ray state for ctprj_bhc_backward; save == 0 writes nothing per ray. */
int ctprj_bhc_forward(ctprj_bhc *model, const float *d_x, const double *d_Ie,
                      const float *d_imea, double *d_f, int save, void *stream);

/* Gradients of the last forward: d_gx (n*n floats) and d_gIe (J doubles,
 * FP64); either may be NULL.  When the last forward did not save its state,
 * the fused forward is recomputed from d_x, d_Ie, d_imea first. */
int ctprj_bhc_backward(ctprj_bhc *model, const float *d_x, const double *d_Ie,
                       const float *d_imea, float *d_gx, double *d_gIe, void *stream);

/* The same per-ray terms as the fused epilogue, evaluated by a separate kernel
 * over a sinogram d_sino from ctprj_forward (the unfused path). */
int ctprj_bhc_terms(ctprj_bhc *model, const float *d_sino, const double *d_Ie,
                    const float *d_imea, double *d_f, int save, void *stream);

/* The rays x J basis matrix d_A[i*J + j] = b_j(Ts * d_sino[i]) in FP64
 * (Spline.b1Iout with an empty spectrum, bhc/Spline.m:143), for spectrum
 * solvers that work on the matrix. */
int ctprj_bhc_basis(ctprj_bhc *model, const float *d_sino, double *d_A, void *stream);

/* Device pointers of the saved per-ray state (np*prjWidth entries each): s_i
 * (float), r_i = df/dBL_i (double; 1 - m_i/BL_i for the Poisson model) and
 * r_i dBL/ds (float). */
int ctprj_bhc_state(ctprj_bhc *model, const float **d_s, const double **d_r, const float **d_w);

/* Noise model of the likelihood.  CTPRJ_NOISE_POISSON (the default):
 * bhc/poissLAlpha.m, bhc/poissLI.m as above.  CTPRJ_NOISE_GAUSSIAN: the
 * log-domain least squares of bhc/gaussLAlpha.m and bhc/gaussLI.m,
 *   Err_i = log(BL_i / m_i),  f = sum_i Err_i^2 / 2,
 *   df/dx = Ts A^T [Err/BL dBL/ds],  df/dIe_j = sum_i b_j(s_i) Err_i / BL_i,
 * which needs m_i > 0.  Switching the model discards the saved state. */
#define CTPRJ_NOISE_POISSON 0
#define CTPRJ_NOISE_GAUSSIAN 1
int ctprj_bhc_set_noise(ctprj_bhc *model, int noise);

/* Density Hessian of f at the saved state (the `hessian` closures of
 * bhc/poissLAlpha.m:15-28 and bhc/gaussLAlpha.m:18-31): with y = Ts A v and
 * the per-ray weight h_i = q_i (dBL/ds)^2 + r_i d2BL/ds2 (q = d2f/dBL2:
 * m/BL^2 Poisson, (1 - Err)/BL^2 Gaussian),
 *   d_Hv  (n*n floats, may be NULL)       = Ts A^T (h y)     (opt = 1),
 *   d_vHv (1 double on the device, NULL)  = sum_i h_i y_i^2  (opt = 2).
 * d_Ie and d_imea must be those of the saved forward.  FP64 spline and
 * reduction; one forward projection, plus one backprojection for d_Hv. */
int ctprj_bhc_hessian(ctprj_bhc *model, const double *d_Ie, const float *d_imea, const float *d_v,
                      float *d_Hv, double *d_vHv, void *stream);

/* Static description of a status code, and the message of the last failure on
 * the calling thread. */
const char *ctprj_error_string(int status);
const char *ctprj_last_error(void);

#ifdef __cplusplus
}
#endif

#endif /* CTPRJ_H */

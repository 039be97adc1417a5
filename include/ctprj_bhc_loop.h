/*
 * ctprj_bhc_loop.h -- the alternating beam-hardening reconstruction on the GPU.
 *
 * Counterpart of the reference's BHC driver loop (bhc/beamhardenSpline.m:
 * 340-570): one density step on the likelihood (the reference's NPG class,
 * npg/NPG.m, or its PG class, npg/PG.m, with the non-negativity projection,
 * the TV denoising of include/ctprj_tv.h or the wavelet ADMM of
 * include/ctprj_wavelet.h as the proximal map),
 * then a non-negative spectrum step, repeated.  Built on the model of
 * include/ctprj.h (ctprj_bhc_*): every likelihood and gradient of the density
 * step comes from the fused forward projection and its adjoint; the spectrum
 * step is a Newton method on Ie >= 0 whose gradient, Hessian, bound-
 * constrained quadratic subproblem (active set, J x J Cholesky) and line
 * search run in FP64 on the GPU (bhc/ActiveSet.m is the reference's
 * active-set Newton method for the same objective, bhc/poissLI.m).
 */
#ifndef CTPRJ_BHC_LOOP_H
#define CTPRJ_BHC_LOOP_H

#include "ctprj.h"
#include "ctprj_wavelet.h"

#ifdef __cplusplus
extern "C" {
#endif

#define CTPRJ_BHC_LOOP_MAX_TRACE 256

/* initial density step (the reference's stepSizeInit, npg/Methods.m:98-124) */
#define CTPRJ_STEP_FIXED 0    /* 1/t = x_step */
#define CTPRJ_STEP_BB 1       /* finite-difference curvature along the gradient
                                 (the reference's default, bhc/beamhardenSpline.m:73) */
#define CTPRJ_STEP_HESSIAN 2  /* t = |g'Hg| / g'g from ctprj_bhc_hessian */

/* density step method */
#define CTPRJ_DENSITY_NPG 0   /* Nesterov proximal gradient with restart (npg/NPG.m,
                                 the reference's default, bhc/beamhardenSpline.m:37) */
#define CTPRJ_DENSITY_PG 1    /* proximal (projected) gradient (npg/PG.m) */

/* proximal map of the density step (opt.proximal, bhc/beamhardenSpline.m:199-223) */
#define CTPRJ_PROX_NONNEG 0   /* 'nonneg': x >= 0, no penalty */
#define CTPRJ_PROX_TV_ISO 1   /* 'tviso': u TV_iso(x) + (x >= 0), TV.denoise(..., 'iso') */
#define CTPRJ_PROX_TV_L1 2    /* 'tvl1':  u TV_l1(x) + (x >= 0), TV.denoise(..., 'l1') */
#define CTPRJ_PROX_WVLT_ADMM 3  /* 'wvltADMM' (the reference's default): u |Psit(x)|_1 + (x >= 0),
                                   admm(Psi, Psit, ...) of npg/admm.m, include/ctprj_wavelet.h */

typedef struct {
    int iterations;             /* alternating iterations */
    double x_step;              /* initial density step 1/t (<= 0: 1) */
    int spectrum_newton_steps;  /* at most this many Newton steps per spectrum
                                   update (<= 0: 2); fewer when converged */
    int skip_spectrum;          /* 1: density steps only */
    int unfused;                /* 1: every likelihood from the plain forward projection
                                   plus a separate spectrum-terms kernel (comparison) */
    int init_step;              /* CTPRJ_STEP_*: how the first 1/t is chosen */
    int density_method;         /* CTPRJ_DENSITY_* */
    double thresh;              /* > 0: stop once the density's relative change
                                   |x_new - x| / |x| has been <= thresh in three
                                   iterations after the first, and more than
                                   min_iterations have run (bhc/beamhardenSpline.m:
                                   563-566); <= 0: run `iterations` */
    int min_iterations;
    int proximal;               /* CTPRJ_PROX_* */
    double u;                   /* penalty weight of the TV proximal maps (opt.u) */
    int max_inner;              /* first maxInnerItr of the TV map (<= 0: 100, npg/NPG.m:23) */
    double admm_tol;            /* first admmTol (opt.admmTol; <= 0: 1e-2, npg/NPG.m:11);
                                   the TV map's tolerance is admmTol * difAlpha */
    int no_restart;             /* 1: opt.restart = false (NPG without momentum restart) */
    int no_adaptive_step;       /* 1: opt.adaptiveStep = false (no step growth after
                                   cumu_tol first-try successes) */
    int cumu_tol;               /* opt.cumuTol (<= 0: 4) */
    int wvlt_filter_len;        /* CTPRJ_PROX_WVLT_ADMM: scaling filter length (<= 0: 2, Haar) */
    double wvlt_filter[CTPRJ_WVLT_MAX_FILTER];   /* its taps, daubcqf(daub) (unused when <= 0) */
    int wvlt_levels;            /* dwt_L (<= 0: 6, bhc/doBHC.m:33); n divisible by 2^dwt_L */
    const unsigned char *mask;  /* opt.mask: device n x n bytes, nonzero = a pixel of the
                                   reconstruction (the density is 0 elsewhere, its gradient
                                   and proximal maps are restricted to it); NULL: all pixels */
    const unsigned char *wvlt_mask;  /* maskk: device n x n bytes over the coefficient array,
                                   the coefficients of Psit (utils/Utils.m:445-469); NULL:
                                   those the mask reaches (utils/wvltMask.m), or all */
    int pre_steps;              /* opt.preSteps: iterations in which a successful step is
                                   retried with a larger one (<= 0: 2, the BHC driver's
                                   default, bhc/beamhardenSpline.m:74, :304) */
} ctprj_bhc_loop_opts;

typedef struct {
    int iterations;                           /* completed */
    double final_cost;                        /* f after the last step */
    double final_x_step;                      /* density step 1/t at the end */
    double cost[CTPRJ_BHC_LOOP_MAX_TRACE];    /* f after each iteration */
    double x_step[CTPRJ_BHC_LOOP_MAX_TRACE];  /* density step accepted in each
                                                 iteration (0: x kept) */
    float ms;                                 /* device time of the loop */
    float ms_spectrum;                        /* of which spectrum steps */
    int evaluations;                          /* likelihood evaluations (each one
                                                 forward projection) */
    int restarts;                             /* momentum restarts */
    int newton_steps;                         /* accepted spectrum Newton steps */
    int converged;                            /* 1: stopped by the thresh rule */
    double x_change[CTPRJ_BHC_LOOP_MAX_TRACE];  /* |x_new - x| / |x| of each iteration */
    int inner_iterations;                     /* TV denoising iterations, all steps */
    int prox_retries;                         /* steps retried with a tighter TV map
                                                 (admmTol / 10 or maxInnerItr * 10) */
    double penalty;                           /* u TV of the last density candidate */
} ctprj_bhc_loop_stats;

/* Spectrum update on the projections of the last forward saved by the model
 * (ctprj_bhc_forward with save != 0): at most newton_steps (>= 1) Newton steps
 * on Ie >= 0 (d_Ie: J doubles, updated in place), each minimising the
 * quadratic model over Ie >= 0 and then backtracking (x0.8) to sufficient
 * decrease; stops early when the model predicts no decrease.  *f_out receives
 * f at the returned Ie.  Synchronises `stream`. */
int ctprj_bhc_spectrum_step(ctprj_bhc *model, const float *d_imea, double *d_Ie, int newton_steps,
                            double *f_out, void *stream);

/* The alternating loop on density d_x (n*n floats, updated in place) and
 * spectrum d_Ie (updated in place) for measurement d_imea.  Synchronises
 * `stream` between steps. */
int ctprj_bhc_reconstruct(ctprj_bhc *model, float *d_x, double *d_Ie, const float *d_imea,
                          const ctprj_bhc_loop_opts *opts, ctprj_bhc_loop_stats *stats,
                          void *stream);

#ifdef __cplusplus
}
#endif

#endif /* CTPRJ_BHC_LOOP_H */

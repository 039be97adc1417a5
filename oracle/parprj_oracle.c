/*
 * parprj_oracle.c -- TEST INFRASTRUCTURE ONLY (the oracle).
 *
 * CPU restatement of the reference's double-precision parallel-beam operator
 * over an explicit angle list and a pixel mask (prj/parPrj.c, called from the
 * MEX gateway prj/mParPrj.c).  Checker for the GPU parPrj path; never linked
 * into the product.  Always double precision, as in the reference.
 *
 * Reference behaviour restated on purpose:
 *  - the footprint shape uses the angle |trunc(fmod(theta, 90) - 45)| in whole
 *    degrees: prj/parPrj.c:111 passes a double to the integer abs();
 *  - pi is the truncated constant 3.14159265 (prj/parPrj.c:29);
 *  - detector k (unit pitch, centre at max(nc, nr)/2) is skipped when
 *    k + pC falls outside [0, nc) (prj/parPrj.c:170); this restatement also
 *    skips k + pC >= prjWidth, where the reference would index past the view;
 *  - a beam wider than the whole footprint takes the reference's branch value
 *    area - areaT * ((bias2 - u_r) / (bias2 - bias1))^2 (prj/parPrj.c:140-141);
 *  - the result is divided by the beam width (prj/parPrj.c:72-77).
 */
#include <math.h>
#include <stdlib.h>
#include <stddef.h>
#include "ora_threads.h"

typedef struct {
    double bw;            /* beam width */
    int nc, nr;           /* image columns and rows */
    int np;               /* number of angles */
    int prjWidth;         /* detectors per view */
    const double *theta;  /* angles in degrees, length np */
} ora_par_conf;

#define PAR_PI 3.14159265
#define PAR_EPS 1e-8

typedef struct { double height, b1, b2, areaT, areaR, c, s; } par_view;

static par_view par_view_of(double theta)
{
    par_view v;
    int whole = (int)(fmod(theta, 90) - 45);     /* integer abs() of a double */
    if (whole < 0) whole = -whole;
    double tmp = whole * PAR_PI / 180;
    v.height = 1 / sin(tmp + PAR_PI / 4);
    v.b1 = sqrt(2.0) / 2 * sin(tmp);
    v.b2 = sqrt(2.0) / 2 * cos(tmp);
    v.areaT = 0.5 * v.height * (v.b2 - v.b1);
    v.areaR = v.height * v.b1 * 2;
    v.c = cos(theta * PAR_PI / 180);
    v.s = sin(theta * PAR_PI / 180);
    return v;
}

/* prj/parPrj.c:133-168: overlap of the detector-k beam [k-hb, k+hb] with the
 * trapezoid centred at dist, split by the zones of the two beam edges. */
static double par_overlap(const par_view *v, double dist, double k, double bw)
{
    const double hb = bw / 2, w = v->b2 - v->b1, H = v->height;
    const double ul = k - hb - dist, ur = k + hb - dist;
    const double aT = v->areaT, aR = v->areaR;
    /* zones of an edge: 0 left of the left foot, 1 rising, 2 plateau, 3 beyond */
    int zl = ul <= -v->b2 ? 0 : ul <= -v->b1 ? 1 : ul <= v->b1 ? 2 : 3;
    double rise_l = aT * (1 - pow((ul + v->b2) / w, 2));   /* rising part right of ul */
    switch (zl) {
    case 0:
        if (ur <= -v->b1) return aT * pow((ur + v->b2) / w, 2);
        if (ur <= v->b1) return aT + H * (ur + v->b1);
        return aT * 2 + aR - aT * pow((v->b2 - ur) / w, 2);
    case 1:
        if (ur <= -v->b1) return H / w * (k - dist + v->b2) * bw;
        if (ur <= v->b1) return rise_l + H * (ur + v->b1);
        if (ur <= v->b2) return rise_l + aR + aT * (1 - pow((v->b2 - ur) / w, 2));
        return rise_l + aR + aT;
    case 2:
        if (ur <= v->b1) return H * bw;
        if (ur <= v->b2) return H * (v->b1 - ul) + aT * (1 - pow((v->b2 - ur) / w, 2));
        return H * (v->b1 - ul) + aT;
    default:
        if (ur <= v->b2) return H / w * (dist + v->b2 - k) * bw;
        return 0.5 * H / w * pow(dist + v->b2 - k + hb, 2);
    }
}

/* Walks the detectors one masked pixel touches at angle index it; fwd adds
 * w * img[i] into the view row, bwd adds w * row into img[i]. */
static void par_pixel(const ora_par_conf *cf, const par_view *v, int fwd,
                      double *img_i, double *row, const double *mask_i)
{
    const int xC = cf->nc / 2, yC = cf->nr / 2, pC = xC > yC ? xC : yC;
    const int idx = (int)(*mask_i);
    const int x = idx / cf->nr - xC, y = idx % cf->nr - yC;
    const double dist = x * v->c + y * v->s;
    const double ub = floor(dist + v->b2 + cf->bw / 2 - PAR_EPS);
    const double lb = ceil(dist - v->b2 - cf->bw / 2 + PAR_EPS);
    for (int k = (int)lb; k <= ub; k++) {
        double w = par_overlap(v, dist, (double)k, cf->bw);
        if (k < -pC || k + pC >= cf->nc || k + pC >= cf->prjWidth) continue;
        if (w == 0) continue;
        if (fwd) row[k + pC] += w * (*img_i);
        else *img_i += row[k + pC] * w;
    }
}

/* Forward: prj (np x prjWidth, zero on entry) += A * img over the masked
 * pixels; img has one value per mask entry.  prj/parPrj.c:52-63, :105-183. */
typedef struct {
    const ora_par_conf *cf; const double *maskIdx; long long npix;
    double *img; double *prj; const par_view *views;
} par_ctx;

static void par_fwd_body(long long it, void *vc, long long *acc)
{
    par_ctx *c = (par_ctx *)vc;
    double *row = c->prj + (size_t)c->cf->prjWidth * it;
    for (long long i = 0; i < c->npix; i++)
        par_pixel(c->cf, &c->views[it], 1, &c->img[i], row, &c->maskIdx[i]);
    (void)acc;
}

static void par_bwd_body(long long i, void *vc, long long *acc)
{
    par_ctx *c = (par_ctx *)vc;
    for (int it = 0; it < c->cf->np; it++)
        par_pixel(c->cf, &c->views[it], 0, &c->img[i],
                  c->prj + (size_t)c->cf->prjWidth * it, &c->maskIdx[i]);
    (void)acc;
}

int ora_par_forward(const ora_par_conf *cf, const double *img, const double *maskIdx,
                    long long npix, double *prj, int nthreads)
{
    par_view *views = (par_view *)malloc(sizeof(par_view) * (size_t)(cf->np > 0 ? cf->np : 1));
    if (!views) return -1;
    for (int it = 0; it < cf->np; it++) views[it] = par_view_of(cf->theta[it]);
    par_ctx c = { cf, maskIdx, npix, (double *)img, prj, views };
    ora_parallel_for(cf->np, nthreads, 1, par_fwd_body, &c);
    for (size_t i = 0; i < (size_t)cf->np * cf->prjWidth; i++) prj[i] /= cf->bw;
    free(views);
    return 0;
}

/* Backward: img (one value per mask entry, zero on entry) += A^T * prj. */
int ora_par_backward(const ora_par_conf *cf, const double *prj, const double *maskIdx,
                     long long npix, double *img, int nthreads)
{
    par_view *views = (par_view *)malloc(sizeof(par_view) * (size_t)(cf->np > 0 ? cf->np : 1));
    if (!views) return -1;
    for (int it = 0; it < cf->np; it++) views[it] = par_view_of(cf->theta[it]);
    par_ctx c = { cf, maskIdx, npix, img, (double *)prj, views };
    ora_parallel_for(npix, nthreads, 256, par_bwd_body, &c);
    for (long long i = 0; i < npix; i++) img[i] /= cf->bw;
    free(views);
    return 0;
}

/*
 * ctprj_oracle.c -- TEST INFRASTRUCTURE ONLY (the oracle).
 *
 * A CPU restatement of the reference X-ray CT projector of
 * anindyabijoydas/imgRecSrc (prj/cpuPrj.c, prj/utils.h).  It is the checker
 * used by tests/, by __graft_entry__.smoke() and by the cpu_baseline leg of
 * bench.py.  The product library (imgrecsrc_b200) never links, loads or calls
 * anything in this file, and has no CPU fallback to it.
 *
 * Built twice by oracle/Makefile: with ORA_REAL=double (the FP64 oracle that
 * parity is measured against) and ORA_REAL=float (the arithmetic width of the
 * shipped reference).  The restatement is pinned against the reference's own
 * prj/cpuPrj.c compiled from source (oracle/Makefile target `ref`) and against
 * the committed fixtures in tests/golden/.
 *
 * Conventions restated from the reference (all cited per function below):
 *   image  img[(y + n/2) * n + (x + n/2)], x, y in [-(n-1)/2, (n-1)/2]
 *   sino   sino[view * prjWidth + k], detector k at t = (k - prjWidth/2) * dSize
 *   view i at angle fl(fl(2i * PI_f) / prjFull), PI_f the float pi literal
 *   d > 0 selects fan beam (flat virtual detector through the isocentre)
 *   outputs are divided by effectiveRate
 *   even n: row 0 and column 0 of the image are zero; even prjWidth:
 *   detector 0 is zero.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include <stdint.h>
#include "ora_threads.h"

#ifndef ORA_REAL
#define ORA_REAL double
#endif
typedef ORA_REAL real;

/* prj/prj.h:9 -- the reference's pi is a float literal, and view angles are
 * formed in float arithmetic in both of its precisions (prj/cpuPrj.c:78,215,
 * 342,491: `thetaIdx*2*PI/conf->prjFull`). */
#define REF_PI_F 3.14159265359f

typedef struct {
    int n, prjWidth, np, prjFull;
    double dSize, effectiveRate, d;
    int fbp;      /* backward only: FBP weighting (prj/cpuPrj.c:161-163,258,304-306) */
} ora_geom;

static double view_angle(int i, int P)
{
    float th = (float)(2 * i) * REF_PI_F;
    th = th / (float)P;
    return (double)th;
}

static inline real clampr(real v, real lo, real hi)
{
    return v < lo ? lo : (v > hi ? hi : v);
}

/* Area, in units of the plateau height, of the symmetric trapezoid with feet
 * at +-b2 and shoulders at +-b1, from -inf up to u. */
static inline real trap_cdf(real u, real b1, real b2)
{
    real w = b2 - b1;
    real p = clampr(u + b2, 0, w);
    real q = clampr(u + b1, 0, 2 * b1);
    real r = clampr(u - b1, 0, w);
    real quad = w > 0 ? (p * p - r * r) / (2 * w) : 0;
    return quad + q + r;
}

/* prj/utils.h:12-91 (getWeight): overlap of a beam of width bw centred on the
 * ray with the projected footprint of a unit pixel whose centre lies at signed
 * distance dist from the ray; (c, s) is the ray direction.  The footprint is a
 * trapezoid of height 1/max(|c|,|s|), feet at +-(|c|+|s|)/2 and shoulders at
 * +-||c|-|s||/2.  Restated as a difference of the trapezoid's cumulative area
 * at the two beam edges. */
real ora_weight(real dist, real bw, real c, real s)
{
    c = c < 0 ? -c : c;
    s = s < 0 ? -s : s;
    real hi = c > s ? c : s, lo = c > s ? s : c;
    real h = 1 / hi, b2 = (hi + lo) / 2, b1 = (hi - lo) / 2;
    real hb = bw / 2;
    return h * (trap_cdf(hb - dist, b1, b2) - trap_cdf(-hb - dist, b1, b2));
}

/* The eight images g(x, y) of a pixel under the square's symmetry group, in the
 * order the reference accumulates them (prj/cpuPrj.c:383-397 forward,
 * :308-316 backward):  (x,y) (-y,x) (-x,-y) (y,-x) (x,-y) (y,x) (-x,y) (-y,-x). */
static const int GXX[8] = { 1, 0, -1, 0, 1, 0, -1, 0 };
static const int GXY[8] = { 0, -1, 0, 1, 0, 1, 0, -1 };
static const int GYX[8] = { 0, 1, 0, -1, 0, 1, 0, -1 };
static const int GYY[8] = { 1, 0, -1, 0, -1, 0, 1, 0 };
/* View of image j for base view b: (VQ[j] * P/4 + VS[j] * b) mod P; images
 * 4..7 also mirror the detector (prj/cpuPrj.c:403-460, :117-157). */
static const int VQ[8] = { 0, 1, 2, 3, 2, 3, 4, 1 };
static const int VS[8] = { 1, 1, 1, 1, -1, -1, -1, -1 };
/* Point reflection partner of image j (parallel beam writes both). */
static const int PART[8] = { 2, 3, 0, 1, 6, 7, 4, 5 };

static inline int view_of(int j, int b, int P)
{
    int v = VQ[j] * (P / 4) + VS[j] * b;
    v %= P;
    if (v < 0) v += P;
    return v;
}

static inline size_t pix_index(int n, int x, int y)
{
    return (size_t)(y + n / 2) * (size_t)n + (size_t)(x + n / 2);
}

/* ---------------------------------------------------------------- forward */

/* One base ray (view b <= prjFull/8, detector k): the eight symmetric ray
 * sums.  Parallel beam: prj/cpuPrj.c:319-399; fan beam: :463-573. */
static long long base_ray(const ora_geom *g, const real *img, int b, int k,
                          real S[8])
{
    const int N = g->n, half = (N - 1) / 2, pC = g->prjWidth / 2;
    const real beamWidth = (real)(g->dSize * g->effectiveRate);
    const real hbw = beamWidth / 2;
    const double th = view_angle(b, g->prjFull);
    const real cosT = (real)cos(th), sinT = (real)sin(th);
    const real t = (real)((k - pC) * g->dSize);
    const real tl = t - hbw, tr = t + hbw;
    const int fan = g->d > 0;
    long long nnz = 0;
    for (int j = 0; j < 8; j++) S[j] = 0;

    real d = (real)g->d, bq = 0, cosB = 1, sinB = 0, cosR = cosT, sinR = sinT;
    real bwc = beamWidth, off = t;
    real dtl = 0, dtr = 0, qxl = 0, qxr = 0, qyl = 1, qyr = 1;
    if (fan) {
        bq = (real)sqrt(d * d + t * t);
        cosB = d / bq; sinB = t / bq;
        cosR = cosB * cosT - sinB * sinT;
        sinR = sinB * cosT + cosB * sinT;
        bwc = beamWidth * cosB;
        off = d * t / bq;
        /* the two beam edges, as lines through the source (:514-516) */
        dtl = d * tl; dtr = d * tr;
        qxl = tl * cosT + d * sinT; qxr = tr * cosT + d * sinT;
        qyl = -tl * sinT + d * cosT; qyr = -tr * sinT + d * cosT;
    }
    for (int y = half; y >= -half; y--) {
        real xl, xr;
        if (fan) {
            xl = qxl > 0 ? (dtl - qxl * (real)(y + 0.5)) / qyl
                         : (dtl - qxl * (real)(y - 0.5)) / qyl;
            xr = qxr > 0 ? (dtr - qxr * (real)(y - 0.5)) / qyr
                         : (dtr - qxr * (real)(y + 0.5)) / qyr;
        } else {
            xl = (tl - sinT * (real)(y + 0.5)) / cosT;
            xr = (tr - sinT * (real)(y - 0.5)) / cosT;
        }
        int x0 = (int)round(xl), x1 = (int)round(xr);
        if (x0 < -half) x0 = -half;
        if (x1 > half) x1 = half;
        for (int x = x0; x <= x1; x++) {
            real dist = x * cosR + y * sinR - off;
            real bw = fan ? bwc + (x * sinT - y * cosT) * bwc / d : beamWidth;
            real w = ora_weight(dist, bw, cosR, sinR);
            if (w != 0) nnz++;
            if (img) {
                for (int j = 0; j < 8; j++) {
                    int gx = GXX[j] * x + GXY[j] * y, gy = GYX[j] * x + GYY[j] * y;
                    S[j] += w * img[pix_index(N, gx, gy)];
                }
            }
        }
    }
    return nnz;
}

/* Scatter of the eight sums of base ray (b, k) (prj/cpuPrj.c:401-460 and
 * :575-615).  Returns the number of distinct sinogram entries written. */
static int write_ray(const ora_geom *g, real *sino, int b, int k,
                     const real S[8])
{
    const int P = g->prjFull, W = g->prjWidth, pC = W / 2, fan = g->d > 0;
    const real er = (real)g->effectiveRate;
    const int mirror = b > 0 && (float)b < (float)P * 0.125f;
    int written = 0;
    for (int j = 0; j < 8; j++) {
        if (j >= 4 && !mirror) break;
        int v = view_of(j, b, P);
        if (v >= g->np) continue;
        int det = j < 4 ? k : 2 * pC - k;
        if (sino) sino[(size_t)v * W + det] = S[j] / er;
        written++;
        if (!fan) {
            if (sino) sino[(size_t)v * W + (2 * pC - det)] = S[PART[j]] / er;
            if (2 * pC - det != det) written++;
        }
    }
    return written;
}

static void ray_set(const ora_geom *g, int *nb, int *k0, int *nk)
{
    const int W = g->prjWidth, fan = g->d > 0;
    *nb = g->np < g->prjFull / 8 + 1 ? g->np : g->prjFull / 8 + 1;
    *k0 = (W % 2 == 0) ? 1 : 0;
    if (fan) *nk = (W % 2 == 0) ? W - 1 : W;
    else *nk = (W % 2 == 0) ? W / 2 : (W + 1) / 2;
}

int ora_check(const ora_geom *g)
{
    if (!g || g->n < 1 || g->prjWidth < 1 || g->np < 1 || g->prjFull < 4 ||
        g->prjFull % 4 != 0 || g->np > g->prjFull || !(g->dSize > 0) ||
        !(g->effectiveRate > 0))
        return -1;
    return 0;
}

typedef struct { const ora_geom *g; const real *img; real *sino; int k0, nk; } fwd_ctx;

static void fwd_body(long long r, void *vc, long long *acc)
{
    fwd_ctx *c = (fwd_ctx *)vc;
    int b = (int)(r / c->nk), k = c->k0 + (int)(r % c->nk);
    real S[8];
    long long nz = base_ray(c->g, c->img, b, k, S);
    int written = write_ray(c->g, c->sino, b, k, S);
    if (!c->img) *acc += nz * written;
}

/* prj/cpuPrj.c:679-705 with cmd = FWD_BIT. */
int ora_forward(const ora_geom *g, const real *img, real *sino, int nthreads)
{
    if (ora_check(g)) return -1;
    int nb, k0, nk;
    ray_set(g, &nb, &k0, &nk);
    fwd_ctx c = { g, img, sino, k0, nk };
    ora_parallel_for((long long)nb * nk, nthreads, 16, fwd_body, &c);
    if (g->prjWidth % 2 == 0)
        for (int v = 0; v < g->np; v++) sino[(size_t)v * g->prjWidth] = 0;
    return 0;
}

/* Number of nonzero entries of the forward operator (sinogram entries x
 * pixels), i.e. the ray-pixel updates one forward projection performs. */
long long ora_forward_nnz(const ora_geom *g, int nthreads)
{
    if (ora_check(g)) return -1;
    int nb, k0, nk;
    ray_set(g, &nb, &k0, &nk);
    fwd_ctx c = { g, NULL, NULL, k0, nk };
    return ora_parallel_for((long long)nb * nk, nthreads, 16, fwd_body, &c);
}

/* --------------------------------------------------------------- backward */

/* One octant pixel (0 <= y <= x): the eight symmetric pixel sums.  Parallel
 * beam: prj/cpuPrj.c:46-159 (views 0..prjFull/2-1, each weight also serving
 * the opposite view with the mirrored detector); fan beam: :176-301. */
static long long octant_pixel(const ora_geom *g, const real *sino, int x, int y,
                              int nimg, real S[8])
{
    const int P = g->prjFull, W = g->prjWidth, pC = W / 2, fan = g->d > 0;
    const int dmax = (W - 1) / 2;
    const real dS = (real)g->dSize, d = (real)g->d;
    const real beamWidth = (real)(g->dSize * g->effectiveRate);
    const int nviews = fan ? P : P / 2;
    long long nnz = 0;
    for (int j = 0; j < 8; j++) S[j] = 0;

    for (int i = 0; i < nviews; i++) {
        const double th = view_angle(i, P);
        const real c = (real)cos(th), s = (real)sin(th);
        const real xm = (real)(x - 0.5), xp = (real)(x + 0.5);
        const real ym = (real)(y - 0.5), yp = (real)(y + 0.5);
        real cx[4] = { xm, xp, xp, xm }, cy[4] = { ym, ym, yp, yp };
        real tl = 0, tr = 0, qe = 0;
        for (int q = 0; q < 4; q++) {
            real oc = cx[q] * c + cy[q] * s, tq;
            if (fan) tq = d * oc / (cx[q] * s - cy[q] * c + d);
            else tq = oc;
            if (q == 0 || tq < tl) tl = tq;
            if (q == 0 || tq > tr) tr = tq;
        }
        if (fan) qe = x * s - y * c + d;
        int dl = (int)round(tl / dS), dr = (int)round(tr / dS);
        if (dl < -dmax) dl = -dmax;
        if (dr > dmax) dr = dmax;
        for (int dt = dl; dt <= dr; dt++) {
            real t = dt * dS, w;
            if (fan) {
                real bq = (real)sqrt(d * d + t * t);
                real cosB = d / bq, sinB = t / bq;
                real cosR = cosB * c - sinB * s, sinR = sinB * c + cosB * s;
                real dist = x * cosR + y * sinR - d * t / bq;
                w = ora_weight(dist, qe * beamWidth * cosB / d, cosR, sinR);
                if (g->fbp) w = w * d * d / qe / qe;
            } else {
                w = ora_weight(x * c + y * s - t, beamWidth, c, s);
            }
            if (w == 0) continue;
            for (int j = 0; j < 8; j++) {
                int sg = j < 4 ? 1 : -1;
                int v = view_of(j, i, P);
                if (v < g->np) {
                    if (j < nimg) nnz++;
                    if (sino) S[j] += w * sino[(size_t)v * W + pC + sg * dt];
                }
                if (!fan) {
                    int v2 = (v + P / 2) % P;
                    if (v2 < g->np) {
                        if (j < nimg) nnz++;
                        if (sino) S[j] += w * sino[(size_t)v2 * W + pC - sg * dt];
                    }
                }
            }
        }
    }
    return nnz;
}

typedef struct { const ora_geom *g; const real *sino; real *img; real fbps, er; } bwd_ctx;

/* octant pixel number r -> (x, y) with 0 <= y <= x, row by row of x */
static void octant_xy(long long r, int *x, int *y)
{
    int xx = 0;
    long long yy = r;
    while (yy > xx) { xx++; yy -= xx; }
    *x = xx; *y = (int)yy;
}

static void bwd_body(long long r, void *vc, long long *acc)
{
    bwd_ctx *c = (bwd_ctx *)vc;
    int x, y;
    octant_xy(r, &x, &y);
    real S[8];
    /* on the diagonal and the axis only four of the images are distinct */
    int nimg = (y == 0 || y >= x) ? 4 : 8;
    long long nz = octant_pixel(c->g, c->sino, x, y, nimg, S);
    if (!c->img) { *acc += nz; return; }
    for (int j = 0; j < nimg; j++) {
        real v = c->g->fbp ? S[j] * c->fbps : S[j];
        int gx = GXX[j] * x + GXY[j] * y, gy = GYX[j] * x + GYY[j] * y;
        c->img[pix_index(c->g->n, gx, gy)] = v / c->er;
    }
}

/* prj/cpuPrj.c:706-717 (BWD_BIT) and :161-173, :303-316 (writes). */
int ora_backward(const ora_geom *g, const real *sino, real *img, int nthreads)
{
    if (ora_check(g)) return -1;
    const int N = g->n, half = (N - 1) / 2, no = half + 1;
    const real er = (real)g->effectiveRate;
    /* prj/cpuPrj.c:161,304: FBP scale PI/np/dSize/dSize (float pi / int) */
    const real fbps = (real)(REF_PI_F / (float)g->np) / (real)g->dSize / (real)g->dSize;
    bwd_ctx c = { g, sino, img, fbps, er };
    ora_parallel_for((long long)no * (no + 1) / 2, nthreads, 8, bwd_body, &c);
    if (N % 2 == 0)
        for (int i = 0; i < N; i++) { img[i] = 0; img[(size_t)i * N] = 0; }
    return 0;
}

/* Nonzero (pixel, sinogram entry) pairs the backprojector visits. */
long long ora_backward_nnz(const ora_geom *g, int nthreads)
{
    if (ora_check(g)) return -1;
    const int half = (g->n - 1) / 2, no = half + 1;
    bwd_ctx c = { g, NULL, NULL, 0, 1 };
    return ora_parallel_for((long long)no * (no + 1) / 2, nthreads, 8, bwd_body, &c);
}

int ora_real_bytes(void) { return (int)sizeof(real); }

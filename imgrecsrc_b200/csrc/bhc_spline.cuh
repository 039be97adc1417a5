// bhc_spline.cuh -- FP64 evaluation of the degree-1 B-spline mass-attenuation
// basis of the polychromatic model (bhc/Spline.m:122-203, b1Iout).
//
// For nodes a < b < c of basis function j,
//   b_j(s)  = -(e^{-as} - e^{-bs}) / (s^2 (a-b)) + (e^{-bs} - e^{-cs}) / (s^2 (b-c))
//   b_j'(s) = 2(e^{-as}-e^{-bs})/(s^3(a-b)) + (a e^{-as} - b e^{-bs})/(s^2(a-b))
//           - 2(e^{-bs}-e^{-cs})/(s^3(b-c)) - (b e^{-bs} - c e^{-cs})/(s^2(b-c))
// and, for |s| below a per-function threshold, the cubic Taylor polynomials the
// reference substitutes (its 1/s terms cancel there).  The J + 2 exponentials
// of a ray are rolled along the nodes.  Everything here is double precision:
// the cancellation costs up to ~3 digits, which FP32 cannot spare.
#pragma once

namespace ctprj {

constexpr int kMaxJ = 32;
// per basis function: a, b, c, 1/(a-b), 1/(b-c), Taylor B[4], thrB, Taylor D[4], thrD
constexpr int kSplStride = 15;

struct SplineEval {
    double BL, sBL;
};

// table: J * kSplStride doubles (shared memory); Ie: J doubles (shared memory)
__device__ __forceinline__ SplineEval b1_eval(double s, const double *tab, const double *Ie, int J)
{
    const double s2 = s * s, is2 = 1.0 / s2, is3 = is2 / s, as = fabs(s);
    double eL = exp(-tab[0] * s), eC = exp(-tab[1] * s);
    SplineEval r = {0.0, 0.0};
    for (int j = 0; j < J; ++j) {
        const double *t = tab + j * kSplStride;
        const double a = t[0], b = t[1], c = t[2], ia = t[3], ic = t[4];
        const double eR = exp(-c * s);
        const double dl = (eL - eC) * ia, dr = (eC - eR) * ic;
        double bj = (dr - dl) * is2;
        if (as < t[9]) bj = fma(fma(fma(t[8], s, t[7]), s, t[6]), s, t[5]);
        double dj = 2.0 * (dl - dr) * is3 + ((a * eL - b * eC) * ia - (b * eC - c * eR) * ic) * is2;
        if (as < t[14]) dj = fma(fma(fma(t[13], s, t[12]), s, t[11]), s, t[10]);
        r.BL = fma(Ie[j], bj, r.BL);
        r.sBL = fma(Ie[j], dj, r.sBL);
        eL = eC;
        eC = eR;
    }
    return r;
}

// basis values only, b_j(s) for j < J, into out[]
__device__ __forceinline__ void b1_basis(double s, const double *tab, int J, double *out)
{
    const double is2 = 1.0 / (s * s), as = fabs(s);
    double eL = exp(-tab[0] * s), eC = exp(-tab[1] * s);
#pragma unroll
    for (int j = 0; j < kMaxJ; ++j) {
        if (j < J) {
            const double *t = tab + j * kSplStride;
            const double eR = exp(-t[2] * s);
            double bj = ((eC - eR) * t[4] - (eL - eC) * t[3]) * is2;
            if (as < t[9]) bj = fma(fma(fma(t[8], s, t[7]), s, t[6]), s, t[5]);
            out[j] = bj;
            eL = eC;
            eC = eR;
        }
    }
}

// Poisson term f_i = BL - m - m log(BL / m), with m log(.) = 0 for m = 0
// (bhc/poissLAlpha.m:10-11).
__device__ __forceinline__ double poisson_term(double BL, double m)
{
    return BL - m - (m > 0.0 ? m * log(BL / m) : 0.0);
}

// Noise models of the likelihood, per ray in terms of BL (the modelled
// intensity) and m (the measured one):
//   Poisson  (bhc/poissLAlpha.m, poissLI.m): f = BL - m - m log(BL/m),
//            r = df/dBL = 1 - m/BL,  q = d2f/dBL2 = m / BL^2;
//   Gaussian (bhc/gaussLAlpha.m, gaussLI.m): Err = log(BL/m), f = Err^2 / 2,
//            r = Err / BL,           q = (1 - Err) / BL^2.
// Then the density gradient weight is r dBL/ds and the density Hessian weight
// q (dBL/ds)^2 + r d2BL/ds2 (the `weight` of each file's hessian closure).
enum { kNoisePoisson = 0, kNoiseGaussian = 1 };

struct RayTerms {
    double f, r;
};

__device__ __forceinline__ RayTerms ray_terms(int noise, double BL, double m)
{
    if (noise == kNoiseGaussian) {
        const double e = log(BL / m);
        return {0.5 * e * e, e / BL};
    }
    return {poisson_term(BL, m), 1.0 - m / BL};
}

__device__ __forceinline__ double ray_curvature(int noise, double BL, double m)
{
    if (noise == kNoiseGaussian) return (1.0 - log(BL / m)) / (BL * BL);
    return m / (BL * BL);
}

// The curvature the spectrum step's Newton model uses: exact for the Poisson
// model (never negative), Gauss-Newton 1 / BL^2 for the Gaussian one, whose
// exact (1 - Err) / BL^2 turns negative where the model is far from the data
// and then stalls a bound-constrained Newton method.
__device__ __forceinline__ double ray_curvature_model(int noise, double BL, double m)
{
    if (noise == kNoiseGaussian) return 1.0 / (BL * BL);
    return m / (BL * BL);
}

// Second derivatives: per basis function the Taylor coefficients DD[4] and
// the threshold below which they replace the closed form (bhc/Spline.m:
// 186-197), kSpl2Stride doubles each.
constexpr int kSpl2Stride = 5;

struct SplineEval2 {
    double BL, sBL, ssBL;
};

// BL, dBL/ds and d2BL/ds2; tab2: J * kSpl2Stride doubles
__device__ __forceinline__ SplineEval2 b1_eval2(double s, const double *tab, const double *tab2,
                                                const double *Ie, int J)
{
    const double s2 = s * s, is2 = 1.0 / s2, is3 = is2 / s, is4 = is2 * is2, as = fabs(s);
    double eL = exp(-tab[0] * s), eC = exp(-tab[1] * s);
    SplineEval2 r = {0.0, 0.0, 0.0};
    for (int j = 0; j < J; ++j) {
        const double *t = tab + j * kSplStride;
        const double *u = tab2 + j * kSpl2Stride;
        const double a = t[0], b = t[1], c = t[2], ia = t[3], ic = t[4];
        const double eR = exp(-c * s);
        const double dl = (eL - eC) * ia, dr = (eC - eR) * ic;
        double bj = (dr - dl) * is2;
        if (as < t[9]) bj = fma(fma(fma(t[8], s, t[7]), s, t[6]), s, t[5]);
        double dj = 2.0 * (dl - dr) * is3 + ((a * eL - b * eC) * ia - (b * eC - c * eR) * ic) * is2;
        if (as < t[14]) dj = fma(fma(fma(t[13], s, t[12]), s, t[11]), s, t[10]);
        const double nl = 6.0 * (eL - eC) + s2 * (a * a * eL - b * b * eC) + s * (4.0 * a * eL - 4.0 * b * eC);
        const double nr = 6.0 * (eC - eR) + s2 * (b * b * eC - c * c * eR) + s * (4.0 * b * eC - 4.0 * c * eR);
        double ddj = (nr * ic - nl * ia) * is4;
        if (as < u[4]) ddj = fma(fma(fma(u[3], s, u[2]), s, u[1]), s, u[0]);
        r.BL = fma(Ie[j], bj, r.BL);
        r.sBL = fma(Ie[j], dj, r.sBL);
        r.ssBL = fma(Ie[j], ddj, r.ssBL);
        eL = eC;
        eC = eR;
    }
    return r;
}

}  // namespace ctprj

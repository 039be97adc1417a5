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

}  // namespace ctprj

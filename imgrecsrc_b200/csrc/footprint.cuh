// footprint.cuh -- the pixel-footprint weight, branch-free, for sm_100a.
//
// Same quantity as getWeight() of the reference (prj/utils.h:12-91): the area
// of overlap between a beam of width bw centred on the ray and the projection
// of a unit pixel whose centre lies at signed distance `dist` from the ray.
// For a ray with direction (c, s) the projection is a symmetric trapezoid of
// height 1/max(|c|,|s|) with feet at +-(|c|+|s|)/2 and shoulders at
// +-||c|-|s||/2.  The reference walks a 4x4 tree of cases; here the overlap is
// the difference of the trapezoid's cumulative area at the two beam edges, each
// a sum of three clamped ramps, so a warp never diverges on it.
#pragma once

namespace ctprj {

struct Footprint {
    float h;     // plateau height 1/max(|c|,|s|)
    float b1;    // shoulder half-width ||c|-|s||/2
    float b2;    // foot half-width (|c|+|s|)/2
    float w;     // ramp width b2 - b1
    float iw2;   // 1 / (2 w), 0 for an axis-aligned ray (no ramps)
};

__host__ __device__ __forceinline__ Footprint make_footprint(float c, float s)
{
    c = fabsf(c);
    s = fabsf(s);
    const float hi = fmaxf(c, s), lo = fminf(c, s);
    Footprint f;
    f.h = 1.0f / hi;
    f.b2 = 0.5f * (hi + lo);
    f.b1 = 0.5f * (hi - lo);
    f.w = f.b2 - f.b1;
    f.iw2 = f.w > 0.0f ? 0.5f / f.w : 0.0f;
    return f;
}

// Area of the unit-plateau trapezoid from -inf up to u.
__device__ __forceinline__ float trap_cdf(float u, const Footprint &f)
{
    const float p = fminf(fmaxf(u + f.b2, 0.0f), f.w);          // rising ramp
    const float q = fminf(fmaxf(u + f.b1, 0.0f), 2.0f * f.b1);  // plateau
    const float r = fminf(fmaxf(u - f.b1, 0.0f), f.w);          // falling ramp
    return fmaf(fmaf(p, p, -r * r), f.iw2, q + r);
}

__device__ __forceinline__ float footprint_weight(float dist, float bw, const Footprint &f)
{
    const float hb = 0.5f * bw;
    return f.h * (trap_cdf(hb - dist, f) - trap_cdf(-hb - dist, f));
}

// The same weight with every clamp done by the FMA pipe's saturation to [0, 1]
// instead of min/max on the ALU pipe.  With P = sat((u + b2)/w),
// R = sat((u - b1)/w) and Q = sat((u + b1)/(2 b1)) the cumulative area is
//   G(u) = w/2 (P^2 - R^2) + 2 b1 Q + w R,
// and the coefficients below fold in the plateau height.  A ramp width or
// shoulder width of zero gets a huge finite reciprocal whose saturated terms
// are multiplied by that zero width, so axis-aligned and diagonal rays need no
// branch.  The rounding of (u + b2)/w is bounded by b2 ulp(1) / w and is scaled
// back by w, so the absolute error stays below ~1e-7 for any ramp width.
struct FootprintSat {
    float hw;    // h w / 2
    float tb;    // h 2 b1
    float hwr;   // h w
    float iw;    // 1 / w
    float c1;    // b2 / w
    float c2;    // -b1 / w
    float i2b;   // 1 / (2 b1)
};

__host__ __device__ __forceinline__ FootprintSat make_footprint_sat(float c, float s)
{
    const Footprint f = make_footprint(c, s);
    FootprintSat q;
    const float w = f.w > 1e-30f ? f.w : 1e-30f;
    const float tb = 2.0f * f.b1 > 1e-30f ? 2.0f * f.b1 : 1e-30f;
    q.iw = 1.0f / w;
    q.c1 = f.b2 * q.iw;
    q.c2 = -f.b1 * q.iw;
    q.i2b = 1.0f / tb;
    q.hw = f.h * 0.5f * f.w;
    q.tb = f.h * 2.0f * f.b1;
    q.hwr = f.h * f.w;
    return q;
}

__device__ __forceinline__ float trap_cdf_sat(float u, const FootprintSat &q)
{
    const float P = __saturatef(fmaf(u, q.iw, q.c1));
    const float R = __saturatef(fmaf(u, q.iw, q.c2));
    const float Q = __saturatef(fmaf(u, q.i2b, 0.5f));
    return fmaf(q.hw, fmaf(P, P, -R * R), fmaf(q.tb, Q, q.hwr * R));
}

// footprint weight for a beam of half-width hb
__device__ __forceinline__ float footprint_weight_sat(float dist, float hb, const FootprintSat &q)
{
    return trap_cdf_sat(hb - dist, q) - trap_cdf_sat(-hb - dist, q);
}

}  // namespace ctprj

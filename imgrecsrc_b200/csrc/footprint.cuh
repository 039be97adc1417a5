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

}  // namespace ctprj

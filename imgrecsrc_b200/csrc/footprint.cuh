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

// The beam edges' offsets are formed with __fsub_rn: callers pass products as
// dist or the beam width, and a fused multiply-subtract would round them
// differently in different kernels (the batched and per-plan launches must
// give the same bits).
__device__ __forceinline__ float footprint_weight(float dist, float bw, const Footprint &f)
{
    const float hb = 0.5f * bw;
    return f.h * (trap_cdf(__fsub_rn(hb, dist), f) - trap_cdf(__fsub_rn(-hb, dist), f));
}

// The same weight without branches or min/max, every clamp done by the
// arithmetic pipes' saturation to [0, 1].  In units of the ramp width w, with
// v = u / w, the cumulative area of the trapezoid (plateau height h) is
//   G(u) = h w/2 (P^2 - R'^2) + h 2 b1 Q + h w/2,
//   P = sat(b2/w + v),  R' = sat(b2/w - v),  Q = sat(1/2 + v w/(2 b1))
// (P: the rising ramp, R' = 1 - the falling ramp, Q: the plateau), and the
// constant cancels in the difference of the two beam edges.  With
// hi = max(|c|,|s|) and lo = min(|c|,|s|): h = 1/hi, w = lo, 2 b1 = hi - lo, so
// the plateau's factor h 2 b1 = 1 - lo/hi = 1 - 2 (h w/2) and the difference
// is hw (dX - 2 dQ) + dQ with hw = h w/2: a footprint is three numbers (hw,
// b2/w, w/(2 b1)) besides the scale 1/w.  Callers pass the distance and the
// half beam width already multiplied by 1/w (folded into their per-ray
// coefficients), so a weight costs 14 arithmetic instructions.
// A ramp width or shoulder width of zero (axis-aligned or diagonal rays) gets
// a tiny floor: the huge ratios saturate and are multiplied by the zero width,
// so no branch is needed.  The rounding of b2/w +- v is bounded by
// b2 ulp(1) / w and is scaled back by h w/2: the absolute error stays below
// ~1e-7 for any ramp width.
struct FootprintV {
    float hw;    // h w / 2 (the plateau's factor h 2 b1 is 1 - 2 hw)
    float c1;    // b2 / w
    float rho;   // w / (2 b1)
    float iw;    // 1 / w: the caller's scale of distances and beam widths
};

__host__ __device__ __forceinline__ FootprintV make_footprint_v(float c, float s)
{
    const Footprint f = make_footprint(c, s);
    FootprintV q;
    const float w = f.w > 1e-30f ? f.w : 1e-30f;
    const float tb = 2.0f * f.b1 > 1e-30f ? 2.0f * f.b1 : 1e-30f;
    q.iw = 1.0f / w;
    q.c1 = f.b2 * q.iw;
    q.rho = w / tb;
    q.hw = f.h * 0.5f * f.w;
    return q;
}

// weight for distance D = dist / w and half beam width H = hb / w (the edge
// offsets unfused, as in footprint_weight)
__device__ __forceinline__ float footprint_weight_v(float D, float H, const FootprintV &q)
{
    const float v1 = __fsub_rn(H, D), v2 = __fsub_rn(-H, D);
    const float P1 = __saturatef(q.c1 + v1), R1 = __saturatef(q.c1 - v1);
    const float P2 = __saturatef(q.c1 + v2), R2 = __saturatef(q.c1 - v2);
    const float Q1 = __saturatef(fmaf(v1, q.rho, 0.5f)), Q2 = __saturatef(fmaf(v2, q.rho, 0.5f));
    const float X1 = fmaf(P1, P1, -R1 * R1), X2 = fmaf(P2, P2, -R2 * R2);
    const float dQ = Q1 - Q2;
    return fmaf(q.hw, fmaf(-2.0f, dQ, X1 - X2), dQ);
}

}  // namespace ctprj

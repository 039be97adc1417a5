// projector.cu -- forward projection and backprojection kernels for sm_100a.
//
// Both passes exploit the eight-fold symmetry of the square pixel grid under
// rotations by 90 degrees and reflections, exactly as the reference does
// (prj/cpuPrj.c:46-616): one footprint weight, computed for a base view, serves
// the eight mirrored (view, detector, pixel) triples.  That keeps the effective
// view angles of every output identical to the reference's (they are the
// base view's float-formed angle carried through exact symmetries) and divides
// the arithmetic per ray-pixel update by eight.
//
//  forward   one thread per base ray (view b <= prjFull/8, detector k), marching
//            down the image rows (ray-driven, prj/cpuPrj.c:319-616).  The eight
//            mirrored pixels of a pixel come from the plan's quad image (two
//            float4 per pixel, built at the start of each call), so that every
//            gather is a 16-byte load coalesced along x.
//  backward  one thread per octant pixel 0 <= y <= x (pixel-driven,
//            prj/cpuPrj.c:46-317), looping over the base views and the
//            detectors under the pixel's shadow; each thread owns its eight
//            output pixels, so no atomics are needed.
//
// Precision: the weights are FP32 but each distance from a ray is evaluated in
// FP64 before rounding (x cos R + y sin R - offset cancels to O(1) from terms
// of O(n)); that keeps the projections within 1e-7..1e-6 of the FP64 oracle,
// where the reference's own FP32 build is 1.5e-5 off on signed inputs.
// The footprint itself is branch-free (footprint.cuh).
#include <climits>
#include <cstdio>
#include <type_traits>

#include "ctprj_internal.h"
#include "footprint.cuh"
#include "bhc_spline.cuh"

namespace ctprj {

// a forward block is kFwdViews adjacent base views x 32 adjacent rays, one view
// per warp: the warps march over nearly the same image lines at the same time,
// so the rows they gather are shared in L1.  CTPRJ_FWD_VIEWS and
// CTPRJ_FWD_MINBLOCKS (resident blocks asked of the register allocator) are
// build-time launch-shape choices, as is CTPRJ_BWD_MINBLOCKS for the staged
// backprojection.
#ifndef CTPRJ_FWD_VIEWS
#define CTPRJ_FWD_VIEWS 4
#endif
#ifndef CTPRJ_FWD_MINBLOCKS
#define CTPRJ_FWD_MINBLOCKS 5
#endif
#ifndef CTPRJ_BWD_MINBLOCKS
#define CTPRJ_BWD_MINBLOCKS 4
#endif
// CTPRJ_BWD_DERIVE = 1: the staged fan backprojection keeps one coefficient
// plane per detector and derives the footprint's hw and w / (2 b1) from its
// b2 / w (two reciprocals) instead of reading them from a second plane
#ifndef CTPRJ_BWD_DERIVE
#define CTPRJ_BWD_DERIVE 0
#endif
constexpr bool kBwdDerive = CTPRJ_BWD_DERIVE != 0;
// CTPRJ_BWD_ASYNC = 1: the staged backprojection copies its mirrored sinogram
// samples into shared memory by 4-byte cp.async (no register round trip; the
// lane computes the ray coefficients while they are in flight)
#ifndef CTPRJ_BWD_ASYNC
#define CTPRJ_BWD_ASYNC 0
#endif
constexpr int kFwdViews = CTPRJ_FWD_VIEWS;
constexpr int kFwdThreads = 32 * kFwdViews;
constexpr int kBwdTile = 16;   // 16 x 16 octant pixels per block

// --------------------------------------------------------------- quad image

// The forward pass reads, for each pixel (x, y) a ray crosses, the eight images
// of (x, y) under the symmetries of the square.  The quad image holds them as
// two float4 per pixel: Q[yy][c] = {I(x, yy), I(x, -yy), I(yy, x), I(-yy, x)}
// for rows yy = 0..half and columns c = x + half, x = -half..half, where
// I(a, b) = img[(b + n/2) n + a + n/2]; (x, y) and (-x, y) give all eight.
// One 32 x 32 tile of Q: the I(yy, x) and I(-yy, x) components are image
// columns, staged through shared memory so that every global read is along a
// row.
__device__ __forceinline__ void quad_tile(const float *__restrict__ img, float4 *__restrict__ Q, int n,
                                          int tile, float (&tz)[32][33], float (&tw)[32][33])
{
    const int half = (n - 1) / 2, h2 = n / 2, QW = 2 * half + 1;
    const int tcols = (QW + 31) / 32;
    const int c0 = (tile % tcols) * 32, y0 = (tile / tcols) * 32;
    __syncthreads();
    // tz[i][j] = I(y0 + j, x_i), tw[i][j] = I(-(y0 + j), x_i) with x_i = c0 + i - half
    for (int i = threadIdx.y; i < 32; i += 8) {
        const int c = c0 + i, yy = y0 + threadIdx.x;
        if (c < QW && yy <= half) {
            const float *row = img + (size_t)(c - half + h2) * n + h2;
            tz[i][threadIdx.x] = row[yy];
            tw[i][threadIdx.x] = row[-yy];
        }
    }
    __syncthreads();
    for (int j = threadIdx.y; j < 32; j += 8) {
        const int c = c0 + threadIdx.x, yy = y0 + j;
        if (c < QW && yy <= half) {
            const int x = c - half;
            const float a = img[(size_t)(yy + h2) * n + x + h2];
            const float b = img[(size_t)(h2 - yy) * n + x + h2];
            Q[(size_t)yy * QW + c] = make_float4(a, b, tz[threadIdx.x][j], tw[threadIdx.x][j]);
        }
    }
}

__global__ void __launch_bounds__(256) k_quad(const float *__restrict__ img, float4 *__restrict__ Q, int n)
{
    __shared__ float tz[32][33], tw[32][33];
    quad_tile(img, Q, n, blockIdx.x, tz, tw);
}

int launch_quad(const float *img, float4 *Q, int n, cudaStream_t s)
{
    k_quad<<<quad_tiles(n), dim3(32, 8), 0, s>>>(img, Q, n);
    return cuda_error(cudaGetLastError(), "quad image launch");
}

// ----------------------------------------------------------------- forward

// Polychromatic epilogue of one sinogram entry (bhc/poissLAlpha.m:2-13 and
// bhc/gaussLAlpha.m:2-16 per ray): s = Ts * proj, BL(s) and dBL/ds over the
// spectrum (FP64), and the likelihood term; keeps s, r = df/dBL and
// r dBL/ds when asked.
__device__ __forceinline__ double bhc_entry(const BhcArgs &a, const double *tab,
                                            const double *Ie, float proj, size_t idx)
{
    const double s = a.Ts * (double)proj;
    const SplineEval e = b1_eval(s, tab, Ie, a.J);
    const double m = (double)__ldg(a.imea + idx);
    const RayTerms t = ray_terms(a.noise, e.BL, m);
    if (a.w_out) {
        a.w_out[idx] = (float)(t.r * e.sBL);
        a.s_out[idx] = (float)s;
        a.r_out[idx] = t.r;
    }
    return t.f;
}

__device__ __forceinline__ double block_sum(double v, double *red)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) red[warp] = v;
    __syncthreads();
    double t = 0.0;
    if (threadIdx.x == 0)
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += red[w];
    return t;
}

// Constants of forward ray (base view b, detector k): its direction
// (cos R, sin R) and offset from the isocentre, the pixel range of each row
// as xl(y) = Al - y Sl, xr(y) = Ar - y Sr -- the intersections of the two beam
// edges with the row's band (prj/cpuPrj.c:365-369 parallel, :514-536 fan) --
// the fan's magnified beam width bwc + (x sinT - y cosT) kbw, and the
// footprint with its per-pixel steps in ramp units.
struct FwdRay {
    double cR, sR, off;
    float Al, Sl, Ar, Sr;
    float cT, sT, bwc, kbw;
    FootprintV fp;
    float cRw, dhbw;
};

template <bool FAN>
__device__ __forceinline__ FwdRay fwd_ray(const FwdParams &p, int b, int k)
{
    const Geo &g = p.g;
    const double cT = p.view[b].c, sT = p.view[b].s;
    const DetEntry de = p.det[k];
    const double hbw = 0.5 * g.beamWidth;
    const double tl = de.t - hbw, tr = de.t + hbw;
    // every product-sum is an explicit fma, so that no kernel this is inlined
    // into contracts it differently: the batched and per-plan launches must
    // give the same bits
    double cR, sR, off, Al, Sl, Ar, Sr;
    float bwc = g.beamWidthF, kbw = 0.0f;
    if (FAN) {
        const double d = g.d;
        cR = fma(de.cB, cT, -(de.sB * sT));
        sR = fma(de.sB, cT, de.cB * sT);
        off = de.t * de.cB;   // d t / bq
        const double qxl = fma(tl, cT, d * sT), qyl = fma(-tl, sT, d * cT);
        const double qxr = fma(tr, cT, d * sT), qyr = fma(-tr, sT, d * cT);
        Al = fma(qxl > 0 ? -0.5 : 0.5, qxl, d * tl) / qyl;
        Sl = qxl / qyl;
        Ar = fma(qxr > 0 ? 0.5 : -0.5, qxr, d * tr) / qyr;
        Sr = qxr / qyr;
        const double bwcd = g.beamWidth * de.cB;
        bwc = (float)bwcd;
        kbw = (float)(bwcd / d);
    } else {
        cR = cT;
        sR = sT;
        off = de.t;
        Al = fma(-0.5, sT, tl) / cT;
        Sl = sT / cT;
        Ar = fma(0.5, sT, tr) / cT;
        Sr = Sl;
    }
    FwdRay r;
    r.cR = cR;
    r.sR = sR;
    r.off = off;
    r.Al = (float)Al;
    r.Sl = (float)Sl;
    r.Ar = (float)Ar;
    r.Sr = (float)Sr;
    r.cT = (float)cT;
    r.sT = (float)sT;
    r.bwc = bwc;
    r.kbw = kbw;
    const float dhb = FAN ? 0.5f * r.sT * kbw : 0.0f;   // half beam width step per pixel
    r.fp = make_footprint_v((float)cR, (float)sR);
    r.cRw = (float)cR * r.fp.iw;
    r.dhbw = dhb * r.fp.iw;
    return r;
}

// The rays of one forward block: V adjacent base views (one per warp) x 32
// adjacent detectors; block (bx, by) of the per-plan grid.  Returns this
// thread's Poisson terms in polychromatic mode.
// Build-time variant CTPRJ_FWD_WARP_VIEWS = G > 1: a warp takes G adjacent
// views x 32 / G detectors instead (measured slower: G unaligned pixel runs per
// gather touch more 128-byte lines than one contiguous run of 32 rays).
#ifndef CTPRJ_FWD_WARP_VIEWS
#define CTPRJ_FWD_WARP_VIEWS 1
#endif
template <bool FAN, int MODE, int V>
__device__ __forceinline__ double forward_rays(const FwdParams &p, int bx, int by,
                                               const float4 *__restrict__ quad,
                                               float *__restrict__ sino,
                                               unsigned long long *__restrict__ counter,
                                               const double *tab, const double *Ie)
{
    const Geo &g = p.g;
    constexpr int G = V < CTPRJ_FWD_WARP_VIEWS ? V : CTPRJ_FWD_WARP_VIEWS, D = 32 / G;
    const int warp = (int)(threadIdx.x >> 5), lane = (int)(threadIdx.x & 31);
    const int b = bx * V + (warp / G) * G + lane / D;
    const int r = by * 32 + (warp % G) * D + lane % D;
    double fsum = 0.0;            // polychromatic mode: this thread's Poisson terms
    // detector 0 of an even-width sinogram: no ray, zero projection
    if (MODE != kModeCount && p.zero_col0 && bx == 0 && by == 0)
        for (int v = threadIdx.x; v < g.np; v += blockDim.x) {
            if constexpr (MODE == kModeBhc) {
                fsum += bhc_entry(p.bhc, tab, Ie, 0.0f, (size_t)v * g.W);
                if (p.bhc.proj_out) p.bhc.proj_out[(size_t)v * g.W] = 0.0f;
            } else {
                sino[(size_t)v * g.W] = 0.0f;
            }
        }

    // The window a warp marches with (below) is the widest any of its rays
    // needs: xr - xl is affine in y, so a ray's widest run is at the first or
    // the last row.  Every lane of the (full) warp takes part in the maximum,
    // lanes without a ray with 0, so the choice depends on the warp's rays
    // alone and a batched launch makes the same one (the variant with G views
    // per warp takes it per view, over that view's lanes).
    const bool live = b < p.nb && r < p.nk;
    const int k = p.k0 + r;
    FwdRay ray = {};
    int wcode = 0;   // 3 / 4: window of 3 / 4 pixels; 5: bounded range loop
    if (live) {
        ray = fwd_ray<FAN>(p, b, k);
        wcode = 5;
        if (MODE != kModeCount && g.half >= 3) {
            const float wa = ray.Ar - ray.Al, ws = ray.Sr - ray.Sl, hf = (float)g.half;
            const float wmax = fmaxf(fabsf(fmaf(-hf, ws, wa)), fabsf(fmaf(hf, ws, wa)));
            wcode = wmax < 1.95f ? 3 : (wmax < 2.95f ? 4 : 5);
        }
    }
    if (G == 1) {
        wcode = __reduce_max_sync(0xffffffffu, wcode);
    } else {
#pragma unroll
        for (int o = 1; o < D; o <<= 1) wcode = max(wcode, __shfl_xor_sync(0xffffffffu, wcode, o));
    }
    if (live) {
        const double cR = ray.cR, sR = ray.sR, off = ray.off;
        const float Alf = ray.Al, Slf = ray.Sl, Arf = ray.Ar, Srf = ray.Sr;
        const float cTf = ray.cT, sTf = ray.sT, bwc = ray.bwc, kbw = ray.kbw;
        const FootprintV fp = ray.fp;
        const float cRw = ray.cRw, dhbw = ray.dhbw;

        const int half = g.half;
        float S[8];
#pragma unroll
        for (int j = 0; j < 8; ++j) S[j] = 0.0f;
        unsigned long long nz = 0;

        // The march down the rows.  Row y reads the quad row |y|:
        // q[x] = {I(x, |y|), I(x, -|y|), I(|y|, x), I(-|y|, x)}, so that for
        // y >= 0 the eight sums take, per pixel x,
        //   S0 += I(x, y), S6 += I(-x, y), S4 += I(x, -y), S2 += I(-x, -y),
        //   S5 += I(y, x), S3 += I(y, -x), S1 += I(-y, x), S7 += I(-y, -x)
        // from q[x] and q[-x]; for y < 0 the pairs of components swap.
        const int QW = 2 * half + 1;
        auto march_row = [&](const int y, const float4 *__restrict__ q, auto neg) {
            constexpr bool NEG = decltype(neg)::value;
            const float yf = (float)y;
            const float xl = fmaf(-yf, Slf, Alf), xr = fmaf(-yf, Srf, Arf);
            // nearest pixel to each edge; exact half-way ties (where the
            // reference rounds away from zero) only decide pixels whose
            // footprint just touches the beam edge, with weight zero; the
            // conversion saturates, so far-out edges clamp
            const int x0 = max(__float2int_rn(xl), -half);
            const int x1 = min(__float2int_rn(xr), half);
            if (x0 > x1) return;
            // distance of pixel (x0, y) from the ray, in FP64 then rounded;
            // distances and half beam widths in units of the footprint's ramp
            const float r0 = (float)fma((double)x0, cR, fma((double)y, sR, -off)) * fp.iw;
            const float hb0 = (FAN ? 0.5f * fmaf(fmaf((float)x0, sTf, -yf * cTf), kbw, bwc)
                                   : 0.5f * g.beamWidthF) * fp.iw;
            auto accumulate = [&](const float w, const float4 pp, const float4 pm) {
                const float ap = NEG ? pp.y : pp.x, am = NEG ? pm.y : pm.x;   // I(+-x, y)
                const float bp = NEG ? pp.x : pp.y, bm = NEG ? pm.x : pm.y;   // I(+-x, -y)
                const float cp = NEG ? pp.w : pp.z, cm = NEG ? pm.w : pm.z;   // I(y, +-x)
                const float dp = NEG ? pp.z : pp.w, dm = NEG ? pm.z : pm.w;   // I(-y, +-x)
                S[0] = fmaf(w, ap, S[0]);
                S[6] = fmaf(w, am, S[6]);
                S[4] = fmaf(w, bp, S[4]);
                S[2] = fmaf(w, bm, S[2]);
                S[5] = fmaf(w, cp, S[5]);
                S[3] = fmaf(w, cm, S[3]);
                S[1] = fmaf(w, dp, S[1]);
                S[7] = fmaf(w, dm, S[7]);
            };
            // Pixel x0 + j sits at D = fma(j, cRw, r0) (j even) or that of
            // j - 1 plus cRw (j odd), and likewise for H.  At unit beam width
            // a ray crosses one to three pixels of a row below 37 degrees of
            // obliquity and two to four above, so one straight-line step takes
            // the first three pixels, their gathers issued together and each
            // predicated on the pixel being in the run (a lane past its run
            // sends no request), and single steps the rest; per sum the order
            // of the terms is x0, x0 + 1, ...
            auto coef = [&](const int j, float &D, float &H) {
                const float je = (float)(j & ~1);
                D = fmaf(je, cRw, r0);
                H = FAN ? fmaf(je, dhbw, hb0) : hb0;
                if (j & 1) {
                    D += cRw;
                    if (FAN) H += dhbw;
                }
            };
            {
                const bool p1 = x0 < x1, p2 = x0 + 1 < x1;
                float D0, H0, D1, H1, D2, H2;
                coef(0, D0, H0);
                coef(1, D1, H1);
                coef(2, D2, H2);
                if (MODE == kModeCount) {
                    nz += (footprint_weight_v(D0, H0, fp) != 0.0f);
                    if (p1) nz += (footprint_weight_v(D1, H1, fp) != 0.0f);
                    if (p2) nz += (footprint_weight_v(D2, H2, fp) != 0.0f);
                } else {
                    const float4 pp0 = __ldg(q + x0), pm0 = __ldg(q - x0);
                    float4 pp1 = {}, pm1 = {}, pp2 = {}, pm2 = {};
                    if (p1) {
                        pp1 = __ldg(q + x0 + 1);
                        pm1 = __ldg(q - x0 - 1);
                    }
                    if (p2) {
                        pp2 = __ldg(q + x0 + 2);
                        pm2 = __ldg(q - x0 - 2);
                    }
                    accumulate(footprint_weight_v(D0, H0, fp), pp0, pm0);
                    if (p1) accumulate(footprint_weight_v(D1, H1, fp), pp1, pm1);
                    if (p2) accumulate(footprint_weight_v(D2, H2, fp), pp2, pm2);
                }
            }
            for (int x = x0 + 3; x <= x1; ++x) {
                float D, H;
                coef(x - x0, D, H);
                if (MODE == kModeCount) {
                    nz += (footprint_weight_v(D, H, fp) != 0.0f);
                    continue;
                }
                accumulate(footprint_weight_v(D, H, fp), __ldg(q + x), __ldg(q - x));
            }
        };
        // The fixed-window march (plain and polychromatic modes).  Where a
        // ray's run across a row is always narrower than 1.95 (2.95) pixels,
        // the pixels of the run lie within the 3 (4) centred on the ray's
        // crossing xc = (xl + xr) / 2: they are summed straight, without the
        // run's bounds.  A pixel of the window outside the run lies beyond
        // the beam and adds a weight of exactly zero (for fan beams: below
        // 1e-7 within ~1e-4 pixel of a run edge, where the footprint and the
        // beam edges differ).  The window is chosen per warp (the widest any
        // of its rays needs), so the warp stays converged.
        const float Acf = 0.5f * (Alf + Arf), Scf = 0.5f * (Slf + Srf);
        auto march_win = [&](const int y, const float4 *__restrict__ q, auto neg, auto wn) {
            constexpr bool NEG = decltype(neg)::value;
            constexpr int WN = decltype(wn)::value;
            const float yf = (float)y;
            const float xc = fmaf(-yf, Scf, Acf);
            // rows whose run misses the image (the run lies within xc +- 1.5)
            if (xc < -(float)half - 2.0f || xc > (float)half + 2.0f) return;
            int xs = (WN == 3 ? __float2int_rn(xc) : __float2int_rd(xc)) - 1;
            xs = min(max(xs, -half), half - (WN - 1));
#if CTPRJ_FWD_PREFETCH
            // Build-time variant: ask L1 for the quad lines this ray will read
            // CTPRJ_FWD_PREFETCH rows further on (at this row's x: the run
            // moves less than a pixel per row), where that row is in the image
            {
                constexpr int PD = CTPRJ_FWD_PREFETCH;
                if (NEG ? PD - y <= half : y - PD >= 0) {
                    const float4 *qa = NEG ? q + PD * QW : q - PD * QW;
                    asm volatile("prefetch.L1 [%0];" ::"l"(qa + xs));
                    asm volatile("prefetch.L1 [%0];" ::"l"(qa - xs));
                }
            }
#endif
            const float r0 = (float)fma((double)xs, cR, fma((double)y, sR, -off)) * fp.iw;
            const float hb0 = (FAN ? 0.5f * fmaf(fmaf((float)xs, sTf, -yf * cTf), kbw, bwc)
                                   : 0.5f * g.beamWidthF) * fp.iw;
            float4 pp[WN], pm[WN];
#pragma unroll
            for (int j = 0; j < WN; ++j) {
                pp[j] = __ldg(q + xs + j);
                pm[j] = __ldg(q - xs - j);
            }
#pragma unroll
            for (int j = 0; j < WN; ++j) {
                const float D = fmaf((float)j, cRw, r0);
                const float H = FAN ? fmaf((float)j, dhbw, hb0) : hb0;
                const float w = footprint_weight_v(D, H, fp);
                const float ap = NEG ? pp[j].y : pp[j].x, am = NEG ? pm[j].y : pm[j].x;
                const float bp = NEG ? pp[j].x : pp[j].y, bm = NEG ? pm[j].x : pm[j].y;
                const float cp = NEG ? pp[j].w : pp[j].z, cm = NEG ? pm[j].w : pm[j].z;
                const float dp = NEG ? pp[j].z : pp[j].w, dm = NEG ? pm[j].z : pm[j].w;
                S[0] = fmaf(w, ap, S[0]);
                S[6] = fmaf(w, am, S[6]);
                S[4] = fmaf(w, bp, S[4]);
                S[2] = fmaf(w, bm, S[2]);
                S[5] = fmaf(w, cp, S[5]);
                S[3] = fmaf(w, cm, S[3]);
                S[1] = fmaf(w, dp, S[1]);
                S[7] = fmaf(w, dm, S[7]);
            }
        };
#if CTPRJ_FWD_PIPE
        // Build-time variant (CTPRJ_FWD_PIPE=1): the window march software-
        // pipelined two rows deep, the next row's gathers issued before this
        // row's footprints (rows ya, ya - 1, ..., yb; q is row ya's quad row
        // and moves by dq per row).  Same sums as march_win.
        auto march_pipe = [&](const int ya, const int yb, const float4 *q, const int dq, auto neg, auto wn) {
            constexpr bool NEG = decltype(neg)::value;
            constexpr int WN = decltype(wn)::value;
            struct Row {
                float4 pp[WN], pm[WN];
                int xs;
                bool on;
            };
            auto fetch = [&](const int y, const float4 *__restrict__ qq, Row &R) {
                const float xc = fmaf(-(float)y, Scf, Acf);
                R.on = !(xc < -(float)half - 2.0f || xc > (float)half + 2.0f);
                int xs = (WN == 3 ? __float2int_rn(xc) : __float2int_rd(xc)) - 1;
                xs = min(max(xs, -half), half - (WN - 1));
                R.xs = xs;
#pragma unroll
                for (int j = 0; j < WN; ++j) {
                    R.pp[j] = __ldg(qq + xs + j);
                    R.pm[j] = __ldg(qq - xs - j);
                }
            };
            auto sum = [&](const int y, const Row &R) {
                if (!R.on) return;
                const float yf = (float)y;
                const float r0 = (float)fma((double)R.xs, cR, fma((double)y, sR, -off)) * fp.iw;
                const float hb0 = (FAN ? 0.5f * fmaf(fmaf((float)R.xs, sTf, -yf * cTf), kbw, bwc)
                                       : 0.5f * g.beamWidthF) * fp.iw;
#pragma unroll
                for (int j = 0; j < WN; ++j) {
                    const float D = fmaf((float)j, cRw, r0);
                    const float H = FAN ? fmaf((float)j, dhbw, hb0) : hb0;
                    const float w = footprint_weight_v(D, H, fp);
                    const float4 pp = R.pp[j], pm = R.pm[j];
                    S[0] = fmaf(w, NEG ? pp.y : pp.x, S[0]);
                    S[6] = fmaf(w, NEG ? pm.y : pm.x, S[6]);
                    S[4] = fmaf(w, NEG ? pp.x : pp.y, S[4]);
                    S[2] = fmaf(w, NEG ? pm.x : pm.y, S[2]);
                    S[5] = fmaf(w, NEG ? pp.w : pp.z, S[5]);
                    S[3] = fmaf(w, NEG ? pm.w : pm.z, S[3]);
                    S[1] = fmaf(w, NEG ? pp.z : pp.w, S[1]);
                    S[7] = fmaf(w, NEG ? pm.z : pm.w, S[7]);
                }
            };
            Row A, B;
            fetch(ya, q, A);
            int y = ya;
            for (; y - 1 >= yb; y -= 2, q += 2 * dq) {
                fetch(y - 1, q + dq, B);
                sum(y, A);
                if (y - 2 >= yb) fetch(y - 2, q + 2 * dq, A);
                sum(y - 1, B);
            }
            if (y == yb) sum(y, A);
        };
        if (wcode == 3 || wcode == 4) {
            const float4 *qp = quad + (size_t)half * QW + half, *qn = quad + (size_t)QW + half;
            if (wcode == 3) {
                march_pipe(half, 0, qp, -QW, std::false_type{}, std::integral_constant<int, 3>{});
                march_pipe(-1, -half, qn, QW, std::true_type{}, std::integral_constant<int, 3>{});
            } else {
                march_pipe(half, 0, qp, -QW, std::false_type{}, std::integral_constant<int, 4>{});
                march_pipe(-1, -half, qn, QW, std::true_type{}, std::integral_constant<int, 4>{});
            }
        } else
#endif
        {
            const float4 *q = quad + (size_t)half * QW + half;   // row |y| = half, x = 0
            if (wcode == 3) {
                for (int y = half; y >= 0; --y, q -= QW)
                    march_win(y, q, std::false_type{}, std::integral_constant<int, 3>{});
            } else if (wcode == 4) {
                for (int y = half; y >= 0; --y, q -= QW)
                    march_win(y, q, std::false_type{}, std::integral_constant<int, 4>{});
            } else {
                for (int y = half; y >= 0; --y, q -= QW) march_row(y, q, std::false_type{});
            }
            q = quad + (size_t)QW + half;                          // row |y| = 1
            if (wcode == 3) {
                for (int y = -1; y >= -half; --y, q += QW)
                    march_win(y, q, std::true_type{}, std::integral_constant<int, 3>{});
            } else if (wcode == 4) {
                for (int y = -1; y >= -half; --y, q += QW)
                    march_win(y, q, std::true_type{}, std::integral_constant<int, 4>{});
            } else {
                for (int y = -1; y >= -half; --y, q += QW) march_row(y, q, std::true_type{});
            }
        }

        // Scatter to the eight symmetric views (prj/cpuPrj.c:577-615); parallel
        // beam also writes the point-reflected detector of the same view
        // (prj/cpuPrj.c:403-460), which image j ^ 2 holds.  Where the two
        // coincide (the central detector) the second write is the one kept.
        const int pC = g.pC;
        unsigned long long entries = 0;
        // polychromatic mode: the entries this ray sum feeds, gathered first so
        // that one copy of the FP64 epilogue serves them all
        float eval[16];
        int eidx[16];
        int ne = 0;
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            const int v = p.view[b].out[j];
            if (v < 0) continue;
            const int det = j < 4 ? k : 2 * pC - k;
            const int det2 = 2 * pC - det;
            const size_t row = (size_t)v * g.W;
            if constexpr (MODE == kModeCount) {
                entries += (!FAN && det2 != det) ? 2 : 1;
            } else if constexpr (MODE == kModeBhc) {
                if (FAN) {
                    eval[ne] = S[j] / g.effRate; eidx[ne++] = (int)(row + det);
                } else if (det2 != det) {
                    eval[ne] = S[j] / g.effRate; eidx[ne++] = (int)(row + det);
                    eval[ne] = S[j ^ 2] / g.effRate; eidx[ne++] = (int)(row + det2);
                } else {
                    eval[ne] = S[j ^ 2] / g.effRate; eidx[ne++] = (int)(row + det);
                }
            } else {
                sino[row + det] = S[j] / g.effRate;
                if (!FAN) sino[row + det2] = S[j ^ 2] / g.effRate;
            }
        }
        if constexpr (MODE == kModeBhc) {
#pragma unroll 1
            for (int e = 0; e < ne; ++e) {
                fsum += bhc_entry(p.bhc, tab, Ie, eval[e], (size_t)eidx[e]);
                if (p.bhc.proj_out) p.bhc.proj_out[eidx[e]] = eval[e];
            }
        }
        if (MODE == kModeCount && nz * entries) atomicAdd(counter, nz * entries);
    }
    return fsum;
}

template <bool FAN, int MODE>
__global__ void __launch_bounds__(kFwdThreads, CTPRJ_FWD_MINBLOCKS)
k_forward(const FwdParams p, const float4 *__restrict__ quad, float *__restrict__ sino,
          unsigned long long *__restrict__ counter)
{
    const double *tab = nullptr, *Ie = nullptr;
    if constexpr (MODE == kModeBhc) {
        __shared__ double sm[kMaxJ * (kSplStride + 1)];
        for (int i = threadIdx.x; i < p.bhc.J * kSplStride; i += blockDim.x) sm[i] = p.bhc.tab[i];
        for (int i = threadIdx.x; i < p.bhc.J; i += blockDim.x) sm[kMaxJ * kSplStride + i] = p.bhc.Ie[i];
        __syncthreads();
        tab = sm;
        Ie = sm + kMaxJ * kSplStride;
    }
    int bx = blockIdx.x, by = blockIdx.y;
#if CTPRJ_FWD_REMAP
    // Build-time variant: the block scheduler starts blocks i, i + S, i + 2S, ...
    // (S = SM count) on one SM in its first wave, so hand them consecutive view
    // groups of one ray group: their rays cross nearly the same quad-image
    // lines and could share that SM's L1.  A bijection of the block indices.
    {
        const int S = p.sms, total = gridDim.x * gridDim.y, i = blockIdx.y * gridDim.x + blockIdx.x;
        const int q = total / S, r = total % S, sl = i % S, k = i / S;
        const int item = sl * q + min(sl, r) + k;
        bx = item % gridDim.x;
        by = item / gridDim.x;
    }
#endif
    const double fsum = forward_rays<FAN, MODE, kFwdViews>(p, bx, by, quad, sino, counter, tab, Ie);
    if constexpr (MODE == kModeBhc) {
        __shared__ double red[kFwdThreads / 32];
        const double t = block_sum(fsum, red);
        if (threadIdx.x == 0) p.bhc.part[(size_t)by * gridDim.x + bx] = t;
    }
}

#if CTPRJ_FWD_STAGE
// -------------------------------------------- forward, staged by bulk copies
//
// Build-time variant (CTPRJ_FWD_STAGE=1), measured against k_forward.  The
// block's rays read the quad-image rows of a chunk of kStRows rows from shared
// memory: one thread brings the row segments in with bulk asynchronous copies
// (cp.async.bulk, completion counted on an mbarrier), double-buffered so that
// the copies of chunk c + 1 are in flight while chunk c is summed.  A segment
// is the union of the block's pixel windows over the chunk's rows, on the +x
// side and its mirror; a chunk whose union exceeds kStCols pixels is read from
// global memory instead, and so are warps whose rays need the range loop.
// Plain mode only.  Waits are bounded (%globaltimer, 1 s): past it the block
// records the timeout in g_fwd_stage_timeout, writes NaN to its outputs and
// returns.

#ifndef CTPRJ_FWD_STAGE_ROWS
#define CTPRJ_FWD_STAGE_ROWS 4
#endif
constexpr int kStRows = CTPRJ_FWD_STAGE_ROWS;
constexpr int kStCols = 128;

struct FwdStage {
    float4 buf[2][kStRows][2][kStCols];   // [buffer][row][+x side, -x side][pixel]
    unsigned long long bar[2];
    int lo[2], hi[2];                      // staged pixels [lo, hi] of each buffer; hi < lo: none
    int wlo[kFwdViews], whi[kFwdViews];
};

__device__ int g_fwd_stage_timeout;

__device__ __forceinline__ unsigned long long stage_ns()
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ unsigned smem_u32(const void *ptr)
{
    return (unsigned)__cvta_generic_to_shared(ptr);
}

// true when the phase of parity `ph` of barrier `bar` completed within 1 s
__device__ __forceinline__ bool stage_wait(unsigned long long *bar, unsigned ph)
{
    const unsigned a = smem_u32(bar);
    const unsigned long long t0 = stage_ns();
    for (;;) {
        unsigned done;
        asm volatile("{\n\t.reg .pred p;\n\t"
                     "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                     "selp.u32 %0, 1, 0, p;\n\t}"
                     : "=r"(done) : "r"(a), "r"(ph) : "memory");
        if (done) return true;
        if (stage_ns() - t0 > 1000000000ull) return false;
    }
}

template <bool FAN>
__global__ void __launch_bounds__(kFwdThreads, CTPRJ_FWD_MINBLOCKS)
k_forward_staged(const FwdParams p, const float4 *__restrict__ quad, float *__restrict__ sino)
{
    __shared__ __align__(128) FwdStage st;
    const Geo &g = p.g;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int b = blockIdx.x * kFwdViews + warp;
    const int r = blockIdx.y * 32 + lane;
    const bool live = b < p.nb && r < p.nk;
    if (p.zero_col0 && blockIdx.x == 0 && blockIdx.y == 0)
        for (int v = threadIdx.x; v < g.np; v += blockDim.x) sino[(size_t)v * g.W] = 0.0f;
    const int half = g.half, QW = 2 * half + 1;
    const int k = p.k0 + r;
    FwdRay ray = {};
    int wcode = 0;   // 0: no ray, 3 / 4: window, 5: range loop (global reads)
    if (live) {
        ray = fwd_ray<FAN>(p, b, k);
        const float wa = ray.Ar - ray.Al, ws = ray.Sr - ray.Sl;
        const float wmax = fmaxf(fabsf(fmaf(-(float)half, ws, wa)), fabsf(fmaf((float)half, ws, wa)));
        wcode = half < 3 ? 5 : (wmax < 1.95f ? 3 : (wmax < 2.95f ? 4 : 5));
    }
    wcode = __reduce_max_sync(0xffffffffu, wcode);
    const float Acf = 0.5f * (ray.Al + ray.Ar), Scf = 0.5f * (ray.Sl + ray.Sr);
    // the window start of this lane's ray at row y (window rays only)
    auto wstart = [&](int y) {
        const float xc = fmaf(-(float)y, Scf, Acf);
        const int xs = (wcode == 3 ? __float2int_rn(xc) : __float2int_rd(xc)) - 1;
        return min(max(xs, -half), half - (wcode - 1));
    };
    const int steps = 2 * half + 1;               // rows y = half - m, m = 0 .. 2 half
    const int nchunks = (steps + kStRows - 1) / kStRows;
    // this warp's union of windows over chunk c, then the block's, into buffer c & 1
    auto plan_chunk = [&](int c) {
        int lo = INT_MAX, hi = INT_MIN;
        if (live && (wcode == 3 || wcode == 4)) {
            const int m0 = c * kStRows, m1 = min(m0 + kStRows, steps) - 1;
            const int a0 = wstart(half - m0), a1 = wstart(half - m1);
            lo = min(a0, a1);
            hi = max(a0, a1) + wcode - 1;
        }
        lo = __reduce_min_sync(0xffffffffu, lo);
        hi = __reduce_max_sync(0xffffffffu, hi);
        if (lane == 0) {
            st.wlo[warp] = lo;
            st.whi[warp] = hi;
        }
    };
    auto issue_chunk = [&](int c) {   // thread 0, after a block barrier
        const int bc = c & 1;
        int lo = INT_MAX, hi = INT_MIN;
        for (int w = 0; w < kFwdViews; ++w) {
            lo = min(lo, st.wlo[w]);
            hi = max(hi, st.whi[w]);
        }
        if (hi < lo || hi - lo + 1 > kStCols) {
            st.lo[bc] = 1;
            st.hi[bc] = 0;
            return;
        }
        st.lo[bc] = lo;
        st.hi[bc] = hi;
        const int m0 = c * kStRows, nr = min(kStRows, steps - m0);
        const unsigned bytes = (unsigned)(hi - lo + 1) * 16u;
        const unsigned bar = smem_u32(&st.bar[bc]);
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;"
                     :: "r"(bar), "r"(bytes * 2u * (unsigned)nr) : "memory");
        for (int i = 0; i < nr; ++i) {
            const int y = half - (m0 + i), row = y < 0 ? -y : y;
            const float4 *src = quad + (size_t)row * QW + half;
            asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
                         :: "r"(smem_u32(&st.buf[bc][i][0][0])), "l"(src + lo), "r"(bytes), "r"(bar)
                         : "memory");
            asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
                         :: "r"(smem_u32(&st.buf[bc][i][1][0])), "l"(src - hi), "r"(bytes), "r"(bar)
                         : "memory");
        }
    };

    if (threadIdx.x == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" :: "r"(smem_u32(&st.bar[0])) : "memory");
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" :: "r"(smem_u32(&st.bar[1])) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    plan_chunk(0);
    __syncthreads();
    if (threadIdx.x == 0) issue_chunk(0);

    float S[8];
#pragma unroll
    for (int j = 0; j < 8; ++j) S[j] = 0.0f;
    unsigned ph[2] = {0u, 0u};
    bool failed = false;
    for (int c = 0; c < nchunks; ++c) {
        const int bc = c & 1;
        if (c + 1 < nchunks) plan_chunk(c + 1);
        // chunk c - 1 read; windows of chunk c + 1 visible; a wait that timed
        // out in any thread ends the march of the whole block
        if (__syncthreads_or(failed)) {
            failed = true;
            break;
        }
        if (threadIdx.x == 0 && c + 1 < nchunks) issue_chunk(c + 1);
        const int lo = st.lo[bc], hi = st.hi[bc];
        const bool staged = lo <= hi;
        if (staged) {
            if (!stage_wait(&st.bar[bc], ph[bc])) {
                failed = true;
                continue;
            }
            ph[bc] ^= 1u;
        }
        if (!live) continue;
        const int m0 = c * kStRows, nr = min(kStRows, steps - m0);
        for (int i = 0; i < nr; ++i) {
            const int y = half - (m0 + i), row = y < 0 ? -y : y;
            const bool neg = y < 0;
            const float4 *q = quad + (size_t)row * QW + half;
            const float yf = (float)y;
            if (wcode == 5) {
                // range loop from global memory (prj/cpuPrj.c:365-369, :514-536 ranges)
                const int x0 = max(__float2int_rn(fmaf(-yf, ray.Sl, ray.Al)), -half);
                const int x1 = min(__float2int_rn(fmaf(-yf, ray.Sr, ray.Ar)), half);
                for (int x = x0; x <= x1; ++x) {
                    const float D = (float)fma((double)x, ray.cR, fma((double)y, ray.sR, -ray.off)) * ray.fp.iw;
                    const float H = (FAN ? 0.5f * fmaf(fmaf((float)x, ray.sT, -yf * ray.cT), ray.kbw, ray.bwc)
                                         : 0.5f * g.beamWidthF) * ray.fp.iw;
                    const float w = footprint_weight_v(D, H, ray.fp);
                    const float4 pp = __ldg(q + x), pm = __ldg(q - x);
                    S[0] = fmaf(w, neg ? pp.y : pp.x, S[0]);
                    S[6] = fmaf(w, neg ? pm.y : pm.x, S[6]);
                    S[4] = fmaf(w, neg ? pp.x : pp.y, S[4]);
                    S[2] = fmaf(w, neg ? pm.x : pm.y, S[2]);
                    S[5] = fmaf(w, neg ? pp.w : pp.z, S[5]);
                    S[3] = fmaf(w, neg ? pm.w : pm.z, S[3]);
                    S[1] = fmaf(w, neg ? pp.z : pp.w, S[1]);
                    S[7] = fmaf(w, neg ? pm.z : pm.w, S[7]);
                }
                continue;
            }
            const float xc = fmaf(-yf, Scf, Acf);
            if (xc < -(float)half - 2.0f || xc > (float)half + 2.0f) continue;
            const int xs = wstart(y);
            const float r0 = (float)fma((double)xs, ray.cR, fma((double)y, ray.sR, -ray.off)) * ray.fp.iw;
            const float hb0 = (FAN ? 0.5f * fmaf(fmaf((float)xs, ray.sT, -yf * ray.cT), ray.kbw, ray.bwc)
                                   : 0.5f * g.beamWidthF) * ray.fp.iw;
            // the window's pixels, unrolled for the warp's window width
            auto row_sum = [&](auto wn) {
                constexpr int WN = decltype(wn)::value;
                float4 pp[WN], pm[WN];
#pragma unroll
                for (int j = 0; j < WN; ++j) {
                    pp[j] = staged ? st.buf[bc][i][0][xs + j - lo] : __ldg(q + xs + j);
                    pm[j] = staged ? st.buf[bc][i][1][hi - xs - j] : __ldg(q - xs - j);
                }
#pragma unroll
                for (int j = 0; j < WN; ++j) {
                    const float D = fmaf((float)j, ray.cRw, r0);
                    const float H = FAN ? fmaf((float)j, ray.dhbw, hb0) : hb0;
                    const float w = footprint_weight_v(D, H, ray.fp);
                    S[0] = fmaf(w, neg ? pp[j].y : pp[j].x, S[0]);
                    S[6] = fmaf(w, neg ? pm[j].y : pm[j].x, S[6]);
                    S[4] = fmaf(w, neg ? pp[j].x : pp[j].y, S[4]);
                    S[2] = fmaf(w, neg ? pm[j].x : pm[j].y, S[2]);
                    S[5] = fmaf(w, neg ? pp[j].w : pp[j].z, S[5]);
                    S[3] = fmaf(w, neg ? pm[j].w : pm[j].z, S[3]);
                    S[1] = fmaf(w, neg ? pp[j].z : pp[j].w, S[1]);
                    S[7] = fmaf(w, neg ? pm[j].z : pm[j].w, S[7]);
                }
            };
            if (wcode == 3) row_sum(std::integral_constant<int, 3>{});
            else row_sum(std::integral_constant<int, 4>{});
        }
    }
    failed = __syncthreads_or(failed);
    if (failed) {
        if (threadIdx.x == 0) atomicExch(&g_fwd_stage_timeout, 1);
#pragma unroll
        for (int j = 0; j < 8; ++j) S[j] = __int_as_float(0x7fc00000);
    }
    if (!live) return;
    const int pC = g.pC;
#pragma unroll
    for (int j = 0; j < 8; ++j) {
        const int v = p.view[b].out[j];
        if (v < 0) continue;
        const int det = j < 4 ? k : 2 * pC - k;
        const int det2 = 2 * pC - det;
        const size_t row = (size_t)v * g.W;
        sino[row + det] = S[j] / g.effRate;
        if (!FAN) sino[row + det2] = S[j ^ 2] / g.effRate;
    }
}
#endif

static FwdParams fwd_params(const ctprj_plan *pl)
{
    FwdParams p;
    p.sms = 148;
    cudaDeviceGetAttribute(&p.sms, cudaDevAttrMultiProcessorCount, pl->device);
    p.g = pl->g;
    p.nb = pl->nb;
    p.k0 = pl->k0;
    p.nk = pl->nk;
    p.zero_col0 = (pl->g.W % 2 == 0);
    p.view = pl->d_fview;
    p.det = pl->d_det;
    p.bhc = BhcArgs{};
    return p;
}

static dim3 fwd_grid(const ctprj_plan *pl)
{
    return dim3((pl->nb + kFwdViews - 1) / kFwdViews, (pl->nk + 31) / 32);
}

int forward_blocks(const ctprj_plan *pl)
{
    const dim3 g = fwd_grid(pl);
    return (int)(g.x * g.y);
}

int launch_forward(const ctprj_plan *pl, const float4 *quad, float *sino,
                   unsigned long long *counter, cudaStream_t s)
{
    const FwdParams p = fwd_params(pl);
    const dim3 grid = fwd_grid(pl), block(kFwdThreads);
    const bool fan = pl->g.fan != 0;
    if (counter) {
        if (fan) k_forward<true, kModeCount><<<grid, block, 0, s>>>(p, quad, sino, counter);
        else k_forward<false, kModeCount><<<grid, block, 0, s>>>(p, quad, sino, counter);
    } else {
#if CTPRJ_FWD_STAGE
        if (fan) k_forward_staged<true><<<grid, block, 0, s>>>(p, quad, sino);
        else k_forward_staged<false><<<grid, block, 0, s>>>(p, quad, sino);
#else
        if (fan) k_forward<true, kModePlain><<<grid, block, 0, s>>>(p, quad, sino, counter);
        else k_forward<false, kModePlain><<<grid, block, 0, s>>>(p, quad, sino, counter);
#endif
    }
    return cuda_error(cudaGetLastError(), "forward launch");
}

int launch_forward_bhc(const ctprj_plan *pl, const float4 *quad,
                       const BhcArgs &a, int *nparts, cudaStream_t s)
{
    FwdParams p = fwd_params(pl);
    p.bhc = a;
    const dim3 grid = fwd_grid(pl), block(kFwdThreads);
    if (pl->g.fan) k_forward<true, kModeBhc><<<grid, block, 0, s>>>(p, quad, nullptr, nullptr);
    else k_forward<false, kModeBhc><<<grid, block, 0, s>>>(p, quad, nullptr, nullptr);
    if (nparts) *nparts = (int)(grid.x * grid.y);
    return cuda_error(cudaGetLastError(), "fused polychromatic forward launch");
}

// ---------------------------------------------------------------- backward

// The eight images of octant pixel (x, y), in the order of the accumulators
// (prj/cpuPrj.c:308-316): (x,y) (-y,x) (-x,-y) (y,-x) (x,-y) (y,x) (-x,y) (-y,-x).
__device__ __forceinline__ void image_of(int j, int x, int y, int &gx, int &gy)
{
    switch (j) {
    case 0: gx = x; gy = y; break;
    case 1: gx = -y; gy = x; break;
    case 2: gx = -x; gy = -y; break;
    case 3: gx = y; gy = -x; break;
    case 4: gx = x; gy = -y; break;
    case 5: gx = y; gy = x; break;
    case 6: gx = -x; gy = y; break;
    default: gx = -y; gy = -x; break;
    }
}

// One base view of the pixel-driven backprojection for octant pixel (x, y):
// the detectors under the pixel's shadow, one footprint weight each, serving
// the eight symmetric images (prj/cpuPrj.c:213-300).  Everything is read from
// global memory (L1); used by k_backward_direct and, for views whose tile
// shadow exceeds the staging capacity, by k_backward_tiled.
template <bool FAN, bool COUNT, bool FBP>
__device__ __forceinline__ void bwd_view_direct(const BwdParams &p, const float *__restrict__ sino,
                                                int i, int x, int y, int nimg, float (&S)[8],
                                                unsigned long long &nz)
{
    const Geo &g = p.g;
    const int dmax = (g.W - 1) / 2, pC = g.pC;
    const float dSf = (float)g.dSize;
    const double xd = x, yd = y;
    const float xf = (float)x, yf = (float)y;
    const BwdView &bv = p.view[i];
    const double cT = bv.c, sT = bv.s;
    const float cTf = bv.cf, sTf = bv.sf;
    const double u = fma(xd, cT, yd * sT);    // along the detector
    float tlo, thi, qe = 0.0f;
    double v = 0.0;
    if (FAN) {
        // shadow of the pixel's corners on the virtual detector
        // (prj/cpuPrj.c:218-244)
        v = fma(yd, cT, -xd * sT);
        qe = (float)(g.d - v);
        const float ocm = fmaf(xf - 0.5f, cTf, (yf - 0.5f) * sTf);
        const float qem = fmaf(xf - 0.5f, sTf, -(yf - 0.5f) * cTf) + g.dF;
        const float t0 = g.dF * ocm / qem;
        const float t1 = g.dF * (ocm + cTf) / (qem + sTf);
        const float t2 = g.dF * (ocm + cTf + sTf) / (qem + sTf - cTf);
        const float t3 = g.dF * (ocm + sTf) / (qem - cTf);
        tlo = fminf(fminf(t0, t1), fminf(t2, t3));
        thi = fmaxf(fmaxf(t0, t1), fmaxf(t2, t3));
    } else {
        const float hw = 0.5f * (fabsf(cTf) + fabsf(sTf));
        const float uf = (float)u;
        tlo = uf - hw;
        thi = uf + hw;
    }
    int dl = (int)roundf(fmaxf(tlo / dSf, (float)(-dmax - 1)));
    int dr = (int)roundf(fminf(thi / dSf, (float)(dmax + 1)));
    dl = max(dl, -dmax);
    dr = min(dr, dmax);
    Footprint pfp;
    if (!FAN) {
        pfp.h = bv.h; pfp.b1 = bv.b1; pfp.b2 = bv.b2; pfp.w = bv.w; pfp.iw2 = bv.iw2;
    }
    for (int dt = dl; dt <= dr; ++dt) {
        const DetEntry &de = p.det[dt + pC];
        float w;
        if (FAN) {
            // distance from the detector's ray: cos B (u - t) + sin B v
            const float dist = (float)fma(de.cB, u - de.t, de.sB * v);
            const float cR = fmaf(de.cBf, cTf, -de.sBf * sTf);
            const float sR = fmaf(de.sBf, cTf, de.cBf * sTf);
            const Footprint fp = make_footprint(cR, sR);
            w = footprint_weight(dist, qe * g.beamWidthF * de.invbq, fp);
            if (FBP) w = w * g.dF * g.dF / qe / qe;
        } else {
            w = footprint_weight((float)(u - de.t), g.beamWidthF, pfp);
        }
        if (COUNT) {
            if (w != 0.0f) nz += (nimg == 8 ? bv.cnt8 : bv.cnt4);
            continue;
        }
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            const int sg = j < 4 ? dt : -dt;
            const int row = bv.row[j];
            if (row >= 0) S[j] = fmaf(w, __ldg(sino + row + pC + sg), S[j]);
            if (!FAN) {
                const int row2 = bv.row2[j];
                if (row2 >= 0) S[j] = fmaf(w, __ldg(sino + row2 + pC - sg), S[j]);
            }
        }
    }
}

__device__ __forceinline__ void decode_tile(int tile, int &tx, int &ty)
{
    tx = (int)((sqrtf(8.0f * (float)tile + 1.0f) - 1.0f) * 0.5f);
    while ((tx + 1) * (tx + 2) / 2 <= tile) ++tx;
    while (tx * (tx + 1) / 2 > tile) --tx;
    ty = tile - tx * (tx + 1) / 2;
}

__device__ __forceinline__ void write_octant(const BwdParams &p, float *__restrict__ img, int x,
                                             int y, int nimg, const float (&S)[8])
{
    const Geo &g = p.g;
    const int h2 = g.h2, N = g.n;
#pragma unroll
    for (int j = 0; j < 8; ++j) {
        if (j >= nimg) break;
        int gx, gy;
        image_of(j, x, y, gx, gy);
        const float val = S[j] * p.scale;
        img[(size_t)(gy + h2) * N + (gx + h2)] = val / g.effRate;
    }
}

// one tile of the unstaged backprojection (plain mode), for persistent use
template <bool FAN>
__device__ __forceinline__ void backward_tile_direct(const BwdParams &p, int tile,
                                                     const float *__restrict__ sino,
                                                     float *__restrict__ img)
{
    const Geo &g = p.g;
    if (p.zero_axes && tile == 0)
        for (int i = threadIdx.x; i < g.n; i += blockDim.x) {
            img[i] = 0.0f;
            img[(size_t)i * g.n] = 0.0f;
        }
    int tx, ty;
    decode_tile(tile, tx, ty);
    const int x = tx * kBwdTile + (int)(threadIdx.x % kBwdTile);
    const int y = ty * kBwdTile + (int)(threadIdx.x / kBwdTile);
    if (x > g.half || y > x) return;
    const int nimg = (y == 0 || y == x) ? 4 : 8;
    float S[8];
#pragma unroll
    for (int j = 0; j < 8; ++j) S[j] = 0.0f;
    unsigned long long nz = 0;
    for (int i = 0; i < p.nv; ++i) bwd_view_direct<FAN, false, false>(p, sino, i, x, y, nimg, S, nz);
    write_octant(p, img, x, y, nimg, S);
}

template <bool FAN, bool COUNT, bool FBP>
__global__ void __launch_bounds__(kBwdTile * kBwdTile)
k_backward(const BwdParams p, const float *__restrict__ sino, float *__restrict__ img,
           unsigned long long *__restrict__ counter)
{
    const Geo &g = p.g;
    if (!COUNT && p.zero_axes && blockIdx.x == 0)
        for (int i = threadIdx.x; i < g.n; i += blockDim.x) {
            img[i] = 0.0f;
            img[(size_t)i * g.n] = 0.0f;
        }
    int tx, ty;
    decode_tile(blockIdx.x, tx, ty);
    const int x = tx * kBwdTile + (int)(threadIdx.x % kBwdTile);
    const int y = ty * kBwdTile + (int)(threadIdx.x / kBwdTile);
    if (x > g.half || y > x) return;
    const int nimg = (y == 0 || y == x) ? 4 : 8;
    float S[8];
#pragma unroll
    for (int j = 0; j < 8; ++j) S[j] = 0.0f;
    unsigned long long nz = 0;
    for (int i = 0; i < p.nv; ++i) bwd_view_direct<FAN, COUNT, FBP>(p, sino, i, x, y, nimg, S, nz);
    if (COUNT) {
        if (nz) atomicAdd(counter, nz);
        return;
    }
    write_octant(p, img, x, y, nimg, S);
}

// ------------------------------------------------------ backward, staged tiles
//
// The same backprojection with the per-(view, detector) work hoisted out of the
// per-pixel loop.  A block owns a 16 x 16 tile of octant pixels; for a batch of
// VB base views it first stages, for every detector under the tile's shadow,
// (a) the ray's footprint coefficients and its distance from the tile centre,
// computed in FP64 and rounded, and (b) the eight mirrored sinogram samples the
// weight will multiply.  Each pixel then needs only its offset from the tile
// centre: dist = D_k + cos B_k du + sin B_k dv, a saturating-FMA footprint and
// eight shared-memory reads per detector.  The staging capacity SEG (detectors
// per view and tile) is chosen per plan from the exact maximum shadow width,
// found once by k_tile_span_max; geometries whose shadows exceed 64 detectors
// use the unstaged kernel.

struct TileSpan {
    int klo, nseg;
};

// Detectors any pixel of tile (tx, ty) can reach in base view bv, as the first
// one (relative to the centre bin) and a count, with one spare on each side
// (the pixels' own shadows are rounded to the nearest bin from FP32 corners).
// nseg = 1 << 20 flags a tile the source sees from behind or edge-on.
__device__ __forceinline__ TileSpan tile_span(const Geo &g, const BwdView &bv, int tx, int ty)
{
    const int dmax = (g.W - 1) / 2;
    const float X0 = tx * kBwdTile - 0.5f, X1 = X0 + kBwdTile;
    const float Y0 = ty * kBwdTile - 0.5f, Y1 = Y0 + kBwdTile;
    const float cx[4] = {X0, X1, X1, X0}, cy[4] = {Y0, Y0, Y1, Y1};
    float lo = 0.0f, hi = 0.0f;
    bool bad = false;
    for (int q = 0; q < 4; ++q) {
        const float oc = fmaf(cx[q], bv.cf, cy[q] * bv.sf);
        float tq = oc;
        if (g.fan) {
            const float qe = fmaf(cx[q], bv.sf, -cy[q] * bv.cf) + g.dF;
            bad |= !(qe > 1e-3f * g.dF);
            tq = g.dF * oc / qe;
        }
        lo = q == 0 ? tq : fminf(lo, tq);
        hi = q == 0 ? tq : fmaxf(hi, tq);
    }
    TileSpan sp;
    const float inv = (float)(1.0 / g.dSize), lim = (float)dmax + 2.0f;
    const int klo = max(__float2int_rd(fminf(fmaxf(lo * inv, -lim), lim)) - 1, -dmax);
    const int khi = min(__float2int_ru(fminf(fmaxf(hi * inv, -lim), lim)) + 1, dmax);
    sp.klo = klo;
    sp.nseg = bad ? (1 << 20) : khi - klo + 1;
    return sp;
}

// The same span from a full warp: lane l takes corner l % 4, the four
// corners' projections are reduced over aligned groups of four lanes (min and
// max are exact, so every lane gets tile_span's result)
__device__ __forceinline__ TileSpan tile_span_lanes(const Geo &g, const BwdView &bv, int tx, int ty, int lane)
{
    const int dmax = (g.W - 1) / 2, q = lane & 3;
    const float X0 = tx * kBwdTile - 0.5f, Y0 = ty * kBwdTile - 0.5f;
    const float cx = (q == 1 || q == 2) ? X0 + kBwdTile : X0, cy = q >= 2 ? Y0 + kBwdTile : Y0;
    const float oc = fmaf(cx, bv.cf, cy * bv.sf);
    float tq = oc;
    int bad = 0;
    if (g.fan) {
        const float qe = fmaf(cx, bv.sf, -cy * bv.cf) + g.dF;
        bad = !(qe > 1e-3f * g.dF);
        tq = g.dF * oc / qe;
    }
    float lo = tq, hi = tq;
#pragma unroll
    for (int o = 1; o <= 2; o <<= 1) {
        lo = fminf(lo, __shfl_xor_sync(0xffffffffu, lo, o));
        hi = fmaxf(hi, __shfl_xor_sync(0xffffffffu, hi, o));
        bad |= __shfl_xor_sync(0xffffffffu, bad, o);
    }
    TileSpan sp;
    const float inv = (float)(1.0 / g.dSize), lim = (float)dmax + 2.0f;
    const int klo = max(__float2int_rd(fminf(fmaxf(lo * inv, -lim), lim)) - 1, -dmax);
    const int khi = min(__float2int_ru(fminf(fmaxf(hi * inv, -lim), lim)) + 1, dmax);
    sp.klo = klo;
    sp.nseg = bad ? (1 << 20) : khi - klo + 1;
    return sp;
}

__global__ void k_tile_span_max(const BwdParams p, int tiles, int *__restrict__ out)
{
    int m = 0;
    const long long total = (long long)tiles * p.nv;
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < total;
         e += (long long)gridDim.x * blockDim.x) {
        int tx, ty;
        decode_tile((int)(e / p.nv), tx, ty);
        m = max(m, tile_span(p.g, p.view[e % p.nv], tx, ty).nseg);
    }
    atomicMax(out, m);
}

struct TileView {
    double uc, vc;        // tile centre along / across the detector (FP64)
    float cT, sT;
    float ucf, qec;       // u of the centre; d - v of the centre
    float hw;             // parallel: (|cos| + |sin|) / 2
    float A, B, AB;       // fan: (cos + sin) / 2, (cos - sin) / 2 (pixel corner offsets), A B
    int klo, nseg;
};

// shared memory of one staged tile
template <bool FAN, int SEG, int VB>
struct TiledSmem {
    // per staged detector, fan beam: D, cos B, sin B (all / w) and the
    // footprint's b2 / w; its hw and w / (2 b1) (the half beam width at depth
    // qe is qe (beam width / 2d) cos B / w: a multiple of the second
    // component).  Parallel beam: D / w.  A pixel reads 24 (4) bytes of them
    // per detector; the second plane keeps the 16-byte stride of the first
    // (measured faster than a packed 8-byte plane: 4.70 against 4.75 ms at the
    // 2048^2 fan workload, 0.90 against 1.00 ms at 1024^2 with d = 2048)
    float4 ra[FAN ? VB : 1][FAN ? SEG : 1];
    float4 rb[FAN && !kBwdDerive ? VB : 1][FAN && !kBwdDerive ? SEG : 1];
    float rx[FAN ? 1 : VB][FAN ? 1 : SEG];
    // the eight (sixteen) mirrored samples of a staged ray as two (four)
    // float4 planes: two (four) 16-byte reads per detector and pixel, and
    // consecutive detectors in consecutive banks
    float4 seg[VB][2][SEG];
    float4 seg2[FAN ? 1 : VB][2][FAN ? 1 : SEG];
    TileView tv[VB];
    FootprintV pfs[VB];
};

// one float from global into shared memory without a register round trip;
// an invalid source reads nothing and writes zero
__device__ __forceinline__ void stage_async4(float *smem, const float *gmem, bool valid)
{
    const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;\n" ::"r"(sa), "l"(gmem), "r"(valid ? 4 : 0)
                 : "memory");
}

// The footprint numbers of a staged fan detector.  All three follow from
// t = lo / hi of the ray's direction: b2 / w = (1 + t) / (2 t), hw = t / 2 =
// 1 / (4 b2/w - 2) and w / (2 b1) = t / (1 - t) = 1 / (2 b2/w - 2).  The
// derived pair also holds where make_footprint_v floors a zero width: for
// w = 0, hw comes out ~1e-31 (it multiplies a bounded term) and w / (2 b1)
// matches the floored ratio; for b1 = 0 the floor below keeps the ratio
// finite.  Each is within ~1e-7 of the stored value's effect on a weight.
__device__ __forceinline__ FootprintV staged_footprint(const float4 a, const float4 &b)
{
    FootprintV f;
    f.c1 = a.w;
    if (kBwdDerive) {
        f.hw = __fdividef(1.0f, fmaf(4.0f, a.w, -2.0f));
        f.rho = __fdividef(1.0f, fmaxf(fmaf(2.0f, a.w, -2.0f), 1e-30f));
    } else {
        f.hw = b.x;
        f.rho = b.y;
    }
    return f;
}

// Staging of one batch of VB base views for tile (tx, ty) (every thread of the
// block takes part; ends with a block barrier), a warp per view: A, the
// tile's detector span and centre in the view (every lane computes it, lane 0
// keeps it for the pixels' pass); B1, the footprint coefficients of the staged
// detectors; B2, their mirrored sinogram samples (a lane per detector: each
// load instruction reads one sinogram row contiguously).
template <bool FAN, int SEG, int VB>
__device__ __forceinline__ void stage_batch(const BwdParams &p, const float *__restrict__ sino, int tx, int ty,
                                            double xc, double yc, int i0, int nb, TiledSmem<FAN, SEG, VB> &sm)
{
    const Geo &g = p.g;
    auto &ra = sm.ra;
    auto &rb = sm.rb;
    auto &rx = sm.rx;
    auto &seg = sm.seg;
    auto &seg2 = sm.seg2;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, kWarps = blockDim.x >> 5;
    const int pC = g.pC;
    for (int iv = warp; iv < nb; iv += kWarps) {
        const BwdView &bv = p.view[i0 + iv];
        // A
        const TileSpan sp = tile_span_lanes(g, bv, tx, ty, lane);
        TileView t;
        t.cT = bv.cf;
        t.sT = bv.sf;
        t.uc = fma(xc, bv.c, yc * bv.s);
        t.vc = fma(yc, bv.c, -xc * bv.s);
        t.ucf = (float)t.uc;
        t.qec = (float)(g.d - t.vc);
        t.hw = 0.5f * (fabsf(bv.cf) + fabsf(bv.sf));
        t.A = 0.5f * (bv.cf + bv.sf);
        t.B = 0.5f * (bv.cf - bv.sf);
        t.AB = t.A * t.B;
        t.klo = sp.klo;
        t.nseg = min(sp.nseg, SEG);   // the plan chose SEG above every span
        const FootprintV pf = FAN ? FootprintV{} : make_footprint_v(bv.cf, bv.sf);
        if (lane == 0) {
            sm.tv[iv] = t;
            if (!FAN) sm.pfs[iv] = pf;
        }
#if CTPRJ_BWD_ASYNC
        // B2 first, asynchronously: the same samples as below, in flight while
        // B1 runs; the block barrier at the end follows a wait for them
        for (int kk = lane; kk < t.nseg; kk += 32) {
            const int dt = t.klo + kk;
#pragma unroll
            for (int j = 0; j < 8; ++j) {
                const int row = bv.row[j];
                stage_async4(&seg[iv][j >> 2][kk].x + (j & 3),
                             sino + (row >= 0 ? row + pC + (j < 4 ? dt : -dt) : 0), row >= 0);
            }
            if (!FAN) {
#pragma unroll
                for (int j = 0; j < 8; ++j) {
                    const int row2 = bv.row2[j];
                    stage_async4(&seg2[FAN ? 0 : iv][j >> 2][FAN ? 0 : kk].x + (j & 3),
                                 sino + (row2 >= 0 ? row2 + pC - (j < 4 ? dt : -dt) : 0), row2 >= 0);
                }
            }
        }
#endif
        for (int kk = lane; kk < t.nseg; kk += 32) {
            // B1
            const DetEntry &de = p.det[t.klo + kk + pC];
            if (FAN) {
                const double D = fma(de.cB, t.uc - de.t, de.sB * t.vc);
                const float cR = fmaf(de.cBf, t.cT, -de.sBf * t.sT);
                const float sR = fmaf(de.sBf, t.cT, de.cBf * t.sT);
                const FootprintV f = make_footprint_v(cR, sR);
                ra[FAN ? iv : 0][FAN ? kk : 0] = make_float4((float)D * f.iw, de.cBf * f.iw, de.sBf * f.iw, f.c1);
                if (!kBwdDerive)
                    rb[FAN && !kBwdDerive ? iv : 0][FAN && !kBwdDerive ? kk : 0] = make_float4(f.hw, f.rho, 0.0f, 0.0f);
            } else {
                rx[FAN ? 0 : iv][FAN ? 0 : kk] = (float)(t.uc - de.t) * pf.iw;
            }
#if !CTPRJ_BWD_ASYNC
            // B2
            const int dt = t.klo + kk;
            float v[8];
#pragma unroll
            for (int j = 0; j < 8; ++j) {
                const int row = bv.row[j];
                v[j] = row >= 0 ? __ldg(sino + row + pC + (j < 4 ? dt : -dt)) : 0.0f;
            }
            seg[iv][0][kk] = make_float4(v[0], v[1], v[2], v[3]);
            seg[iv][1][kk] = make_float4(v[4], v[5], v[6], v[7]);
            if (!FAN) {   // the point-reflected detectors of the opposite view
#pragma unroll
                for (int j = 0; j < 8; ++j) {
                    const int row2 = bv.row2[j];
                    v[j] = row2 >= 0 ? __ldg(sino + row2 + pC - (j < 4 ? dt : -dt)) : 0.0f;
                }
                seg2[FAN ? 0 : iv][0][FAN ? 0 : kk] = make_float4(v[0], v[1], v[2], v[3]);
                seg2[FAN ? 0 : iv][1][FAN ? 0 : kk] = make_float4(v[4], v[5], v[6], v[7]);
            }
#endif
        }
    }
#if CTPRJ_BWD_ASYNC
    asm volatile("cp.async.wait_all;\n" ::: "memory");
#endif
    __syncthreads();
}

// One tile of the staged backprojection (all threads of the block take part).
// WIN = 3: every pixel shadow of the plan is narrower than 1.9 detectors (the
// plan's bound), so the detectors a pixel reaches in a view always lie within
// the three centred on the projection of its centre, tc; WIN = 4: narrower
// than 2.85, and they lie within the four from floor(tc) - 1.  Those detectors
// are summed straight, without the per-pixel shadow range (WIN = 0: the
// range).  A detector of the window that the reference's range rule
// (prj/cpuPrj.c:218-244) leaves out lies beyond the pixel's footprint and adds
// a weight of exactly zero, except within ~1e-4 detector of a shadow edge,
// where the footprint and the exact corner shadow differ and the weight is
// below 1e-7.
template <bool FAN, bool FBP, int SEG, int VB, int WIN>
__device__ __forceinline__ void backward_tile(const BwdParams &p, int tile,
                                              const float *__restrict__ sino,
                                              float *__restrict__ img,
                                              TiledSmem<FAN, SEG, VB> &sm)
{
    const Geo &g = p.g;
    auto &ra = sm.ra;
    auto &rb = sm.rb;
    auto &rx = sm.rx;
    auto &seg = sm.seg;
    auto &seg2 = sm.seg2;
    auto &tv = sm.tv;
    auto &pfs = sm.pfs;

    if (p.zero_axes && tile == 0)
        for (int i = threadIdx.x; i < g.n; i += blockDim.x) {
            img[i] = 0.0f;
            img[(size_t)i * g.n] = 0.0f;
        }
    int tx, ty;
    decode_tile(tile, tx, ty);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    // a warp takes an 8 x 4 block of the tile, each half-warp a 4 x 4 square:
    // the 16 pixels of a square project onto at most 3 sqrt(2) m + 1
    // consecutive staged detectors (m the magnification), fewer than the
    // eight 16-byte entries that share no bank, so a half-warp's window loads
    // never conflict (8 x 2 rows do)
#if CTPRJ_BWD_ROWS
    const int x = tx * kBwdTile + ((warp & 1) << 3) + (lane & 7);
    const int y = ty * kBwdTile + ((warp >> 1) << 2) + (lane >> 3);
#else
    const int x = tx * kBwdTile + ((warp & 1) << 3) + ((lane >> 4) << 2) + (lane & 3);
    const int y = ty * kBwdTile + ((warp >> 1) << 2) + ((lane >> 2) & 3);
#endif
    const bool valid = x <= g.half && y <= x;
    const int nimg = (y == 0 || y == x) ? 4 : 8;
    const double xc = tx * kBwdTile + 0.5 * (kBwdTile - 1), yc = ty * kBwdTile + 0.5 * (kBwdTile - 1);
    const float dx = (float)(x - xc), dy = (float)(y - yc);
    const int dmax = (g.W - 1) / 2;
    const float invdS = (float)(1.0 / g.dSize), dFs = (float)((double)g.dF / g.dSize);
    const float hbpar = 0.5f * g.beamWidthF;
    // fan beam: the half beam width at depth qe on ray B, over w, is
    // qe Kb (cos B / w) (prj/cpuPrj.c:254: bw = qe beamWidth cos B / d)
    const float Kb = FAN ? (float)(0.5 * g.beamWidth / g.d) : 0.0f;
    // the eight sums, S[j] += w p[j], in pairs: one fma.rn.f32x2 for two
    // sums (each rounded as one fmaf)
    float2 S2[4];
#pragma unroll
    for (int j = 0; j < 4; ++j) S2[j] = make_float2(0.0f, 0.0f);
    auto accumulate = [&](const float w, const float4 p0, const float4 p1) {
        const float2 ww = make_float2(w, w);
        S2[0] = __ffma2_rn(ww, make_float2(p0.x, p0.y), S2[0]);
        S2[1] = __ffma2_rn(ww, make_float2(p0.z, p0.w), S2[1]);
        S2[2] = __ffma2_rn(ww, make_float2(p1.x, p1.y), S2[2]);
        S2[3] = __ffma2_rn(ww, make_float2(p1.z, p1.w), S2[3]);
    };

    for (int i0 = 0; i0 < p.nv; i0 += VB) {
        const int nb = min(VB, p.nv - i0);
        stage_batch<FAN, SEG, VB>(p, sino, tx, ty, xc, yc, i0, nb, sm);
        // C: every pixel of the tile over the batch
        if (valid) {
            for (int iv = 0; iv < nb; ++iv) {
                const TileView &t = tv[iv];
                const float du = fmaf(dx, t.cT, dy * t.sT);
                const float dv = fmaf(dy, t.cT, -dx * t.sT);
                const float u = t.ucf + du;
                if (WIN > 0 && t.nseg >= WIN) {   // t.nseg is the same for the whole block
                    const float qe = FAN ? t.qec - dv : 0.0f;
                    // the detector under the pixel centre, in staged units
                    const float tc = FAN ? __fdividef(dFs * u, qe) : u * invdS;
                    // nearest detector, half to even as __float2int_rn, by an FP32
                    // add: for |tc| < 2^22 (staged units: |tc| < the row length)
                    // tc + 1.5 * 2^23 lies in [2^23, 2^24), where the add rounds to
                    // an integer, so its low mantissa bits are that integer (one
                    // arithmetic op instead of a conversion on the XU pipe: 0.5 %
                    // at the 2048^2 fan workload, 1.5-2 % at 512^2 and 256^2)
                    const int ks = WIN == 3 ? __float_as_int(tc + 12582912.0f) - 0x4B400000 : __float2int_rd(tc);
                    const int k0 = min(max(ks - 1 - t.klo, 0), t.nseg - WIN);
                    const float fbpw = FBP ? __fdividef(g.dF, qe) * __fdividef(g.dF, qe) : 1.0f;
                    const FootprintV fpar = FAN ? FootprintV{} : pfs[iv];
                    const float duw = FAN ? 0.0f : du * fpar.iw, Hpar = FAN ? 0.0f : hbpar * fpar.iw;
                    const float qeK = qe * Kb;
                    float w[WIN > 0 ? WIN : 1];
#pragma unroll
                    for (int q = 0; q < WIN; ++q) {
                        if (FAN) {
                            const float4 a = ra[FAN ? iv : 0][FAN ? k0 + q : 0];
                            const float D = fmaf(a.y, du, fmaf(a.z, dv, a.x));
                            const FootprintV f = staged_footprint(a, rb[FAN && !kBwdDerive ? iv : 0]
                                                                        [FAN && !kBwdDerive ? k0 + q : 0]);
                            w[q] = footprint_weight_v(D, qeK * a.y, f);
                            if (FBP) w[q] *= fbpw;
                        } else {
                            w[q] = footprint_weight_v(rx[FAN ? 0 : iv][FAN ? 0 : k0 + q] + duw, Hpar, fpar);
                        }
                    }
#pragma unroll
                    for (int q = 0; q < WIN; ++q) {
                        accumulate(w[q], seg[iv][0][k0 + q], seg[iv][1][k0 + q]);
                        if (!FAN)
                            accumulate(w[q], seg2[FAN ? 0 : iv][0][FAN ? 0 : k0 + q],
                                       seg2[FAN ? 0 : iv][1][FAN ? 0 : k0 + q]);
                    }
                    continue;
                }
                float tlo, thi, qe = 0.0f;
                if (FAN) {
                    // the pixel's corner shadows (prj/cpuPrj.c:218-244), in
                    // detector units; only which detector each edge falls in
                    // matters here
                    qe = t.qec - dv;
                    const float A = t.A, B = t.B;
                    if (p.fast_shadow) {
                        // corner i at (u + du_i, qe + dq_i): t_i = K (u + du_i) / (1 + r dq_i)
                        // ~ K (u + du_i - rho dq_i - r du_i dq_i), K = d r, rho = r u; the
                        // corners pair up as u + c +- a1 and u - c +- a2
                        const float r = __fdividef(1.0f, qe), rho = r * u, c = __fmul_rn(r, t.AB);
                        const float a1 = fabsf(fmaf(rho, B, A)), a2 = fabsf(fmaf(-rho, A, B));
                        const float K = dFs * r;
                        tlo = K * (u + fminf(c - a1, -c - a2));
                        thi = K * (u + fmaxf(c + a1, a2 - c));
                    } else {
                        const float t0 = __fdividef(dFs * (u - A), qe + B);
                        const float t1 = __fdividef(dFs * (u + B), qe + A);
                        const float t2 = __fdividef(dFs * (u + A), qe - B);
                        const float t3 = __fdividef(dFs * (u - B), qe - A);
                        tlo = fminf(fminf(t0, t1), fminf(t2, t3));
                        thi = fmaxf(fmaxf(t0, t1), fmaxf(t2, t3));
                    }
                } else {
                    tlo = (u - t.hw) * invdS;
                    thi = (u + t.hw) * invdS;
                }
                // float-to-int conversion saturates, so far-out shadows clamp
                int dl = __float2int_rn(tlo);
                int dr = __float2int_rn(thi);
                dl = max(max(dl, -dmax) - t.klo, 0);
                dr = min(min(dr, dmax) - t.klo, t.nseg - 1);
                const float fbpw = FBP ? __fdividef(g.dF, qe) * __fdividef(g.dF, qe) : 1.0f;
                const FootprintV fpar = FAN ? FootprintV{} : pfs[iv];
                const float duw = FAN ? 0.0f : du * fpar.iw, Hpar = FAN ? 0.0f : hbpar * fpar.iw;
                const float qeK = qe * Kb;
                // the weight of staged detector kk for this pixel
                auto weight = [&](const int kk) {
                    float w;
                    if (FAN) {
                        const float4 a = ra[FAN ? iv : 0][FAN ? kk : 0];
                        const float D = fmaf(a.y, du, fmaf(a.z, dv, a.x));
                        const FootprintV f = staged_footprint(a, rb[FAN && !kBwdDerive ? iv : 0]
                                                                    [FAN && !kBwdDerive ? kk : 0]);
                        w = footprint_weight_v(D, qeK * a.y, f);
                        if (FBP) w *= fbpw;
                    } else {
                        w = footprint_weight_v(rx[FAN ? 0 : iv][FAN ? 0 : kk] + duw, Hpar, fpar);
                    }
                    return w;
                };
                // two detectors per step, their shared-memory reads issued
                // together (the second of an odd-length run re-reads dr and is
                // skipped); per sum the order of the terms is unchanged
                for (int kk = dl; kk <= dr; kk += 2) {
                    const bool two = kk < dr;
                    const int kb = two ? kk + 1 : kk;
                    const float4 p0 = seg[iv][0][kk], p1 = seg[iv][1][kk];
                    const float4 r0 = seg[iv][0][kb], r1 = seg[iv][1][kb];
                    const float w0 = weight(kk);
                    const float w1 = weight(kb);
                    accumulate(w0, p0, p1);
                    if (!FAN) accumulate(w0, seg2[FAN ? 0 : iv][0][FAN ? 0 : kk], seg2[FAN ? 0 : iv][1][FAN ? 0 : kk]);
                    if (two) {
                        accumulate(w1, r0, r1);
                        if (!FAN) accumulate(w1, seg2[FAN ? 0 : iv][0][FAN ? 0 : kb], seg2[FAN ? 0 : iv][1][FAN ? 0 : kb]);
                    }
                }
            }
        }
        __syncthreads();
    }
    float S[8];
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        S[2 * j] = S2[j].x;
        S[2 * j + 1] = S2[j].y;
    }
    if (valid) write_octant(p, img, x, y, nimg, S);
}

#if CTPRJ_BWD_PAIR
// ------------------------------------- backward, two pixels per thread
//
// Build-time variant (CTPRJ_BWD_PAIR=1) of the fan-beam window kernel: a
// thread owns two horizontally adjacent pixels of the tile (128 threads per
// 16 x 16 tile), and for each view reads the staged detectors of the union of
// their two windows once: three to five detectors for two pixels instead of
// six.  Each pixel takes a weight for every detector of the union; those
// outside its own window lie beyond its shadow and add exactly zero, so the
// sums equal the one-pixel kernel's.
template <bool FBP, int SEG, int VB>
__global__ void __launch_bounds__(kBwdTile * kBwdTile / 2, 6)
k_backward_pair(const BwdParams p, const float *__restrict__ sino, float *__restrict__ img)
{
    __shared__ TiledSmem<true, SEG, VB> sm;
    const Geo &g = p.g;
    const int tile = blockIdx.x;
    if (p.zero_axes && tile == 0)
        for (int i = threadIdx.x; i < g.n; i += blockDim.x) {
            img[i] = 0.0f;
            img[(size_t)i * g.n] = 0.0f;
        }
    int tx, ty;
    decode_tile(tile, tx, ty);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    // a warp takes 8 x 8 pixels: lane (2 (lane % 4), lane / 4) and its right
    // neighbour.  Eight lanes of a quarter-warp then span 8 x 2 pixels, whose
    // windows fall in consecutive staged detectors (16 x 1 would spread them
    // over twice as many entries and double the shared-memory wavefronts)
    const int x1 = tx * kBwdTile + ((warp & 1) << 3) + ((lane & 3) << 1), x2 = x1 + 1;
    const int y = ty * kBwdTile + ((warp >> 1) << 3) + (lane >> 2);
    const bool valid1 = x1 <= g.half && y <= x1, valid2 = x2 <= g.half && y <= x2;
    const double xc = tx * kBwdTile + 0.5 * (kBwdTile - 1), yc = ty * kBwdTile + 0.5 * (kBwdTile - 1);
    const float dx1 = (float)(x1 - xc), dx2 = (float)(x2 - xc), dy = (float)(y - yc);
    const float dFs = (float)((double)g.dF / g.dSize);
    const float Kb = (float)(0.5 * g.beamWidth / g.d);
    float S1[8], S2[8];
#pragma unroll
    for (int j = 0; j < 8; ++j) S1[j] = S2[j] = 0.0f;
#if CTPRJ_BWD_PAIR == 2
    unsigned long long A1[4] = {0ull, 0ull, 0ull, 0ull}, A2[4] = {0ull, 0ull, 0ull, 0ull};
#endif

    for (int i0 = 0; i0 < p.nv; i0 += VB) {
        const int nb = min(VB, p.nv - i0);
        stage_batch<true, SEG, VB>(p, sino, tx, ty, xc, yc, i0, nb, sm);
        for (int iv = 0; iv < nb; ++iv) {
            const TileView &t = sm.tv[iv];
            const float du1 = fmaf(dx1, t.cT, dy * t.sT), du2 = fmaf(dx2, t.cT, dy * t.sT);
            const float dv1 = fmaf(dy, t.cT, -dx1 * t.sT), dv2 = fmaf(dy, t.cT, -dx2 * t.sT);
            const float qe1 = t.qec - dv1, qe2 = t.qec - dv2;
            const float tc1 = __fdividef(dFs * (t.ucf + du1), qe1);
            const float tc2 = __fdividef(dFs * (t.ucf + du2), qe2);
            // each pixel's window (staged units, unclipped) and their union, as
            // wide as the widest of the warp; a detector of the union outside
            // the staged span [0, nseg) lies beyond the tile's reach or the
            // detector's edge and is skipped
            const int k1 = __float2int_rn(tc1) - 1 - t.klo, k2 = __float2int_rn(tc2) - 1 - t.klo;
            const int un = __reduce_max_sync(0xffffffffu, max(k1, k2) - min(k1, k2) + 3);
            const int kb = min(k1, k2);
            const float fbpw1 = FBP ? __fdividef(g.dF, qe1) * __fdividef(g.dF, qe1) : 1.0f;
            const float fbpw2 = FBP ? __fdividef(g.dF, qe2) * __fdividef(g.dF, qe2) : 1.0f;
            auto slot = [&](const int kk) {
                if ((unsigned)kk >= (unsigned)t.nseg) return;
                const float4 a = sm.ra[iv][kk];
                const FootprintV f = staged_footprint(a, sm.rb[kBwdDerive ? 0 : iv][kBwdDerive ? 0 : kk]);
                float w1 = footprint_weight_v(fmaf(a.y, du1, fmaf(a.z, dv1, a.x)), (qe1 * Kb) * a.y, f);
                float w2 = footprint_weight_v(fmaf(a.y, du2, fmaf(a.z, dv2, a.x)), (qe2 * Kb) * a.y, f);
                if (FBP) {
                    w1 *= fbpw1;
                    w2 *= fbpw2;
                }
#if CTPRJ_BWD_PAIR == 2
                // packed: {S[2i], S[2i+1]} += {w, w} {p[2i], p[2i+1]}, one
                // fma.rn.f32x2 for two sums (each lane rounds as fmaf)
                const ulonglong2 q0 = *reinterpret_cast<const ulonglong2 *>(&sm.seg[iv][0][kk]);
                const ulonglong2 q1 = *reinterpret_cast<const ulonglong2 *>(&sm.seg[iv][1][kk]);
                unsigned long long ww1, ww2;
                asm("mov.b64 %0, {%1, %1};" : "=l"(ww1) : "f"(w1));
                asm("mov.b64 %0, {%1, %1};" : "=l"(ww2) : "f"(w2));
                asm("fma.rn.f32x2 %0, %1, %2, %0;" : "+l"(A1[0]) : "l"(ww1), "l"(q0.x));
                asm("fma.rn.f32x2 %0, %1, %2, %0;" : "+l"(A1[1]) : "l"(ww1), "l"(q0.y));
                asm("fma.rn.f32x2 %0, %1, %2, %0;" : "+l"(A1[2]) : "l"(ww1), "l"(q1.x));
                asm("fma.rn.f32x2 %0, %1, %2, %0;" : "+l"(A1[3]) : "l"(ww1), "l"(q1.y));
                asm("fma.rn.f32x2 %0, %1, %2, %0;" : "+l"(A2[0]) : "l"(ww2), "l"(q0.x));
                asm("fma.rn.f32x2 %0, %1, %2, %0;" : "+l"(A2[1]) : "l"(ww2), "l"(q0.y));
                asm("fma.rn.f32x2 %0, %1, %2, %0;" : "+l"(A2[2]) : "l"(ww2), "l"(q1.x));
                asm("fma.rn.f32x2 %0, %1, %2, %0;" : "+l"(A2[3]) : "l"(ww2), "l"(q1.y));
#else
                const float4 p0 = sm.seg[iv][0][kk], p1 = sm.seg[iv][1][kk];
                S1[0] = fmaf(w1, p0.x, S1[0]);
                S1[1] = fmaf(w1, p0.y, S1[1]);
                S1[2] = fmaf(w1, p0.z, S1[2]);
                S1[3] = fmaf(w1, p0.w, S1[3]);
                S1[4] = fmaf(w1, p1.x, S1[4]);
                S1[5] = fmaf(w1, p1.y, S1[5]);
                S1[6] = fmaf(w1, p1.z, S1[6]);
                S1[7] = fmaf(w1, p1.w, S1[7]);
                S2[0] = fmaf(w2, p0.x, S2[0]);
                S2[1] = fmaf(w2, p0.y, S2[1]);
                S2[2] = fmaf(w2, p0.z, S2[2]);
                S2[3] = fmaf(w2, p0.w, S2[3]);
                S2[4] = fmaf(w2, p1.x, S2[4]);
                S2[5] = fmaf(w2, p1.y, S2[5]);
                S2[6] = fmaf(w2, p1.z, S2[6]);
                S2[7] = fmaf(w2, p1.w, S2[7]);
#endif
            };
            slot(kb);
            slot(kb + 1);
            slot(kb + 2);
            if (un > 3) slot(kb + 3);
            if (un > 4) slot(kb + 4);
        }
        __syncthreads();
    }
#if CTPRJ_BWD_PAIR == 2
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        asm("mov.b64 {%0, %1}, %2;" : "=f"(S1[2 * j]), "=f"(S1[2 * j + 1]) : "l"(A1[j]));
        asm("mov.b64 {%0, %1}, %2;" : "=f"(S2[2 * j]), "=f"(S2[2 * j + 1]) : "l"(A2[j]));
    }
#endif
    if (valid1) write_octant(p, img, x1, y, (y == 0 || y == x1) ? 4 : 8, S1);
    if (valid2) write_octant(p, img, x2, y, (y == 0 || y == x2) ? 4 : 8, S2);
}
#endif

template <bool FAN, bool FBP, int SEG, int VB, int WIN>
__global__ void __launch_bounds__(kBwdTile * kBwdTile, CTPRJ_BWD_MINBLOCKS)
k_backward_tiled(const BwdParams p, const float *__restrict__ sino, float *__restrict__ img)
{
    __shared__ TiledSmem<FAN, SEG, VB> sm;
    backward_tile<FAN, FBP, SEG, VB, WIN>(p, blockIdx.x, sino, img, sm);
}

// upper bound of a pixel's shadow width in detectors, or 0 where none holds
// (a fan source inside or next to the image)
static double shadow_width_bound(const Geo &g)
{
    const double s2 = 1.4142135623730951;
    if (!g.fan) return s2 / g.dSize;
    const double R = (g.half + 1.0) * s2, d = g.d;
    if (!(d > 2.0 * R)) return 0.0;
    const double tg = R / (d - R);
    return s2 * d / (d - R) * (1.0 + tg * tg) / g.dSize;
}

static BwdParams bwd_params(const ctprj_plan *pl, int fbp, float scale)
{
    BwdParams p;
    p.g = pl->g;
    p.nv = pl->nv;
    const int T = (pl->g.half + 1 + kBwdTile - 1) / kBwdTile;
    p.tiles_side = T;
    p.zero_axes = (pl->g.n % 2 == 0);
    p.scale = fbp ? (float)((double)(kRefPiF / (float)pl->g.np) / pl->g.dSize / pl->g.dSize)
                  : scale;
    p.view = pl->d_bview;
    p.det = pl->d_det;
    // The staged fan kernel may bound a pixel's shadow from 1/qe and a first-
    // order expansion in (pixel half-diagonal) / qe instead of four divisions
    // when the dropped second-order terms stay below 1e-4 detector: at most
    //   K (h + 1) r^2 / 2,  r = 1 / (d - h),  K = d r / dSize,
    // h = the image's half-diagonal.  Detectors that the exact and the
    // bounded shadow disagree on lie within that distance of a shadow edge,
    // where the footprint weight is of the order of its square.
    p.fast_shadow = 0;
    if (pl->g.fan) {
        const double h = (pl->g.half + 0.5) * 1.4142135623730951 + 1.0;
        const double d = pl->g.d;
        if (d > 2.0 * h) {
            const double r = 1.0 / (d - h), K = d * r / pl->g.dSize;
            p.fast_shadow = K * (h + 1.0) * r * r * 0.5 <= 1e-4;
        }
    }
    // Widest pixel shadow, in detectors: a unit pixel spans at most sqrt(2)
    // across any ray; a fan magnifies that by d / qe <= d / (d - R) at the
    // pixel nearest the source (R: the image corner's distance from the
    // isocentre) and the detector's obliquity adds 1 + tan^2 of the fan
    // angle, tan <= R / (d - R).  Below 1.9 detectors the three detectors
    // centred on a pixel's projection hold its whole shadow.  (Below 2.85 the
    // four from floor(tc) - 1 would, but at the 1024^2 fan configuration, the
    // one such plan measured, four straight detectors ran slower than the
    // range: 1.82 against 1.66 ms per polychromatic gradient iteration.)  A
    // beam wider than the detector pitch (effectiveRate > 1) also reaches
    // detectors outside the shadow, which the reference's range rule leaves
    // out: such plans keep the per-pixel range.
    const double width = shadow_width_bound(pl->g);
    p.win = width > 0.0 && width <= 1.9 && pl->g.effRate <= 1.0f ? 3 : 0;
    return p;
}

// widest tile shadow of the plan's geometry, in detectors (plan creation)
int backward_max_span(const ctprj_plan *pl, int *max_span)
{
    const BwdParams p = bwd_params(pl, 0, 1.0f);
    const int tiles = p.tiles_side * (p.tiles_side + 1) / 2;
    int *d = nullptr;
    int st = cuda_error(cudaMalloc((void **)&d, sizeof(int)), "span scratch");
    if (st) return st;
    int h = 0;
    if (!(st = cuda_error(cudaMemset(d, 0, sizeof(int)), "span reset"))) {
        k_tile_span_max<<<296, 256>>>(p, tiles, d);
        if (!(st = cuda_error(cudaGetLastError(), "span launch")))
            st = cuda_error(cudaMemcpy(&h, d, sizeof(int), cudaMemcpyDeviceToHost), "span readback");
    }
    cudaFree(d);
    *max_span = h;
    return st;
}

template <int SEG, int VB, int WIN>
static void launch_tiled_win(const BwdParams &p, bool fan, int fbp, dim3 grid, dim3 block,
                             const float *sino, float *img, cudaStream_t s)
{
    if (fan) {
        if (fbp) k_backward_tiled<true, true, SEG, VB, WIN><<<grid, block, 0, s>>>(p, sino, img);
        else k_backward_tiled<true, false, SEG, VB, WIN><<<grid, block, 0, s>>>(p, sino, img);
    } else {
        if (fbp) k_backward_tiled<false, true, SEG, VB, WIN><<<grid, block, 0, s>>>(p, sino, img);
        else k_backward_tiled<false, false, SEG, VB, WIN><<<grid, block, 0, s>>>(p, sino, img);
    }
}

template <int SEG, int VB>
static void launch_tiled(const BwdParams &p, bool fan, int fbp, dim3 grid, dim3 block,
                         const float *sino, float *img, cudaStream_t s)
{
    if (p.win == 3) launch_tiled_win<SEG, VB, 3>(p, fan, fbp, grid, block, sino, img, s);
    else launch_tiled_win<SEG, VB, 0>(p, fan, fbp, grid, block, sino, img, s);
}

int launch_backward(const ctprj_plan *pl, const float *sino, float *img, int fbp,
                    unsigned long long *counter, cudaStream_t s, float scale)
{
    const BwdParams p = bwd_params(pl, fbp, scale);
    const int T = p.tiles_side;
    dim3 grid(T * (T + 1) / 2), block(kBwdTile * kBwdTile);
    const bool fan = pl->g.fan != 0;
    if (counter) {
        if (fan) k_backward<true, true, false><<<grid, block, 0, s>>>(p, sino, img, counter);
        else k_backward<false, true, false><<<grid, block, 0, s>>>(p, sino, img, counter);
    } else if (pl->bwd_seg == 0) {
        if (fbp) {
            if (fan) k_backward<true, false, true><<<grid, block, 0, s>>>(p, sino, img, counter);
            else k_backward<false, false, true><<<grid, block, 0, s>>>(p, sino, img, counter);
        } else {
            if (fan) k_backward<true, false, false><<<grid, block, 0, s>>>(p, sino, img, counter);
            else k_backward<false, false, false><<<grid, block, 0, s>>>(p, sino, img, counter);
        }
#if CTPRJ_BWD_PAIR
    } else if (fan && p.win == 3) {
        const dim3 pblock(kBwdTile * kBwdTile / 2);
        if (pl->bwd_seg <= 32) {
            if (fbp) k_backward_pair<true, 32, 16><<<grid, pblock, 0, s>>>(p, sino, img);
            else k_backward_pair<false, 32, 16><<<grid, pblock, 0, s>>>(p, sino, img);
        } else {
            if (fbp) k_backward_pair<true, 64, 8><<<grid, pblock, 0, s>>>(p, sino, img);
            else k_backward_pair<false, 64, 8><<<grid, pblock, 0, s>>>(p, sino, img);
        }
#endif
    } else if (pl->bwd_seg <= 32) {
        launch_tiled<32, 16>(p, fan, fbp, grid, block, sino, img, s);
    } else {
        launch_tiled<64, 8>(p, fan, fbp, grid, block, sino, img, s);
    }
    return cuda_error(cudaGetLastError(), "backward launch");
}

// ------------------------------------------------------------ batched launches
//
// One persistent launch serves a batch of slices of different geometries: each
// block repeatedly takes the next work item from a device counter -- a forward
// block (V views x 32 rays) or a backprojection tile of some slice -- finds its
// slice by binary search over the item prefix sums, and runs the same block
// body as the per-slice kernels.  Work is handed out in the slice order the
// host chose (e.g. largest slices first), so the tail of the launch is short.

__device__ __forceinline__ int find_slot(const long long *prefix, int n, long long item)
{
    int lo = 0, hi = n;
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (prefix[mid] <= item) lo = mid;
        else hi = mid;
    }
    return lo;
}

__device__ __forceinline__ long long next_item(unsigned long long *counter, long long *slot)
{
    __syncthreads();
    if (threadIdx.x == 0) *slot = (long long)atomicAdd(counter, 1ULL);
    __syncthreads();
    return *slot;
}

__global__ void __launch_bounds__(256) k_quad_batch(const BatchArgs a)
{
    __shared__ float tz[32][33], tw[32][33];
    for (long long e = blockIdx.x; e < a.ttotal; e += gridDim.x) {
        const int i = find_slot(a.tprefix, a.nslices, e);
        const BatchSlice &sl = a.slices[i];
        quad_tile(sl.img, sl.quad, sl.fp.g.n, (int)(e - a.tprefix[i]), tz, tw);
    }
}

// resident blocks asked of the register allocator: as many warps per SM as the
// per-plan forward
template <int V>
__global__ void __launch_bounds__(32 * V, 4 * CTPRJ_FWD_MINBLOCKS / V) k_forward_batch(const BatchArgs a)
{
    __shared__ long long slot;
    for (;;) {
        const long long item = next_item(a.counter, &slot);
        if (item >= a.total) return;
        const int i = find_slot(a.prefix, a.nslices, item);
        const BatchSlice &sl = a.slices[a.order[i]];
        const int local = (int)(item - a.prefix[i]);
        const int gx = (sl.fp.nb + V - 1) / V;
        const int bx = local % gx, by = local / gx;
        if (sl.fp.g.fan)
            forward_rays<true, kModePlain, V>(sl.fp, bx, by, sl.quad, sl.sino, nullptr, nullptr, nullptr);
        else
            forward_rays<false, kModePlain, V>(sl.fp, bx, by, sl.quad, sl.sino, nullptr, nullptr, nullptr);
    }
}

template <int SEG, int VB>
constexpr size_t tiled_smem_bytes()
{
    return sizeof(TiledSmem<true, SEG, VB>) > sizeof(TiledSmem<false, SEG, VB>)
               ? sizeof(TiledSmem<true, SEG, VB>)
               : sizeof(TiledSmem<false, SEG, VB>);
}

// one staged tile of a batch slice, with the slice's own window choice
template <int SEG, int VB>
__device__ __forceinline__ void batch_tile(const BatchSlice &sl, int tile, unsigned char *raw)
{
    if (sl.bp.g.fan) {
        auto &sm = *reinterpret_cast<TiledSmem<true, SEG, VB> *>(raw);
        if (sl.bp.win == 3) backward_tile<true, false, SEG, VB, 3>(sl.bp, tile, sl.bsino, sl.bimg, sm);
        else backward_tile<true, false, SEG, VB, 0>(sl.bp, tile, sl.bsino, sl.bimg, sm);
    } else {
        auto &sm = *reinterpret_cast<TiledSmem<false, SEG, VB> *>(raw);
        if (sl.bp.win == 3) backward_tile<false, false, SEG, VB, 3>(sl.bp, tile, sl.bsino, sl.bimg, sm);
        else backward_tile<false, false, SEG, VB, 0>(sl.bp, tile, sl.bsino, sl.bimg, sm);
    }
}

template <int SEG, int VB>
__global__ void __launch_bounds__(kBwdTile * kBwdTile, 4) k_backward_batch(const BatchArgs a)
{
    __shared__ __align__(16) unsigned char raw[tiled_smem_bytes<SEG, VB>()];
    __shared__ long long slot;
    for (;;) {
        const long long item = next_item(a.counter, &slot);
        if (item >= a.total) return;
        const int i = find_slot(a.prefix, a.nslices, item);
        const BatchSlice &sl = a.slices[a.order[i]];
        const int tile = (int)(item - a.prefix[i]);
        const bool fan = sl.bp.g.fan != 0;
        if (sl.tiled) {
            batch_tile<SEG, VB>(sl, tile, raw);
        } else {
            if (fan) backward_tile_direct<true>(sl.bp, tile, sl.bsino, sl.bimg);
            else backward_tile_direct<false>(sl.bp, tile, sl.bsino, sl.bimg);
        }
    }
}

// ------------------------------------------------- streaming backprojection
//
// A persistent backprojection whose inputs arrive while it runs: the host
// publishes slice i by setting ready[i] != 0 in host-mapped memory once its
// sinogram is on the device.  A block that takes a tile of slice i waits for
// that flag -- polling with __nanosleep -- for at most timeout_ns of
// %globaltimer time; past it, the slice is marked timed out (status[i] = 1),
// its remaining tiles are skipped by every block, and the host reports
// CTPRJ_ETIMEOUT.  No wait is unbounded and nothing traps, so the context stays
// usable after a timeout.

__device__ __forceinline__ unsigned long long global_ns()
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

template <int SEG, int VB>
__global__ void __launch_bounds__(kBwdTile * kBwdTile, 4)
k_backward_stream(const BatchArgs a, const volatile int *__restrict__ ready,
                  int *__restrict__ status, unsigned long long timeout_ns)
{
    __shared__ __align__(16) unsigned char raw[tiled_smem_bytes<SEG, VB>()];
    __shared__ long long slot;
    __shared__ int go;
    for (;;) {
        const long long item = next_item(a.counter, &slot);
        if (item >= a.total) return;
        const int i = find_slot(a.prefix, a.nslices, item);
        const int s = a.order[i];
        if (threadIdx.x == 0) {
            int ok = 0;
            if (((volatile int *)status)[s] == 0) {
                const unsigned long long t0 = global_ns();
                for (;;) {
                    if (ready[s]) { ok = 1; break; }
                    if (((volatile int *)status)[s] != 0) break;
                    if (global_ns() - t0 > timeout_ns) {
                        atomicExch(&status[s], 1);
                        break;
                    }
                    __nanosleep(1000);
                }
            }
            go = ok;
        }
        __syncthreads();
        if (!go) continue;
        __threadfence();   // the sinogram was published before the flag
        const BatchSlice &sl = a.slices[s];
        const int tile = (int)(item - a.prefix[i]);
        const bool fan = sl.bp.g.fan != 0;
        if (sl.tiled) {
            batch_tile<SEG, VB>(sl, tile, raw);
        } else {
            if (fan) backward_tile_direct<true>(sl.bp, tile, sl.bsino, sl.bimg);
            else backward_tile_direct<false>(sl.bp, tile, sl.bsino, sl.bimg);
        }
    }
}

int launch_backward_stream(const BatchArgs &a, int seg, int vb, int ctas, const int *ready,
                           int *status, unsigned long long timeout_ns, cudaStream_t s)
{
    if (seg <= 32 && vb == 16)
        k_backward_stream<32, 16><<<ctas, 256, 0, s>>>(a, ready, status, timeout_ns);
    else if (seg <= 32)
        k_backward_stream<32, 8><<<ctas, 256, 0, s>>>(a, ready, status, timeout_ns);
    else
        k_backward_stream<64, 8><<<ctas, 256, 0, s>>>(a, ready, status, timeout_ns);
    return cuda_error(cudaGetLastError(), "streaming backward launch");
}

int launch_quad_batch(const BatchArgs &a, cudaStream_t s)
{
    const long long blocks = a.ttotal < 65536 ? a.ttotal : 65536;
    k_quad_batch<<<(int)(blocks > 0 ? blocks : 1), dim3(32, 8), 0, s>>>(a);
    return cuda_error(cudaGetLastError(), "batched quad image launch");
}

int launch_forward_batch(const BatchArgs &a, int views, int ctas, cudaStream_t s)
{
    switch (views) {
    case 2: k_forward_batch<2><<<ctas, 64, 0, s>>>(a); break;
    case 8: k_forward_batch<8><<<ctas, 256, 0, s>>>(a); break;
    default: k_forward_batch<4><<<ctas, 128, 0, s>>>(a); break;
    }
    return cuda_error(cudaGetLastError(), "batched forward launch");
}

int launch_backward_batch(const BatchArgs &a, int seg, int vb, int ctas, cudaStream_t s)
{
    if (seg <= 32 && vb == 16) k_backward_batch<32, 16><<<ctas, 256, 0, s>>>(a);
    else if (seg <= 32) k_backward_batch<32, 8><<<ctas, 256, 0, s>>>(a);
    else k_backward_batch<64, 8><<<ctas, 256, 0, s>>>(a);
    return cuda_error(cudaGetLastError(), "batched backward launch");
}

// resident blocks per SM of a batched kernel: kind 0 forward (param = views),
// kind 1 backward (param = seg * 100 + vb)
int batch_max_ctas(int kind, int param, int *per_sm)
{
    cudaError_t e;
    if (kind == 0) {
        if (param == 2) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(per_sm, k_forward_batch<2>, 64, 0);
        else if (param == 8) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(per_sm, k_forward_batch<8>, 256, 0);
        else e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(per_sm, k_forward_batch<4>, 128, 0);
    } else {
        if (param == 3216) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(per_sm, k_backward_batch<32, 16>, 256, 0);
        else if (param == 3208) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(per_sm, k_backward_batch<32, 8>, 256, 0);
        else e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(per_sm, k_backward_batch<64, 8>, 256, 0);
    }
    return cuda_error(e, "occupancy query");
}

FwdParams make_fwd_params(const ctprj_plan *pl) { return fwd_params(pl); }
BwdParams make_bwd_params(const ctprj_plan *pl) { return bwd_params(pl, 0, 1.0f); }

}  // namespace ctprj

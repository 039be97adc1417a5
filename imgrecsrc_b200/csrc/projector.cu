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
//            mirrored pixels of a row come from four contiguous row segments:
//            rows y and -y of the image and of its transpose, which the plan
//            keeps in scratch so that every gather is coalesced along x.
//  backward  one thread per octant pixel 0 <= y <= x (pixel-driven,
//            prj/cpuPrj.c:46-317), looping over the base views and the
//            detectors under the pixel's shadow; each thread owns its eight
//            output pixels, so no atomics are needed.
//
// Precision: the weights are FP32 but each distance from a ray is evaluated in
// FP64 before rounding (x cos R + y sin R - offset cancels to O(1) from terms
// of O(n)); that keeps the projections within 1e-7..1e-6 of the FP64 oracle,
// where the reference's own FP32 build is 1.5e-5 off on signed inputs.
#include <cstdio>

#include "ctprj_internal.h"
#include "footprint.cuh"
#include "bhc_spline.cuh"

namespace ctprj {

constexpr int kFwdThreads = 128;
constexpr int kBwdTile = 16;   // 16 x 16 octant pixels per block

// --------------------------------------------------------------- transpose

__global__ void __launch_bounds__(256) k_transpose(const float *__restrict__ src,
                                                   float *__restrict__ dst, int n)
{
    __shared__ float tile[32][33];
    const int bx = blockIdx.x * 32, by = blockIdx.y * 32;
    for (int r = threadIdx.y; r < 32; r += 8) {
        const int row = by + r, col = bx + threadIdx.x;
        if (row < n && col < n) tile[r][threadIdx.x] = src[(size_t)row * n + col];
    }
    __syncthreads();
    for (int r = threadIdx.y; r < 32; r += 8) {
        const int row = bx + r, col = by + threadIdx.x;
        if (row < n && col < n) dst[(size_t)row * n + col] = tile[threadIdx.x][r];
    }
}

int launch_transpose(const float *src, float *dst, int n, cudaStream_t s)
{
    dim3 grid((n + 31) / 32, (n + 31) / 32), block(32, 8);
    k_transpose<<<grid, block, 0, s>>>(src, dst, n);
    return cuda_error(cudaGetLastError(), "transpose launch");
}

// ----------------------------------------------------------------- forward

// Polychromatic epilogue of one sinogram entry (bhc/poissLAlpha.m:2-13 per
// ray): s = Ts * proj, BL(s) and dBL/ds over the spectrum (FP64), and the
// Poisson term; keeps s, 1 - m/BL and (1 - m/BL) dBL/ds when asked.
__device__ __forceinline__ double bhc_entry(const BhcArgs &a, const double *tab,
                                            const double *Ie, float proj, size_t idx)
{
    const double s = a.Ts * (double)proj;
    const SplineEval e = b1_eval(s, tab, Ie, a.J);
    const double m = (double)__ldg(a.imea + idx);
    const double r = 1.0 - m / e.BL;
    if (a.w_out) {
        a.w_out[idx] = (float)(r * e.sBL);
        a.s_out[idx] = (float)s;
        a.r_out[idx] = (float)r;
    }
    return poisson_term(e.BL, m);
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

template <bool FAN, int MODE>
__global__ void __launch_bounds__(kFwdThreads)
k_forward(const FwdParams p, const float *__restrict__ img, const float *__restrict__ imgT,
          float *__restrict__ sino, unsigned long long *__restrict__ counter)
{
    const Geo &g = p.g;
    const int b = blockIdx.x;
    const int r = blockIdx.y * blockDim.x + threadIdx.x;
    double fsum = 0.0;            // polychromatic mode: this thread's Poisson terms
    const double *tab = nullptr, *Ie = nullptr;
    if constexpr (MODE == kModeBhc) {
        __shared__ double sm[kMaxJ * (kSplStride + 1)];
        for (int i = threadIdx.x; i < p.bhc.J * kSplStride; i += blockDim.x) sm[i] = p.bhc.tab[i];
        for (int i = threadIdx.x; i < p.bhc.J; i += blockDim.x) sm[kMaxJ * kSplStride + i] = p.bhc.Ie[i];
        __syncthreads();
        tab = sm;
        Ie = sm + kMaxJ * kSplStride;
    }
    // detector 0 of an even-width sinogram: no ray, zero projection
    if (MODE != kModeCount && p.zero_col0 && b == 0 && blockIdx.y == 0)
        for (int v = threadIdx.x; v < g.np; v += blockDim.x) {
            if constexpr (MODE == kModeBhc) fsum += bhc_entry(p.bhc, tab, Ie, 0.0f, (size_t)v * g.W);
            else sino[(size_t)v * g.W] = 0.0f;
        }

    if (r < p.nk) {
        const int k = p.k0 + r;
        const double cT = p.view[b].c, sT = p.view[b].s;
        const DetEntry de = p.det[k];
        const double hbw = 0.5 * g.beamWidth;
        const double tl = de.t - hbw, tr = de.t + hbw;

        // Ray direction (cos R, sin R), its offset from the isocentre, and the
        // pixel range of each row as xl(y) = Al - y Sl, xr(y) = Ar - y Sr: the
        // intersections of the two beam edges with the row's band
        // (prj/cpuPrj.c:365-369 parallel, :514-536 fan).
        double cR, sR, off, Al, Sl, Ar, Sr;
        float bwc = g.beamWidthF, kbw = 0.0f;
        if (FAN) {
            const double d = g.d;
            cR = de.cB * cT - de.sB * sT;
            sR = de.sB * cT + de.cB * sT;
            off = de.t * de.cB;   // d t / bq
            const double qxl = tl * cT + d * sT, qyl = -tl * sT + d * cT;
            const double qxr = tr * cT + d * sT, qyr = -tr * sT + d * cT;
            Al = (d * tl - (qxl > 0 ? 0.5 : -0.5) * qxl) / qyl;
            Sl = qxl / qyl;
            Ar = (d * tr + (qxr > 0 ? 0.5 : -0.5) * qxr) / qyr;
            Sr = qxr / qyr;
            // magnified beam width at pixel (x, y): bwc + (x sinT - y cosT) bwc / d
            const double bwcd = g.beamWidth * de.cB;
            bwc = (float)bwcd;
            kbw = (float)(bwcd / d);
        } else {
            cR = cT;
            sR = sT;
            off = de.t;
            Al = (tl - 0.5 * sT) / cT;
            Sl = sT / cT;
            Ar = (tr + 0.5 * sT) / cT;
            Sr = Sl;
        }
        const float Alf = (float)Al, Slf = (float)Sl, Arf = (float)Ar, Srf = (float)Sr;
        const float cRf = (float)cR, cTf = (float)cT, sTf = (float)sT;
        const float dbw = FAN ? sTf * kbw : 0.0f;
        const Footprint fp = make_footprint(cRf, (float)sR);

        const int N = g.n, half = g.half, h2 = g.h2;
        float S[8];
#pragma unroll
        for (int j = 0; j < 8; ++j) S[j] = 0.0f;
        unsigned long long nz = 0;

        for (int y = half; y >= -half; --y) {
            const float yf = (float)y;
            const float xl = fmaf(-yf, Slf, Alf), xr = fmaf(-yf, Srf, Arf);
            int x0 = (int)roundf(fmaxf(xl, (float)(-half - 1)));
            int x1 = (int)roundf(fminf(xr, (float)(half + 1)));
            x0 = max(x0, -half);
            x1 = min(x1, half);
            if (x0 > x1) continue;
            // distance of pixel (x0, y) from the ray, in FP64 then rounded
            const float r0 = (float)fma((double)x0, cR, fma((double)y, sR, -off));
            const float bw0 = FAN ? fmaf(fmaf((float)x0, sTf, -yf * cTf), kbw, bwc) : g.beamWidthF;
            // rows y and -y of the image and of its transpose, centred on x = 0:
            // a0[x] = I(x, y), a0[-x] = I(-x, y), a1[+-x] = I(+-x, -y),
            // t0[x] = I(y, x), t0[-x] = I(y, -x), t1[+-x] = I(-y, +-x)
            const float *a0 = img + (size_t)(y + h2) * N + h2;
            const float *a1 = img + (size_t)(h2 - y) * N + h2;
            const float *t0 = imgT + (size_t)(y + h2) * N + h2;
            const float *t1 = imgT + (size_t)(h2 - y) * N + h2;
            for (int x = x0; x <= x1; ++x) {
                const float jf = (float)(x - x0);
                const float dist = fmaf(jf, cRf, r0);
                const float bw = FAN ? fmaf(jf, dbw, bw0) : bw0;
                const float w = footprint_weight(dist, bw, fp);
                if (MODE == kModeCount) {
                    nz += (w != 0.0f);
                    continue;
                }
                S[0] = fmaf(w, __ldg(a0 + x), S[0]);
                S[6] = fmaf(w, __ldg(a0 - x), S[6]);
                S[4] = fmaf(w, __ldg(a1 + x), S[4]);
                S[2] = fmaf(w, __ldg(a1 - x), S[2]);
                S[5] = fmaf(w, __ldg(t0 + x), S[5]);
                S[3] = fmaf(w, __ldg(t0 - x), S[3]);
                S[1] = fmaf(w, __ldg(t1 + x), S[1]);
                S[7] = fmaf(w, __ldg(t1 - x), S[7]);
            }
        }

        // Scatter to the eight symmetric views (prj/cpuPrj.c:577-615); parallel
        // beam also writes the point-reflected detector of the same view
        // (prj/cpuPrj.c:403-460), which image j ^ 2 holds.  Where the two
        // coincide (the central detector) the second write is the one kept.
        const int pC = g.pC;
        unsigned long long entries = 0;
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
                    fsum += bhc_entry(p.bhc, tab, Ie, S[j] / g.effRate, row + det);
                } else if (det2 != det) {
                    fsum += bhc_entry(p.bhc, tab, Ie, S[j] / g.effRate, row + det);
                    fsum += bhc_entry(p.bhc, tab, Ie, S[j ^ 2] / g.effRate, row + det2);
                } else {
                    fsum += bhc_entry(p.bhc, tab, Ie, S[j ^ 2] / g.effRate, row + det);
                }
            } else {
                sino[row + det] = S[j] / g.effRate;
                if (!FAN) sino[row + det2] = S[j ^ 2] / g.effRate;
            }
        }
        if (MODE == kModeCount && nz * entries) atomicAdd(counter, nz * entries);
    }

    if constexpr (MODE == kModeBhc) {
        __shared__ double red[kFwdThreads / 32];
        const double t = block_sum(fsum, red);
        if (threadIdx.x == 0) p.bhc.part[(size_t)blockIdx.y * gridDim.x + blockIdx.x] = t;
    }
}

static FwdParams fwd_params(const ctprj_plan *pl)
{
    FwdParams p;
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
    return dim3(pl->nb, (pl->nk + kFwdThreads - 1) / kFwdThreads);
}

int forward_blocks(const ctprj_plan *pl)
{
    const dim3 g = fwd_grid(pl);
    return (int)(g.x * g.y);
}

int launch_forward(const ctprj_plan *pl, const float *img, const float *imgT, float *sino,
                   unsigned long long *counter, cudaStream_t s)
{
    const FwdParams p = fwd_params(pl);
    const dim3 grid = fwd_grid(pl), block(kFwdThreads);
    const bool fan = pl->g.fan != 0;
    if (counter) {
        if (fan) k_forward<true, kModeCount><<<grid, block, 0, s>>>(p, img, imgT, sino, counter);
        else k_forward<false, kModeCount><<<grid, block, 0, s>>>(p, img, imgT, sino, counter);
    } else {
        if (fan) k_forward<true, kModePlain><<<grid, block, 0, s>>>(p, img, imgT, sino, counter);
        else k_forward<false, kModePlain><<<grid, block, 0, s>>>(p, img, imgT, sino, counter);
    }
    return cuda_error(cudaGetLastError(), "forward launch");
}

int launch_forward_bhc(const ctprj_plan *pl, const float *img, const float *imgT,
                       const BhcArgs &a, int *nparts, cudaStream_t s)
{
    FwdParams p = fwd_params(pl);
    p.bhc = a;
    const dim3 grid = fwd_grid(pl), block(kFwdThreads);
    if (pl->g.fan) k_forward<true, kModeBhc><<<grid, block, 0, s>>>(p, img, imgT, nullptr, nullptr);
    else k_forward<false, kModeBhc><<<grid, block, 0, s>>>(p, img, imgT, nullptr, nullptr);
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
    // triangular tile number -> tile (tx, ty), ty <= tx
    const int tile = blockIdx.x;
    int tx = (int)((sqrtf(8.0f * (float)tile + 1.0f) - 1.0f) * 0.5f);
    while ((tx + 1) * (tx + 2) / 2 <= tile) ++tx;
    while (tx * (tx + 1) / 2 > tile) --tx;
    const int ty = tile - tx * (tx + 1) / 2;
    const int x = tx * kBwdTile + (int)(threadIdx.x % kBwdTile);
    const int y = ty * kBwdTile + (int)(threadIdx.x / kBwdTile);
    if (x > g.half || y > x) return;

    const int nimg = (y == 0 || y == x) ? 4 : 8;
    const double xd = x, yd = y;
    const float xf = (float)x, yf = (float)y;
    const int dmax = (g.W - 1) / 2, pC = g.pC;
    const float dSf = (float)g.dSize;
    float S[8];
#pragma unroll
    for (int j = 0; j < 8; ++j) S[j] = 0.0f;
    unsigned long long nz = 0;

    for (int i = 0; i < p.nv; ++i) {
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

    if (COUNT) {
        if (nz) atomicAdd(counter, nz);
        return;
    }
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

int launch_backward(const ctprj_plan *pl, const float *sino, float *img, int fbp,
                    unsigned long long *counter, cudaStream_t s, float scale)
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
    dim3 grid(T * (T + 1) / 2), block(kBwdTile * kBwdTile);
    const bool fan = pl->g.fan != 0;
    if (counter) {
        if (fan) k_backward<true, true, false><<<grid, block, 0, s>>>(p, sino, img, counter);
        else k_backward<false, true, false><<<grid, block, 0, s>>>(p, sino, img, counter);
    } else if (fbp) {
        if (fan) k_backward<true, false, true><<<grid, block, 0, s>>>(p, sino, img, counter);
        else k_backward<false, false, true><<<grid, block, 0, s>>>(p, sino, img, counter);
    } else {
        if (fan) k_backward<true, false, false><<<grid, block, 0, s>>>(p, sino, img, counter);
        else k_backward<false, false, false><<<grid, block, 0, s>>>(p, sino, img, counter);
    }
    return cuda_error(cudaGetLastError(), "backward launch");
}

}  // namespace ctprj

"""FP64 restatement of the alternating beam-hardening reconstruction loop --
TEST INFRASTRUCTURE ONLY (the oracle; never imported by the product).

The same algorithm as the engine's ctprj_bhc_reconstruct, step for step, in
double precision over the FP64 projector restatement (oracle.forward /
oracle.backward):

* density step: the reference's NPG class (npg/NPG.m:45-146) or PG class
  (npg/PG.m:41-124) with the projection on x >= 0 as the proximal map, the
  majorisation test of utils/Utils.m:470-480, and the initial step rules of
  npg/Methods.m:98-124 ('fixed', 'bb', 'hessian'); with proximal 'tviso' /
  'tvl1' the proximal map is the TV denoising of utils/TV.m (tv_oracle) and the
  objective carries u TV(x);
* spectrum step: Newton steps on Ie >= 0 for the objective of bhc/poissLI.m
  (Gauss-Newton curvature for bhc/gaussLI.m), each minimising the quadratic
  model over Ie >= 0 with a primal active-set method on a diagonally lifted,
  Jacobi-scaled Hessian (bhc/ActiveSet.m:62-76 lifts its eigenvalues the same
  way), then backtracking by 0.8 (bhc/ActiveSet.m stepShrnk) to
  f <= f0 + 1e-4 g.d;
* alternation as bhc/beamhardenSpline.m:380-470: one density step, then the
  spectrum step, whose f becomes the cost the next density step compares to;
  optionally the stopping rule of :563-566 on the relative density change.
"""
import math

import numpy as np

from . import bhc_oracle as BO
from . import tv_oracle as TV
from . import wavelet_oracle as WV


def _cholesky_lifted(M, lift):
    """Lower Cholesky factor of M + lift I, or None when a pivot is not above
    1e-14 (1 + lift)."""
    n = M.shape[0]
    A = M + lift * np.eye(n)
    L = np.zeros_like(A)
    for k in range(n):
        d = A[k, k] - L[k, :k] @ L[k, :k]
        if not d > 1e-14 * (1.0 + lift):
            return None
        L[k, k] = math.sqrt(d)
        for r in range(k + 1, n):
            L[r, k] = (A[r, k] - L[r, :k] @ L[k, :k]) / L[k, k]
    return L


def _factor(M):
    lift = 0.0
    for _ in range(40):
        L = _cholesky_lifted(M, lift)
        if L is not None:
            return L, lift
        lift = 1e-14 if lift == 0.0 else lift * 10.0
    return None, lift


def qp_direction(H, g, Ie):
    """Newton direction of the spectrum step: y minimising 1/2 y'Hy + c'y,
    c = g - H Ie, over y >= 0 (H lifted once to positive definite), minus Ie."""
    H = np.array(H, np.float64)
    J = g.size
    fixed = ~(np.diag(H) > 0)
    dg = np.where(fixed, 1.0, np.sqrt(np.where(fixed, 1.0, np.diag(H))))
    idx = np.where(~fixed)[0]
    if idx.size:
        L, lift = _factor(H[np.ix_(idx, idx)] / np.outer(dg[idx], dg[idx]))
        if L is None:
            return np.zeros(J)
        H[idx, idx] *= 1.0 + lift
    c = g - H @ Ie
    y = np.where(fixed, Ie, np.maximum(Ie, 0.0))
    W = (~fixed) & ~(Ie > 0)
    for _ in range(8 * J + 16):
        F = (~W) & (~fixed)
        idx = np.where(F)[0]
        z = y.copy()
        if idx.size:
            L, _ = _factor(H[np.ix_(idx, idx)] / np.outer(dg[idx], dg[idx]))
            if L is None:
                break
            w = np.linalg.solve(L.T, np.linalg.solve(L, -c[idx] / dg[idx]))
            z[idx] = w / dg[idx]
        p = np.where(F, z - y, 0.0)
        ratio = np.full(J, np.inf)
        neg = F & (p < 0)
        ratio[neg] = -y[neg] / p[neg]
        j = int(np.argmin(ratio))
        if ratio[j] >= 1.0:
            y = np.where(F, z, y)
            Hy = H @ y
            lam = Hy + c
            cand = W & (lam < -1e-13 * (np.abs(c) + np.abs(Hy)))
            if not cand.any():
                break
            W[int(np.argmin(np.where(cand, lam, np.inf)))] = False
        else:
            y = np.where(F, y + ratio[j] * p, y)
            y[j] = 0.0
            W[j] = True
    return y - Ie


def _spectrum_objective(noise, A, m):
    if noise == "poisson":
        return lambda I: BO.poiss_ie(m, A, I)

    def gauss_newton(I):
        Ir = A @ I
        err = np.log(Ir / m)
        return 0.5 * err @ err, A.T @ (err / Ir), A.T @ (A * (1.0 / Ir ** 2)[:, None])
    return gauss_newton


def spectrum_steps(A, m, Ie, newton_steps, noise="poisson"):
    """At most newton_steps Newton steps; returns (Ie, f at Ie, steps taken)."""
    obj = _spectrum_objective(noise, A, np.asarray(m, np.float64).ravel())
    Ie = np.asarray(Ie, np.float64).copy()
    fcur, done = None, 0
    with np.errstate(all="ignore"):
        for _ in range(newton_steps):
            f, g, H = obj(Ie)
            fcur = f
            d = qp_direction(H, g, Ie)
            step, accepted, converged = 1.0, False, False
            for ls in range(40):
                trial = np.maximum(0.0, Ie + step * d)
                gd = g @ (trial - Ie)
                if ls == 0 and not gd < -1e-14 * abs(fcur):
                    converged = True
                    break
                fn = obj(trial)[0]
                if fn <= fcur + 1e-4 * gd:
                    Ie, fcur, accepted = trial, fn, True
                    break
                step *= 0.8
            if not accepted or converged:
                break
            done += 1
        if fcur is None:
            fcur = obj(Ie)[0]
    return Ie, fcur, done


class _Density:
    """f and its gradient in the density for fixed Ie (bhc/poissLAlpha.m,
    bhc/gaussLAlpha.m) over the FP64 projector."""

    def __init__(self, forward, backward, k, Ts, m, noise):
        self.fw, self.bw, self.k, self.Ts = forward, backward, k, Ts
        self.m = np.asarray(m, np.float64).ravel()
        self.noise = noise

    def s(self, x):
        return self.Ts * self.fw(x).ravel()

    def f(self, x, Ie, grad=False):
        s = self.s(x)
        BL, sBL, _ = BO.b1_iout(self.k, s, Ie)
        with np.errstate(divide="ignore", invalid="ignore"):
            if self.noise == "poisson":
                f = BO.poisson_terms(BL, self.m).sum()
                r = 1.0 - self.m / BL
            else:
                err = np.log(BL / self.m)
                f = 0.5 * err @ err
                r = err / BL
        if not grad:
            return f
        return f, self.Ts * self.bw(r * sBL).reshape(x.shape)

    def hessian_weight(self, x, Ie):
        w = BO.poiss_hessian_weight if self.noise == "poisson" else BO.gauss_hessian_weight
        return w(self.m, Ie, self.s(x), self.k)


def reconstruct(forward, backward, k, Ts, x, Ie, imea, iterations, x_step=1.0, newton_steps=2,
                method="npg", init_step="fixed", noise="poisson", skip_spectrum=False, thresh=0.0,
                min_iterations=0, proximal="nonneg", u=0.0, max_inner=100, admm_tol=1e-2, restart=True,
                adaptive_step=True, cumu_tol=4, wvlt_h=None, wvlt_levels=6, mask=None, wvlt_mask=None,
                pre_steps=2):
    """The alternating loop; forward(x) -> sinogram and backward(sino) -> image
    are FP64 projector callables.  Returns (x, Ie, stats) with stats holding
    the cost and accepted density step of every iteration.

    proximal "tviso" / "tvl1" regularises the density with u TV(x): the
    density step's proximal map becomes TV.denoise (utils/TV.m:56-80, the
    FGP of tv_oracle.tv_denoise with lambda = u/t, bounds [0, inf),
    epsilon = admmTol * difAlpha, maxInnerItr iterations), the objective
    f + u TV, and a rejected step is retried with admmTol / 10 (down to 1e-6)
    or, when the inner iteration ran out, maxInnerItr * 10 (up to 1000) before
    x is kept (npg/NPG.m:99-134, npg/PG.m:97-121).  restart, adaptive_step,
    cumu_tol and admm_tol are the reference's opt.restart, opt.adaptiveStep,
    opt.cumuTol and opt.admmTol (bhc/beamhardenSpline.m:277-294).  proximal
    "wvltADMM" (the reference's default) regularises with u |Psit(x)|_1: the
    proximal map is admm(Psi, Psit, xbar - g/t, u/t, admmTol * difAlpha,
    maxInnerItr, false, x) (npg/admm.m, wavelet_oracle.admm) with the wavelet
    of scaling filter wvlt_h (default daubcqf(2)) and wvlt_levels levels.
    mask is opt.mask: the density is the masked pixel vector (held here as the
    full image with zeros outside), so gradients are gathered on the mask and
    TV.denoise scatters, denoises and gathers (utils/TV.m:56-80); wvlt_mask is
    maskk (default: utils/wvltMask.m of the mask)."""
    dens = _Density(forward, backward, k, Ts, imea, noise)
    x = np.maximum(np.asarray(x, np.float64), 0.0)     # alpha = max(alpha, 0): :232, :236
    pm = 1.0 if mask is None else (np.asarray(mask) != 0).astype(np.float64).reshape(x.shape)
    x = x * pm
    grad_of = lambda xx: (lambda fg: (fg[0], fg[1] * pm))(dens.f(xx, Ie, grad=True))
    Ie = np.asarray(Ie, np.float64).copy()
    t = 1.0 / (x_step if x_step > 0 else 1.0)
    if init_step != "fixed":
        f0, g = grad_of(x)
        gg = float((g * g).sum())
        if init_step == "hessian":
            y = Ts * forward(g).ravel()
            t = abs(float(dens.hessian_weight(x, Ie) @ (y * y))) / gg
        else:
            xx = float((x * x).sum())
            dn = 1e-3 * math.sqrt(xx) if xx > 0 else 1e-3
            scale = dn / math.sqrt(gg)
            _, g2 = grad_of(x - scale * g)
            t = abs(float(((g - g2) * g).sum()) * scale) / (scale * scale * gg)
        if math.isnan(t):
            t = 1.0
        if t == 0.0:
            t = np.finfo(np.float64).eps
    pg = method == "pg"
    wv = proximal.lower() == "wvltadmm"
    tv = proximal in ("tviso", "tvl1")
    reg = tv or wv
    tvkind = "iso" if proximal == "tviso" else "l1"
    shape = x.shape if x.ndim == 2 else (int(round(math.sqrt(x.size))),) * 2
    wh = WV.daubcqf(2) if wvlt_h is None else np.asarray(wvlt_h, np.float64)
    if wv:
        if wvlt_mask is None and mask is not None:
            wvlt_mask = WV.wvlt_mask(np.asarray(mask).reshape(shape), wh, wvlt_levels)
        tlv = lambda v: WV.l1_penalty(v.reshape(shape), wh, wvlt_levels, wvlt_mask)
    else:
        tlv = lambda v: TV.tlv(v.reshape(shape), tvkind) if tv else 0.0
    dif_alpha, pen = 1.0, 0.0
    inner = 0
    theta, cost, p, cumu = 0.0, math.inf, 0, 0
    xprev = x.copy()
    costs, steps, changes = [], [], []
    conv, converged = 0, False
    inner_total, retries = 0, 0

    def retry():
        nonlocal admm_tol, max_inner, retries
        if inner < max_inner and admm_tol > 1e-6:
            admm_tol /= 10.0
        elif inner >= max_inner and max_inner < 1000:
            max_inner *= 10
        else:
            return False
        retries += 1
        return True

    max_pass = 12 if reg else 3
    for it in range(iterations):
        moved = False
        for pass_ in range(max_pass):
            last = pass_ == max_pass - 1
            p += 1
            theta1 = (1.0 + math.sqrt(1.0 + 4.0 * theta * theta)) / 2.0
            coef = 0.0 if pg else (theta - 1.0) / theta1
            xbar = np.maximum(0.0, x + coef * (x - xprev))
            mom = float(np.abs(xbar - x).sum())
            f0, g = grad_of(xbar)
            ppp, good, inc, good_mm = 0, True, False, True
            if adaptive_step and cumu >= cumu_tol:
                t *= 0.5
                cumu, inc = 0, True
            while True:
                ppp += 1
                if reg:
                    v = (xbar - g / t).reshape(shape)
                    if tv:
                        xn, inner = TV.tv_denoise(v, u / t, 0.0, math.inf, tvkind, max_inner,
                                                  admm_tol * dif_alpha)
                    else:
                        xn, inner = WV.admm(v, u / t, wh, wvlt_levels, rel_tol=admm_tol * dif_alpha,
                                            max_itr=max_inner, init=x.reshape(shape),
                                            mask=None if mask is None else pm.reshape(shape), maskk=wvlt_mask)
                    xn = xn.reshape(xbar.shape) * pm
                    inner_total += inner
                else:
                    xn = np.maximum(0.0, xbar - g / t)
                dx = xn - xbar
                nc = dens.f(xn, Ie)
                if nc - f0 <= float((g * dx).sum()) + 0.5 * t * float((dx * dx).sum()):
                    if p <= pre_steps and ppp < 18 and good:
                        t *= 0.5
                        continue
                    break
                if ppp <= 20:
                    t /= 0.5
                    good = False
                    if inc:
                        cumu_tol += 4
                        inc = False
                else:
                    good_mm = False
                    break
            pen = u * tlv(xn)
            new_obj = nc + pen
            moved = True
            if pg:
                if not good_mm or new_obj > cost:
                    if reg and not last and retry():
                        continue
                    moved = False
            elif new_obj > cost:
                if good_mm and mom != 0.0 and restart and not last:
                    theta = 1.0
                    continue
                if not good_mm or f0 + u * tlv(xbar) < new_obj:
                    if not good_mm:
                        theta = 1.0
                    if reg and not last and retry():
                        continue
                    moved = False
            if not moved:
                new_obj = cost
            theta = theta1
            xprev = x
            if moved:
                x = xn
            if reg:
                dif_alpha = float(np.linalg.norm(xprev - x)) / max(float(np.linalg.norm(x)), 1e-10)
            cumu = cumu + 1 if ppp == 1 and adaptive_step else 0
            break
        cost = new_obj
        steps.append(1.0 / t if moved else 0.0)
        if not skip_spectrum:
            A, _, _ = BO.b1_basis(k, dens.s(x), derivs=0)
            Ie, cost, _ = spectrum_steps(A, imea, Ie, newton_steps, noise)
            # alphaStep.cost = IeStep.cost + u fVal(3) (bhc/beamhardenSpline.m:460): the
            # penalty of the last candidate, also when it was not accepted
            cost += pen
        costs.append(cost)
        # relativeDif(x_new, x) and the stopping rule of bhc/beamhardenSpline.m:563-566
        change = float(np.linalg.norm(x - xprev)) / max(float(np.linalg.norm(xprev)), 1e-10)
        changes.append(change)
        if thresh > 0 and it > 0 and change <= thresh:
            conv += 1
        if conv > 2 and it + 1 > min_iterations:
            converged = True
            break
    return x, Ie, {"cost": costs, "x_step": steps, "final_x_step": 1.0 / t, "x_change": changes,
                   "converged": converged, "inner_iterations": inner_total, "prox_retries": retries,
                   "penalty": pen}

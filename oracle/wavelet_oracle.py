"""FP64 restatement of the wavelet regulariser of the reference's density step
-- TEST INFRASTRUCTURE ONLY (the oracle; never imported by the product).

The reference's default proximal map (opt.proximal = 'wvltADMM',
bhc/beamhardenSpline.m:36, :205-209) solves

    min_alpha  1/2 ||alpha - a||^2 + I(alpha >= 0) + u ||Psit(alpha)||_1

by ADMM (npg/admm.m), with Psi / Psit the inverse / forward orthogonal
discrete wavelet transforms of the vendored Rice Wavelet Toolbox
(utils/Utils.m:445-469 getPsiPsit: midwt / mdwt with daubcqf(daub), dwt_L
levels; the BHC examples use daub = 2, dwt_L = 6, bhc/doBHC.m:33).  Restated
here:

* daubcqf: the Daubechies minimum-phase scaling filter (rwt/daubcqf.m, after
  I. Daubechies, "Orthonormal bases of compactly supported wavelets", CPAM
  41, 1988): the polynomial construction, the K-1 roots of smallest modulus
  (MATLAB's sort orders complex roots by modulus, then angle), normalised to
  sum sqrt(2);
* mdwt / midwt: the periodic 2-D transform of rwt/mdwt_r.c and
  rwt/midwt_r.c, level by level on the top-left block, rows then columns,
  lowpass outputs first: lo[k] = sum_j h[j] x[(2k+j) mod N],
  hi[k] = sum_j (-1)^j h[lh-1-j] x[(2k+j) mod N]; the inverse is the exact
  adjoint (the transform is orthogonal);
* admm: npg/admm.m step for step (scaling by ||a||, nu = 0, rho = 1, the
  rho adaptation every 20+ iterations, the stopping rule on the primal
  change and residual, the final alpha from the last s and nu).

Arrays are MATLAB matrices as numpy arrays indexed [row, column].  Pinned
against the reference's own rwt cores compiled into oracle/_ref (``ref_mdwt``
/ ``ref_midwt``) and against the worked examples in rwt's help texts.
"""
import ctypes
import math
import os

import numpy as np

from . import REFDIR


def daubcqf(N):
    """Minimum-phase Daubechies scaling filter of even length N (rwt/daubcqf.m)."""
    if N % 2:
        raise ValueError("no Daubechies filter of odd length")
    K = N // 2
    a = 1.0
    h0 = np.array([1.0, 1.0])
    p = np.array([1.0])
    q = np.array([1.0])
    for j in range(1, K):
        a = -a * 0.25 * (j + K - 1) / j
        h0 = np.concatenate([[0.0], h0]) + np.concatenate([h0, [0.0]])
        for _ in range(2):
            p = np.concatenate([[0.0], -p]) + np.concatenate([p, [0.0]])
        q = np.concatenate([[0.0], q, [0.0]]) + a * p
    if K > 1:
        r = np.roots(q)
        r = np.array(sorted(r, key=lambda z: (abs(z), np.angle(z))))
        h0 = np.convolve(h0, np.real(np.poly(r[:K - 1])))
    return math.sqrt(2.0) * h0 / h0.sum()


def _highpass(h):
    lh = len(h)
    return np.array([(-1.0) ** j * h[lh - 1 - j] for j in range(lh)])


def _analysis_1d(x, h):
    """(lo, hi) of one level along the last axis, periodic."""
    N = x.shape[-1]
    g = _highpass(h)
    lo = np.zeros(x.shape[:-1] + (N // 2,))
    hi = np.zeros_like(lo)
    for j in range(len(h)):
        idx = (2 * np.arange(N // 2) + j) % N
        lo += h[j] * x[..., idx]
        hi += g[j] * x[..., idx]
    return lo, hi


def _synthesis_1d(lo, hi, h):
    """Adjoint (= inverse) of _analysis_1d along the last axis."""
    M = lo.shape[-1]
    N = 2 * M
    g = _highpass(h)
    lo2 = lo.reshape(-1, M)
    hi2 = hi.reshape(-1, M)
    x = np.zeros((lo2.shape[0], N))
    for j in range(len(h)):
        idx = (2 * np.arange(M) + j) % N
        np.add.at(x, (slice(None), idx), h[j] * lo2 + g[j] * hi2)
    return x.reshape(lo.shape[:-1] + (N,))


def _levels_ok(shape, L):
    m, n = shape
    if (m > 1 and m % (1 << L)) or n % (1 << L):
        raise ValueError("dimensions must be divisible by 2^L")


def mdwt(x, h, L):
    """y = mdwt(x, h, L) for a 2-D array (or a 1-row array: the 1-D transform)."""
    x = np.asarray(x, np.float64)
    y = x.copy()
    if y.ndim == 1:
        y = y[None, :]
    _levels_ok(y.shape, L)
    m, n = y.shape
    for lev in range(L):
        am = m if m == 1 else m >> lev
        an = n >> lev
        blk = y[:am, :an].copy()
        lo, hi = _analysis_1d(blk, h)                      # along rows (the column index)
        blk = np.concatenate([lo, hi], axis=1)
        if m > 1:
            lo, hi = _analysis_1d(blk.T, h)                # along columns
            blk = np.concatenate([lo, hi], axis=1).T
        y[:am, :an] = blk
    return y[0] if np.ndim(x) == 1 else y


def midwt(y, h, L):
    """x = midwt(y, h, L), the inverse of mdwt."""
    y = np.asarray(y, np.float64)
    x = y.copy()
    if x.ndim == 1:
        x = x[None, :]
    _levels_ok(x.shape, L)
    m, n = x.shape
    for lev in range(L - 1, -1, -1):
        am = m if m == 1 else m >> lev
        an = n >> lev
        blk = x[:am, :an].copy()
        if m > 1:
            t = blk.T
            blk = _synthesis_1d(t[:, :am // 2], t[:, am // 2:], h).T
        blk = _synthesis_1d(blk[:, :an // 2], blk[:, an // 2:], h)
        x[:am, :an] = blk
    return x[0] if np.ndim(y) == 1 else x


def soft_thresh(x, thresh):
    """Utils.softThresh (utils/Utils.m:13-20)."""
    t = abs(thresh)
    return np.where(x > t, x - t, np.where(x < -t, x + t, 0.0))


def admm(a, u, h, L, rel_tol=1e-6, max_itr=1000, init=None, mask=None, maskk=None):
    """[alpha, pppp] = admm(Psi, Psit, a, u, relativeTol, maxItr, false, init)
    (npg/admm.m) with Psi = midwt(., h, L), Psit = mdwt(., h, L), or with
    masks the operators of utils/Utils.m:445-469 getPsiPsit:
    Psi = mask.a(midwt(maskk.b(.))), Psit = maskk.a(mdwt(mask.b(.))), the
    masked vectors held as full arrays with zeros outside.  Returns (alpha,
    iterations)."""
    a = np.asarray(a, np.float64)
    pm = 1.0 if mask is None else (np.asarray(mask) != 0).astype(np.float64)
    cm = 1.0 if maskk is None else (np.asarray(maskk) != 0).astype(np.float64)
    Psi = lambda s: midwt(s * cm, h, L) * pm
    Psit = lambda x: mdwt(x * pm, h, L) * cm
    init = a if init is None else np.asarray(init, np.float64)
    rel_tol = min(1e-3, rel_tol)
    scale = float(np.linalg.norm(a))
    if scale == 0.0:
        return np.zeros_like(a), 0
    init, a, u = init / scale, a / scale, u / scale
    nu = 0.0
    rho = 1.0
    cnt = 0
    s = Psit(init)
    pre_s = s
    pppp = 0
    while True:
        pppp += 1
        cnt += 1
        alpha = np.maximum((a + rho * Psi(s + nu)) / (1.0 + rho), 0.0)
        psit_alpha = Psit(alpha)
        s = soft_thresh(psit_alpha - nu, u / rho)
        nu = nu + s - psit_alpha
        dif_s = float(np.linalg.norm(s - pre_s))
        pre_s = s
        residual = float(np.linalg.norm(s - psit_alpha))
        if pppp > max_itr:
            break
        if dif_s <= rel_tol and residual <= rel_tol:
            break
        if cnt > 20:
            if dif_s > 10 * residual:
                rho, nu, cnt = rho / 2, nu * 2, 0
            elif dif_s < residual / 10:
                rho, nu, cnt = rho * 2, nu / 2, 0
    alpha = np.maximum((a + rho * Psi(s + nu)) / (1.0 + rho), 0.0) * scale
    return alpha, pppp


def l1_penalty(x, h, L, maskk=None):
    """pNorm(Psit(x), 1): the 'wvltADMM' penalty (bhc/beamhardenSpline.m:208),
    over the coefficients of maskk when given."""
    y = np.abs(mdwt(x, h, L))
    if maskk is not None:
        y = y * (np.asarray(maskk) != 0)
    return float(y.sum())


def circular_mask(n, m=None):
    """Utils.getCircularMask(n, m) (utils/Utils.m:438-444): the pixels whose
    0-based coordinates lie closer than m/2 - 1 to (n/2, n/2)."""
    m = n if m is None else m
    x, y = np.meshgrid(np.arange(n), np.arange(n))
    return np.sqrt((x - n / 2) ** 2 + (y - n / 2) ** 2) < (m / 2 - 1)


def wvlt_mask(mask, h, L):
    """maskk = wvltMask(Mask, dwt_L, daub) (utils/wvltMask.m), as there: the
    union over the mask's pixels e_i of Wt(e_i) != 0."""
    mask = np.asarray(mask) != 0
    maskk = np.zeros(mask.shape, bool)
    test = np.zeros(mask.shape)
    for idx in zip(*np.nonzero(mask)):
        test[idx] = 1.0
        maskk |= mdwt(test, h, L) != 0
        test[idx] = 0.0
    return maskk


def admm_objective(alpha, a, u, h, L):
    return 0.5 * float(((alpha - a) ** 2).sum()) + u * l1_penalty(alpha, h, L)


# ---- the reference's own rwt cores (oracle/_ref/libref_rwt.so) ------------
_rwt = None


def ref_available():
    return os.path.exists(os.path.join(REFDIR, "libref_rwt.so"))


def _ref_lib():
    global _rwt
    if _rwt is None:
        lib = ctypes.CDLL(os.path.join(REFDIR, "libref_rwt.so"))
        sig = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_int, ctypes.c_int,
               ctypes.c_void_p]
        for f in (lib.MDWT, lib.MIDWT):   # rwt/mdwt_r.c, rwt/midwt_r.c: (x, m, n, h, lh, L, y)
            f.argtypes = sig
            f.restype = None
        _rwt = lib
    return _rwt


def _ref_call(fname, x, h, L):
    x = np.asarray(x, np.float64)
    one_d = x.ndim == 1
    X = x[:, None] if one_d else x                    # MATLAB column vector: m = N, n = 1
    m, n = X.shape
    xin = np.asfortranarray(X).copy(order="F")
    yout = np.zeros((m, n), order="F")
    hh = np.ascontiguousarray(h, np.float64)
    getattr(_ref_lib(), fname)(xin.ctypes.data, m, n, hh.ctypes.data, len(hh), int(L), yout.ctypes.data)
    return yout[:, 0].copy() if one_d else np.ascontiguousarray(yout)


def ref_mdwt(x, h, L):
    """mdwt through the reference's compiled MDWT (column-major, as MATLAB)."""
    return _ref_call("MDWT", x, h, L)


def ref_midwt(y, h, L):
    """midwt through the reference's compiled MIDWT.  MIDWT(x, m, n, h, lh,
    L, y) writes the signal into its first argument from the coefficients in
    its last."""
    y = np.asarray(y, np.float64)
    one_d = y.ndim == 1
    Y = y[:, None] if one_d else y
    m, n = Y.shape
    xout = np.zeros((m, n), order="F")
    yin = np.asfortranarray(Y).copy(order="F")
    hh = np.ascontiguousarray(h, np.float64)
    _ref_lib().MIDWT(xout.ctypes.data, m, n, hh.ctypes.data, len(hh), int(L), yin.ctypes.data)
    return xout[:, 0].copy() if one_d else np.ascontiguousarray(xout)

"""FP64 restatement of the total-variation proximal map of the reference's
density step -- TEST INFRASTRUCTURE ONLY (the oracle; never imported by the
product).

The reference regularises the density with u TV(x) (proximal options 'tviso'
and 'tvl1' of bhc/beamhardenSpline.m:199-224); its NPG/PG proximal map is
TV.denoise (utils/TV.m:56-80), which calls denoise_bound_mod
(utils/denoise_bound_mod.m): Beck and Teboulle's fast gradient projection
(FGP) on the dual of

    min_X  ||X - Xobs||^2 + 2 lambda TV(X)   subject to  l <= X <= u,

with the difference operators of utils/Ltrans.m and utils/Lforward.m and the
TV of utils/tlv.m.  Restated here from the published algorithm (A. Beck,
M. Teboulle, "Fast gradient-based algorithms for constrained total variation
image denoising and deblurring problems", IEEE TIP 18(11), 2009) with the
reference's stopping rule (five consecutive relative changes below epsilon,
or MAXITER) and restart (t reset when the dual objective rises).  Rows are
the first index, as in MATLAB.
"""
import math

import numpy as np


def ltrans(X):
    """The transposed difference operator: P1 = X[i] - X[i+1] down the rows,
    P2 = X[:, j] - X[:, j+1] along them."""
    return X[:-1, :] - X[1:, :], X[:, :-1] - X[:, 1:]


def lforward(P1, P2):
    """Adjoint of ltrans (a negative divergence)."""
    m, n = P1.shape[0] + 1, P2.shape[1] + 1
    X = np.zeros((m, n))
    X[:-1, :] += P1
    X[1:, :] -= P1
    X[:, :-1] += P2
    X[:, 1:] -= P2
    return X


def tlv(X, tv="iso"):
    P1, P2 = ltrans(np.asarray(X, np.float64))
    if tv == "iso":
        D = np.zeros(X.shape)
        D[:-1, :] = P1 ** 2
        D[:, :-1] += P2 ** 2
        return float(np.sqrt(D).sum())
    return float(np.abs(P1).sum() + np.abs(P2).sum())


def project_dual(P1, P2, tv):
    if tv == "iso":
        m, n = P1.shape[0] + 1, P2.shape[1] + 1
        A = np.zeros((m, n))
        A[:-1, :] = P1 ** 2
        A[:, :-1] += P2 ** 2
        A = np.sqrt(np.maximum(A, 1.0))
        return P1 / A[:-1, :], P2 / A[:, :-1]
    return np.clip(P1, -1.0, 1.0), np.clip(P2, -1.0, 1.0)


def tv_denoise(Xobs, lam, lb=0.0, ub=math.inf, tv="iso", max_iter=100, eps=1e-4):
    """Returns (X, iterations)."""
    Xobs = np.asarray(Xobs, np.float64)
    m, n = Xobs.shape
    project = lambda x: np.minimum(np.maximum(x, lb), ub)
    D = np.zeros((m, n))
    P1, P2 = project_dual(*ltrans(D), tv)
    R1, R2 = P1, P2
    tkp1, count, i, fval = 1.0, 0, 0, math.inf
    while i < max_iter and count < 5:
        fold = fval
        i += 1
        Dold = D
        Pold1, Pold2 = P1, P2
        tk = tkp1
        C = Xobs - lam * lforward(R1, R2)
        D = project(C)
        Q1, Q2 = ltrans(D)
        P1, P2 = project_dual(R1 + Q1 / (8 * lam), R2 + Q2 / (8 * lam), tv)
        tkp1 = (1 + math.sqrt(1 + 4 * tk * tk)) / 2
        R1 = P1 + (tk - 1) * (P1 - Pold1) / tkp1
        R2 = P2 + (tk - 1) * (P2 - Pold2) / tkp1
        with np.errstate(divide="ignore", invalid="ignore"):
            re = np.linalg.norm(D - Dold) / np.linalg.norm(D)   # NaN for D = 0, as there
        count = count + 1 if re < eps else 0
        fval = -np.linalg.norm(C - D) ** 2 + np.linalg.norm(C) ** 2
        if fval > fold:
            tkp1 = 1.0
    return D, i


def tv_objective(X, Xobs, lam, tv="iso"):
    return float(np.sum((X - Xobs) ** 2) + 2 * lam * tlv(X, tv))

"""The FP64 restatement of the reference's TV proximal map (oracle/tv_oracle.py:
FGP on the dual, utils/denoise_bound_mod.m) against an independent solver of
the same strongly convex problem (Chambolle-Pock primal-dual iterations), and
the adjoint relation of its difference operators."""
import math

import numpy as np
import pytest

from oracle import tv_oracle as TV


def chambolle_pock(Xobs, lam, lb, ub, tv, iters=20000):
    """min ||X - Xobs||^2 + 2 lam TV(X), lb <= X <= ub, by primal-dual steps
    with K = the difference operator (|K|^2 <= 8)."""
    X = np.clip(Xobs, lb, ub)
    Xb = X.copy()
    P1, P2 = np.zeros((X.shape[0] - 1, X.shape[1])), np.zeros((X.shape[0], X.shape[1] - 1))
    sigma = tau = 1.0 / math.sqrt(8.0)
    for _ in range(iters):
        Q1, Q2 = TV.ltrans(Xb)
        # dual step: prox of the conjugate of 2 lam TV = projection on the lam-scaled ball
        P1, P2 = P1 + sigma * Q1, P2 + sigma * Q2
        s1, s2 = TV.project_dual(P1 / (2 * lam), P2 / (2 * lam), tv)
        P1, P2 = 2 * lam * s1, 2 * lam * s2
        Xo = X
        # primal step: prox of ||X - Xobs||^2 + box
        V = X - tau * TV.lforward(P1, P2)
        X = np.clip((V + 2 * tau * Xobs) / (1 + 2 * tau), lb, ub)
        Xb = 2 * X - Xo
    return X


def test_difference_operators_are_adjoint():
    rng = np.random.default_rng(0)
    X = rng.standard_normal((7, 9))
    P1, P2 = rng.standard_normal((6, 9)), rng.standard_normal((7, 8))
    Q1, Q2 = TV.ltrans(X)
    assert abs((Q1 * P1).sum() + (Q2 * P2).sum() - (X * TV.lforward(P1, P2)).sum()) < 1e-12


@pytest.mark.parametrize("tv", ["iso", "l1"])
def test_fgp_reaches_the_minimiser(tv):
    rng = np.random.default_rng(1)
    n = 24
    yy, xx = np.mgrid[0:n, 0:n]
    clean = ((xx - 10) ** 2 + (yy - 12) ** 2 < 36).astype(float) + 0.5 * (xx > 16)
    Xobs = clean + 0.2 * rng.standard_normal((n, n))
    lam = 0.15
    X, it = TV.tv_denoise(Xobs, lam, 0.0, math.inf, tv, max_iter=5000, eps=1e-9)
    Xcp = chambolle_pock(Xobs, lam, 0.0, math.inf, tv)
    assert X.min() >= 0
    assert np.linalg.norm(X - Xcp) <= 1e-4 * np.linalg.norm(Xcp)
    assert TV.tv_objective(X, Xobs, lam, tv) <= TV.tv_objective(Xcp, Xobs, lam, tv) * (1 + 1e-7)
    # and the reference's default budget (100 iterations, 1e-4) is close to it
    X100, _ = TV.tv_denoise(Xobs, lam, 0.0, math.inf, tv)
    assert np.linalg.norm(X100 - Xcp) <= 2e-2 * np.linalg.norm(Xcp)

"""The FP64 restatement of the polychromatic model (oracle/bhc_oracle.py),
checked without the MATLAB reference: against quadrature of the integral that
defines each basis function, and by central finite differences."""
import numpy as np
import pytest
from scipy import integrate

from oracle import bhc_oracle as B


def hat_transform(k, j, s):
    """int hat_j(kappa) exp(-kappa s) dkappa over the hat on nodes k[j..j+2]."""
    a, b, c = k[j], k[j + 1], k[j + 2]
    up = integrate.quad(lambda t: (t - a) / (b - a) * np.exp(-t * s), a, b, epsabs=0, epsrel=1e-13)[0]
    dn = integrate.quad(lambda t: (c - t) / (c - b) * np.exp(-t * s), b, c, epsabs=0, epsrel=1e-13)[0]
    return up + dn


def test_kappa_nodes_follow_reference_padding_rule():
    k = B.kappa_nodes(20)
    assert k.size == 22
    assert np.isclose(k[1], 1e-2) and np.isclose(k[-2], 1e2)
    q = k[2] / k[1]
    assert np.isclose(k[0], k[1] / q) and np.isclose(k[-1], k[-2] * q)


@pytest.mark.parametrize("J", [20, 30])
def test_basis_matches_quadrature(J):
    k = B.kappa_nodes(J)
    s = np.array([0.0, 1e-7, 1e-4, 1e-2, 0.1, 0.5, 1.0, 3.0, 10.0, 50.0])
    Bm, _, _ = B.b1_basis(k, s)
    T = B.taylor_tables(k)
    for j in range(J):
        c0 = T["B"][j][0]
        for i, si in enumerate(s):
            ref = hat_transform(k, j, si)
            # the Taylor branch is accurate to 1e-6 of b_j(0) by construction
            tol = 2e-6 * c0 if abs(si) < T["thrB"][j] else 1e-9 * c0 + 1e-9 * abs(ref)
            assert abs(Bm[i, j] - ref) <= tol, (j, si, Bm[i, j], ref)


def test_derivatives_by_central_differences():
    k = B.kappa_nodes(20)
    s = np.array([0.05, 0.3, 1.0, 2.5, 7.0])
    h = 1e-5 * s
    Bp, Dp, _ = B.b1_basis(k, s + h)
    Bm, Dm, _ = B.b1_basis(k, s - h)
    _, D, DD = B.b1_basis(k, s)
    fd1 = (Bp - Bm) / (2 * h[:, None])
    fd2 = (Dp - Dm) / (2 * h[:, None])
    assert np.max(np.abs(fd1 - D)) <= 1e-6 * np.max(np.abs(D))
    assert np.max(np.abs(fd2 - DD)) <= 1e-5 * np.max(np.abs(DD))


def _problem(seed=0, nrays=400, npix=60, J=20):
    rng = np.random.default_rng(seed)
    A = rng.uniform(0, 0.05, (nrays, npix))
    x = rng.uniform(0.5, 3.0, npix)
    k = B.kappa_nodes(J)
    Ie = B.spectrum_bump(J, seed)
    s = A @ x
    BL, _, _ = B.b1_iout(k, s, Ie)
    m = rng.poisson(1e4 * BL) / 1e4
    return A, x, k, Ie, m


def test_alpha_gradient_by_central_differences():
    A, x, k, Ie, m = _problem()
    f = lambda xx: B.poiss_alpha(m, Ie, A @ xx, k, lambda w: A.T @ w)[0]
    _, g, _ = B.poiss_alpha(m, Ie, A @ x, k, lambda w: A.T @ w)
    rng = np.random.default_rng(3)
    for _ in range(8):
        d = rng.standard_normal(x.size)
        h = 1e-3 * np.linalg.norm(x) / np.linalg.norm(d)
        fd = (f(x + h * d) - f(x - h * d)) / (2 * h)
        # central differences with a 1e-3 relative step carry O(h^2) truncation
        assert abs(fd - g @ d) <= 1e-5 * np.linalg.norm(g) * np.linalg.norm(d)


def test_spectrum_gradient_and_hessian_by_central_differences():
    A, x, k, Ie, m = _problem(seed=1)
    Bm, _, _ = B.b1_basis(k, A @ x)
    f0, g, H = B.poiss_ie(m, Bm, Ie)
    rng = np.random.default_rng(4)
    for _ in range(8):
        d = rng.standard_normal(Ie.size)
        h = 1e-4 * np.linalg.norm(Ie) / np.linalg.norm(d)
        fp, gp, _ = B.poiss_ie(m, Bm, Ie + h * d)
        fm, gm, _ = B.poiss_ie(m, Bm, Ie - h * d)
        assert abs((fp - fm) / (2 * h) - g @ d) <= 1e-6 * np.linalg.norm(g) * np.linalg.norm(d)
        assert np.linalg.norm((gp - gm) / (2 * h) - H @ d) <= 1e-5 * np.linalg.norm(H @ d)


def test_zero_counts_contribute_bl_only():
    f = B.poisson_terms(np.array([0.5, 0.2]), np.array([0.0, 0.2]))
    assert np.allclose(f, [0.5, 0.0])


@pytest.mark.parametrize("noise", ["poisson", "gaussian"])
def test_density_hessian_weight_by_central_differences(noise):
    """Phi^T diag(weight) Phi v against differences of the gradient
    (the hessian closures of bhc/poissLAlpha.m:15-18, bhc/gaussLAlpha.m:18-20)."""
    A, x, k, Ie, m = _problem(seed=5)
    alpha = B.poiss_alpha if noise == "poisson" else B.gauss_alpha
    weight = B.poiss_hessian_weight if noise == "poisson" else B.gauss_hessian_weight
    bp = lambda w: A.T @ w
    h_w = weight(m, Ie, A @ x, k)
    rng = np.random.default_rng(6)
    for _ in range(6):
        v = rng.standard_normal(x.size)
        h = 1e-4 * np.linalg.norm(x) / np.linalg.norm(v)
        gp = alpha(m, Ie, A @ (x + h * v), k, bp)[1]
        gm = alpha(m, Ie, A @ (x - h * v), k, bp)[1]
        Hv = A.T @ (h_w * (A @ v))
        assert np.linalg.norm((gp - gm) / (2 * h) - Hv) <= 1e-6 * np.linalg.norm(Hv)


def test_gaussian_pair_by_central_differences():
    A, x, k, Ie, m = _problem(seed=7)
    f = lambda xx: B.gauss_alpha(m, Ie, A @ xx, k, lambda w: A.T @ w)[0]
    _, g, _ = B.gauss_alpha(m, Ie, A @ x, k, lambda w: A.T @ w)
    rng = np.random.default_rng(8)
    for _ in range(6):
        d = rng.standard_normal(x.size)
        h = 1e-3 * np.linalg.norm(x) / np.linalg.norm(d)
        fd = (f(x + h * d) - f(x - h * d)) / (2 * h)
        assert abs(fd - g @ d) <= 1e-5 * np.linalg.norm(g) * np.linalg.norm(d)
    Bm, _, _ = B.b1_basis(k, A @ x)
    _, gI, HI = B.gauss_ie(m, Bm, Ie)
    for _ in range(6):
        d = rng.standard_normal(Ie.size)
        h = 1e-4 * np.linalg.norm(Ie) / np.linalg.norm(d)
        fp, gp, _ = B.gauss_ie(m, Bm, Ie + h * d)
        fm, gm, _ = B.gauss_ie(m, Bm, Ie - h * d)
        assert abs((fp - fm) / (2 * h) - gI @ d) <= 1e-6 * np.linalg.norm(gI) * np.linalg.norm(d)
        assert np.linalg.norm((gp - gm) / (2 * h) - HI @ d) <= 1e-5 * np.linalg.norm(HI @ d)

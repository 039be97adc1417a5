"""The FP64 loop restatement (oracle/bhc_loop_oracle.py) on the CPU: its QP
direction satisfies the KKT conditions of the bound-constrained model, and its
spectrum step reaches at least the likelihood of the true spectrum."""
import numpy as np
import pytest

import oracle
from oracle import bhc_loop_oracle as LO
from oracle import bhc_oracle as BO


@pytest.mark.parametrize("seed", range(5))
def test_qp_direction_satisfies_kkt(seed):
    rng = np.random.default_rng(seed)
    J = 12
    B = rng.standard_normal((40, J)) * np.logspace(0, -4, J)   # columns over four decades
    H = B.T @ B
    g = rng.standard_normal(J)
    Ie = np.abs(rng.standard_normal(J)) * (rng.uniform(size=J) < 0.6)
    y = Ie + LO.qp_direction(H, g, Ie)
    c = g - H @ Ie
    lam = H @ y + c
    scale = np.abs(c) + np.abs(H @ y)
    assert np.all(y >= 0)
    free = y > 0
    assert np.all(np.abs(lam[free]) <= 1e-8 * scale[free] + 1e-12)
    assert np.all(lam[~free] >= -1e-8 * scale[~free] - 1e-12)


def _spectrum_problem(J, seed):
    from imgrecsrc_b200 import Geometry, phantom
    g = Geometry(64, 91, 48, 48, 1.0, 1.0, 300.0)
    Ts = 2.0 / g.n
    x = phantom.two_material_phantom(g.n, seed=seed)
    k = BO.kappa_nodes(J)
    I_true = BO.spectrum_bump(J, seed)
    s = Ts * oracle.forward(g, x.astype(np.float64)).ravel()
    A, _, _ = BO.b1_basis(k, s, derivs=0)
    rng = np.random.default_rng(seed + 1)
    m = rng.poisson(1e5 * (A @ I_true)) / 1e5
    return A, m, I_true


@pytest.mark.parametrize("noise", ["poisson", "gaussian"])
def test_spectrum_steps_reach_the_true_spectrum_likelihood(noise):
    A, m, I_true = _spectrum_problem(20, 2)
    Ie, f, steps = LO.spectrum_steps(A, m, np.full(20, 0.05), 30, noise)
    f_true = (BO.poiss_ie if noise == "poisson" else BO.gauss_ie)(m, A, I_true)[0]
    assert f <= f_true
    assert steps < 30
    assert np.all(Ie >= 0)

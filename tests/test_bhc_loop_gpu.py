"""The alternating BHC reconstruction (include/ctprj_bhc_loop.h) on the GPU:
the spectrum step against an FP64 bound-constrained solve of the same
objective (bhc/poissLI.m) and the first density step (no momentum yet)
against the FP64 oracle's projected-gradient step, plus monotone descent of
the loop and agreement of its fused and unfused likelihoods."""
import numpy as np
import pytest
from scipy import optimize

import oracle
from oracle import bhc_oracle as BO

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

import imgrecsrc_b200 as ct  # noqa: E402
from imgrecsrc_b200 import bhc, phantom  # noqa: E402


def rel(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


def setup_problem(J=20, seed=0):
    g = ct.Geometry(96, 136, 72, 72, 1.0, 1.0, 400.0)
    Ts = 2.0 / g.n
    x_true = phantom.two_material_phantom(g.n, seed=seed)
    k = BO.kappa_nodes(J)
    I_true = BO.spectrum_bump(J, seed)
    s = Ts * oracle.forward(g, x_true.astype(np.float64))
    BL, _, _ = BO.b1_iout(k, s.ravel(), I_true)
    rng = np.random.default_rng(seed + 1)
    m = (rng.poisson(1e5 * BL) / 1e5).reshape(g.np, g.prjWidth).astype(np.float32)
    return g, Ts, x_true, k, I_true, m


def saved_s(pr, dx, Ts):
    """The per-ray s the model saves: float(Ts * proj) of the float projection."""
    sino = pr.forward(dx).double().cpu().numpy().ravel()
    return (Ts * sino).astype(np.float32).astype(np.float64)


@pytest.mark.parametrize("J", [20, 32])
def test_spectrum_step_reaches_the_fp64_constrained_optimum(J):
    g, Ts, x_true, k, I_true, m = setup_problem(J=J)
    pr = ct.Projector(g)
    model = bhc.BHCModel(pr, k, Ts)
    dx = torch.from_numpy(x_true).cuda()
    dm = torch.from_numpy(m).cuda()
    I0 = np.full(I_true.size, 1.0 / I_true.size)
    dI = torch.from_numpy(I0.copy()).cuda()
    model.forward(dx, dI, dm, save=True)
    f_gpu = model.spectrum_step(dm, dI, newton_steps=20)
    # FP64 reference: the same objective on the GPU's own projections, solved by
    # L-BFGS-B in column-scaled variables (the basis columns span four decades)
    A, _, _ = BO.b1_basis(k, saved_s(pr, dx, Ts))
    mm = m.astype(np.float64).ravel()
    sc = A.max(axis=0)

    def fun(u):
        f, gr, _ = BO.poiss_ie(mm, A, u / sc)
        return f, gr / sc
    res = optimize.minimize(fun, I0 * sc, jac=True, method="L-BFGS-B", bounds=[(0, None)] * I0.size,
                            options=dict(ftol=1e-16, gtol=1e-14, maxiter=20000, maxcor=50))
    f_true = BO.poiss_ie(mm, A, I_true)[0]
    print("spectrum step: f gpu %.12e, f lbfgsb %.12e, f at the true spectrum %.12e"
          % (f_gpu, res.fun, f_true))
    # the maximum-likelihood spectrum is at least as likely as the true one
    assert f_gpu <= f_true
    assert f_gpu <= res.fun + 1e-6 * abs(res.fun)
    I_gpu = dI.cpu().numpy()
    f_at_gpu, _, _ = BO.poiss_ie(mm, A, I_gpu)
    assert abs(f_at_gpu - f_gpu) <= 1e-9 * abs(f_gpu)
    assert np.all(I_gpu >= 0)


def test_density_step_matches_fp64_projected_gradient_step():
    g, Ts, x_true, k, I_true, m = setup_problem(seed=2)
    pr = ct.Projector(g)
    model = bhc.BHCModel(pr, k, Ts)
    x0 = np.clip(x_true * 0.7 + 0.3, 0, None).astype(np.float32)
    dx = torch.from_numpy(x0.copy()).cuda()
    dI = torch.from_numpy(I_true.copy()).cuda()
    dm = torch.from_numpy(m).cuda()
    stats = model.reconstruct(dx, dI, dm, iterations=1, x_step=1e-3, skip_spectrum=True)
    a_used = stats["x_step"][0]
    assert a_used > 0
    s = Ts * oracle.forward(g, x0.astype(np.float64))
    Bm, D, _ = BO.b1_basis(k, s.ravel())
    BL, sBL = Bm @ I_true, D @ I_true
    w = (1 - m.astype(np.float64).ravel() / BL) * sBL
    gx = Ts * oracle.backward(g, w.reshape(g.np, g.prjWidth))
    x1 = np.maximum(0, x0 - a_used * gx)
    err = np.linalg.norm(dx.cpu().numpy() - x1) / np.linalg.norm(x1 - x0)
    print("density step: accepted step %.3e, rel err of the update %.2e" % (a_used, err))
    assert err < 1e-3


def test_loop_descends():
    g, Ts, x_true, k, I_true, m = setup_problem(J=20, seed=4)
    pr = ct.Projector(g)
    model = bhc.BHCModel(pr, k, Ts)
    dx = torch.full((g.n, g.n), 1.0, device="cuda")
    dI = torch.from_numpy(np.full(20, 1.0 / 20)).cuda()
    dm = torch.from_numpy(m).cuda()
    stats = model.reconstruct(dx, dI, dm, iterations=12, x_step=1e-3)
    c = stats["cost"][:stats["iterations"]]
    print("loop cost:", " ".join("%.6e" % v for v in c))
    assert stats["iterations"] == 12
    assert all(c[i + 1] <= c[i] * (1 + 1e-12) for i in range(len(c) - 1))
    assert c[-1] < 0.5 * c[0]
    assert stats["evaluations"] >= 2 * stats["iterations"]
    # the reported cost is the likelihood of the returned state
    A, _, _ = BO.b1_basis(k, saved_s(pr, dx, Ts))
    f_state = BO.poiss_ie(m.astype(np.float64).ravel(), A, dI.cpu().numpy())[0]
    assert abs(f_state - c[-1]) <= 1e-9 * abs(c[-1])


def test_fused_and_unfused_loops_agree():
    g, Ts, x_true, k, I_true, m = setup_problem(J=20, seed=6)
    pr = ct.Projector(g)
    model = bhc.BHCModel(pr, k, Ts)
    dm = torch.from_numpy(m).cuda()
    out = []
    for unfused in (False, True):
        dx = torch.full((g.n, g.n), 1.0, device="cuda")
        dI = torch.from_numpy(np.full(20, 1.0 / 20)).cuda()
        st = model.reconstruct(dx, dI, dm, iterations=5, x_step=1e-3, unfused=unfused)
        out.append((dx.clone(), dI.clone(), st))
    (x1, I1, s1), (x2, I2, s2) = out
    # the per-ray weights are identical; only the summation order of f differs
    assert np.allclose(s1["cost"], s2["cost"], rtol=1e-12, atol=0)
    assert torch.equal(x1, x2)
    assert torch.allclose(I1, I2, rtol=1e-12, atol=0)


@pytest.mark.parametrize("method,noise", [("npg", "poisson"), ("pg", "poisson"), ("npg", "gaussian")])
def test_loop_tracks_the_fp64_oracle_loop(method, noise):
    """12 iterations of the GPU loop against the same algorithm in FP64
    (oracle/bhc_loop_oracle.py over the FP64 projector): the line searches
    take the same decisions, so the cost traces, the density and the spectrum
    agree to the FP32 projections' accuracy."""
    from oracle import bhc_loop_oracle as LO
    g, Ts, x_true, k, I_true, m = setup_problem(J=20, seed=4)
    pr = ct.Projector(g)
    model = bhc.BHCModel(pr, k, Ts)
    model.set_noise(noise)
    dx = torch.full((g.n, g.n), 1.0, device="cuda")
    dI = torch.from_numpy(np.full(20, 1.0 / 20)).cuda()
    dm = torch.from_numpy(m).cuda()
    st = model.reconstruct(dx, dI, dm, iterations=12, x_step=1e-3, method=method)
    fw = lambda x: oracle.forward(g, x)
    bw = lambda y: oracle.backward(g, y.reshape(g.np, g.prjWidth))
    xo, Io, so = LO.reconstruct(fw, bw, k, Ts, np.ones((g.n, g.n)), np.full(20, 1.0 / 20),
                                m.astype(np.float64), 12, x_step=1e-3, method=method, noise=noise)
    c, co = np.array(st["cost"]), np.array(so["cost"])
    ex = rel(dx.cpu().numpy(), xo)
    eI = rel(dI.cpu().numpy(), Io)
    ec = float(np.max(np.abs(c - co) / np.abs(co)))
    steps_equal = np.allclose(st["x_step"], so["x_step"], rtol=1e-12, atol=0)
    print("loop vs FP64 oracle (%s, %s): max cost rel %.2e, x rel %.2e, Ie rel %.2e, same steps %s" % (
        method, noise, ec, ex, eI, steps_equal))
    assert steps_equal
    assert ec < 1e-4
    assert ex < 1e-4
    assert eI < 1e-3


def test_stopping_rule_matches_the_fp64_oracle_loop():
    """The reference's stopping rule (relative density change <= thresh in
    three iterations after the first, more than min_iterations run) stops the
    GPU loop and the FP64 loop at the same iteration, with the same changes."""
    from oracle import bhc_loop_oracle as LO
    g, Ts, x_true, k, I_true, m = setup_problem(J=20, seed=4)
    pr = ct.Projector(g)
    model = bhc.BHCModel(pr, k, Ts)
    dx = torch.full((g.n, g.n), 1.0, device="cuda")
    dI = torch.from_numpy(np.full(20, 1.0 / 20)).cuda()
    dm = torch.from_numpy(m).cuda()
    st = model.reconstruct(dx, dI, dm, iterations=60, x_step=1e-3, method="pg", thresh=2e-2, min_iterations=5)
    fw = lambda x: oracle.forward(g, x)
    bw = lambda y: oracle.backward(g, y.reshape(g.np, g.prjWidth))
    xo, Io, so = LO.reconstruct(fw, bw, k, Ts, np.ones((g.n, g.n)), np.full(20, 1.0 / 20),
                                m.astype(np.float64), 60, x_step=1e-3, method="pg", thresh=2e-2,
                                min_iterations=5)
    print("stopping rule: gpu %d iterations (converged %s), oracle %d (converged %s)" % (
        st["iterations"], st["converged"], len(so["cost"]), so["converged"]))
    assert st["converged"] and so["converged"]
    assert st["iterations"] == len(so["cost"]) < 60
    assert np.allclose(st["x_change"], so["x_change"], rtol=1e-4, atol=0)

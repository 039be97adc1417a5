"""The TV proximal map on the GPU (include/ctprj_tv.h) against the FP64
restatement of utils/denoise_bound_mod.m (oracle/tv_oracle.py), and the
alternating loop with the 'tviso' / 'tvl1' proximal maps against the FP64
loop (oracle/bhc_loop_oracle.py)."""
import ctypes
import math

import numpy as np
import pytest

import oracle
from oracle import bhc_oracle as BO
from oracle import tv_oracle as TVO

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

import imgrecsrc_b200 as ct  # noqa: E402
from imgrecsrc_b200 import bhc, phantom, tv  # noqa: E402
from imgrecsrc_b200._lib import CtprjError  # noqa: E402


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


def rel(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def noisy_image(m, n, seed=0):
    rng = np.random.default_rng(seed)
    yy, xx = np.mgrid[0:m, 0:n]
    img = ((xx - n / 2) ** 2 + (yy - m / 2) ** 2 < (min(m, n) / 3) ** 2).astype(np.float64)
    img += 0.5 * ((xx > n / 4) & (xx < n / 2) & (yy > m / 5) & (yy < m / 2))
    return (img + 0.2 * rng.standard_normal((m, n))).astype(np.float32)


def gpu_denoise(X, lam, lb=0.0, ub=math.inf, kind="iso", max_iter=100, eps=1e-4):
    m, n = X.shape
    dX = torch.from_numpy(X).cuda()
    out = torch.empty_like(dX)
    it = ctypes.c_int(0)
    ct.check(ct.lib().ctprj_tv_denoise(ctypes.c_void_p(dX.data_ptr()), m, n, lam, lb, ub, tv.TV_TYPES[kind],
                                       max_iter, eps, ctypes.c_void_p(out.data_ptr()), ctypes.byref(it), None))
    torch.cuda.synchronize()
    return out.cpu().numpy(), it.value


@pytest.mark.parametrize("kind", ["iso", "l1"])
@pytest.mark.parametrize("shape,lam", [((64, 64), 0.05), ((96, 80), 0.2), ((33, 130), 0.02)])
def test_fixed_iterations_match_the_fp64_fgp(kind, shape, lam):
    """epsilon = 0: both run exactly max_iter iterations of the same FGP
    (dual start, step, momentum, restart); D agrees to FP32 accuracy.  The
    iteration's momentum amplifies rounding: the same 60 iterations carried
    out in numpy float32 differ from float64 by up to 8e-5 on these inputs
    (small lambda, where the dual step 1/(8 lambda) is large), hence 2e-4."""
    X = noisy_image(*shape, seed=shape[0])
    D, it = gpu_denoise(X, lam, kind=kind, max_iter=60, eps=0.0)
    Do, ito = TVO.tv_denoise(X.astype(np.float64), lam, tv=kind, max_iter=60, eps=0.0)
    e = rel(D, Do)
    print("FGP %s %s lam %g: rel %.2e" % (kind, shape, lam, e))
    assert it == ito == 60
    assert e < 2e-4


@pytest.mark.parametrize("kind", ["iso", "l1"])
def test_stopping_rule_and_objective_match(kind):
    """With the reference's default epsilon (1e-4) the FP32 iteration stops
    within an iteration or two of the FP64 one and reaches the same objective
    ||X - Xobs||^2 + 2 lam TV(X) to 1e-5."""
    X = noisy_image(128, 128, seed=3)
    D, it = gpu_denoise(X, 0.1, kind=kind, max_iter=500, eps=1e-4)
    Do, ito = TVO.tv_denoise(X.astype(np.float64), 0.1, tv=kind, max_iter=500, eps=1e-4)
    fo = TVO.tv_objective(Do, X.astype(np.float64), 0.1, kind)
    f = TVO.tv_objective(D.astype(np.float64), X.astype(np.float64), 0.1, kind)
    print("FGP %s: gpu %d iterations, oracle %d; objective rel %.2e; D rel %.2e" % (
        kind, it, ito, abs(f - fo) / fo, rel(D, Do)))
    assert abs(it - ito) <= 2
    assert abs(f - fo) / fo < 1e-5
    assert rel(D, Do) < 1e-3


def test_bounds_are_honoured():
    """lb / ub clamp the primal iterate (denoise_bound_mod's project)."""
    X = 3.0 * noisy_image(64, 72, seed=5) - 1.0
    D, it = gpu_denoise(X, 0.1, lb=-0.25, ub=1.5, max_iter=40, eps=0.0)
    Do, _ = TVO.tv_denoise(X.astype(np.float64), 0.1, lb=-0.25, ub=1.5, max_iter=40, eps=0.0)
    assert D.min() >= -0.25 and D.max() <= 1.5
    assert rel(D, Do) < 2e-4


def test_constant_image_stops_after_five_small_changes():
    """A constant image is a fixed point: D = clamp(Xobs) from the first
    iteration, the relative change is 0 from the second on, and the count
    reaches five at the sixth iteration, as in the reference."""
    X = np.full((40, 50), 0.7, np.float32)
    D, it = gpu_denoise(X, 0.3, max_iter=100, eps=1e-4)
    _, ito = TVO.tv_denoise(X.astype(np.float64), 0.3, max_iter=100, eps=1e-4)
    assert it == ito == 6
    assert np.array_equal(D, X)


def test_zero_image_runs_to_max_iter():
    """Xobs = 0 keeps D = 0, whose relative change is NaN (0/0) and never
    counts: the iteration runs to max_iter, as the reference's does."""
    X = np.zeros((32, 32), np.float32)
    D, it = gpu_denoise(X, 0.3, max_iter=17, eps=1e-4)
    _, ito = TVO.tv_denoise(X.astype(np.float64), 0.3, max_iter=17, eps=1e-4)
    assert it == ito == 17
    assert not D.any()


@pytest.mark.parametrize("kind", ["iso", "l1"])
def test_tv_value_matches_tlv(kind):
    X = noisy_image(75, 61, seed=7)
    v = tv.tlv(torch.from_numpy(X).cuda(), kind)
    vo = TVO.tlv(X.astype(np.float64), kind)
    assert abs(v - vo) / vo < 1e-12


def test_masked_vector_form_matches_the_reference_call():
    """TV.denoise(x, u, thresh, maxItr, maskmt): the masked pixel vector is
    scattered (column-major) into a zero image, denoised, and gathered."""
    n = 48
    X = noisy_image(n, n, seed=9)
    yy, xx = np.mgrid[0:n, 0:n]
    mask = (xx - n / 2) ** 2 + (yy - n / 2) ** 2 < (0.45 * n) ** 2
    idx = np.flatnonzero(mask.T.ravel())                 # MATLAB find(): column-major
    xvec = X.T.ravel()[idx]
    dmask = torch.from_numpy(mask).cuda()
    out, it = tv.denoise(torch.from_numpy(np.ascontiguousarray(xvec)).cuda(), 0.1, 0.0, 50, mask=dmask)
    img = np.zeros(n * n)
    img[idx] = xvec
    Do, ito = TVO.tv_denoise(img.reshape(n, n).T, 0.1, max_iter=50, eps=0.0)   # back to (row, col)
    ref = Do.T.ravel()[idx]
    assert it == ito == 50
    assert rel(out.cpu().numpy(), ref) < 2e-4


def test_invalid_arguments_raise():
    d = torch.zeros(16, device="cuda")
    with pytest.raises(CtprjError):
        tv.denoise(d, 0.0, 1e-4, 10, n_row=4, n_col=4)        # lambda must be positive
    with pytest.raises(CtprjError):
        tv.denoise(d, 0.1, 1e-4, 10, n_row=1, n_col=16)       # at least 2 x 2
    with pytest.raises(CtprjError):
        tv.denoise(d, 0.1, 1e-4, 10, n_row=4, n_col=4, lb=1.0, ub=0.5)


def setup_problem(J=20, seed=4):
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


@pytest.mark.parametrize("method,proximal", [("npg", "tviso"), ("pg", "tviso"), ("npg", "tvl1")])
def test_tv_loop_tracks_the_fp64_oracle_loop(method, proximal):
    """12 alternating iterations with u TV(x) regularisation (u = 1e-2): the
    GPU loop and the FP64 loop take the same density steps and agree in cost,
    density and spectrum to the FP32 projections' accuracy."""
    from oracle import bhc_loop_oracle as LO
    g, Ts, x_true, k, I_true, m = setup_problem()
    pr = ct.Projector(g)
    model = bhc.BHCModel(pr, k, Ts)
    dx = torch.full((g.n, g.n), 1.0, device="cuda")
    dI = torch.from_numpy(np.full(20, 1.0 / 20)).cuda()
    dm = torch.from_numpy(m).cuda()
    st = model.reconstruct(dx, dI, dm, iterations=12, x_step=1e-3, method=method, proximal=proximal, u=1e-2)
    fw = lambda x: oracle.forward(g, x)
    bw = lambda y: oracle.backward(g, y.reshape(g.np, g.prjWidth))
    xo, Io, so = LO.reconstruct(fw, bw, k, Ts, np.ones((g.n, g.n)), np.full(20, 1.0 / 20),
                                m.astype(np.float64), 12, x_step=1e-3, method=method, proximal=proximal,
                                u=1e-2)
    c, co = np.array(st["cost"]), np.array(so["cost"])
    ex = rel(dx.cpu().numpy(), xo)
    eI = rel(dI.cpu().numpy(), Io)
    ec = float(np.max(np.abs(c - co) / np.abs(co)))
    steps_equal = np.allclose(st["x_step"], so["x_step"], rtol=1e-12, atol=0)
    print("TV loop vs FP64 oracle (%s, %s): max cost rel %.2e, x rel %.2e, Ie rel %.2e, same steps %s, "
          "inner %d / %d, retries %d / %d" % (method, proximal, ec, ex, eI, steps_equal,
                                              st["inner_iterations"], so["inner_iterations"],
                                              st["prox_retries"], so["prox_retries"]))
    assert steps_equal
    assert ec < 1e-3
    assert ex < 1e-3
    assert eI < 1e-2
    assert st["penalty"] > 0 and abs(st["penalty"] - so["penalty"]) / so["penalty"] < 1e-3


def test_tv_loop_rejects_zero_weight():
    g, Ts, x_true, k, I_true, m = setup_problem()
    pr = ct.Projector(g)
    model = bhc.BHCModel(pr, k, Ts)
    dx = torch.full((g.n, g.n), 1.0, device="cuda")
    dI = torch.from_numpy(np.full(20, 1.0 / 20)).cuda()
    dm = torch.from_numpy(m).cuda()
    with pytest.raises(CtprjError):
        model.reconstruct(dx, dI, dm, iterations=2, proximal="tviso", u=0.0)


def test_tv_loop_retries_with_more_inner_iterations():
    """PG with a three-iteration inner limit: once a step raises f + u TV the
    reference retries it with maxInnerItr * 10 (npg/PG.m:103-121); the GPU
    loop takes that retry where the FP64 loop does and then follows it.  With
    three FGP iterations per step, each step's accept / halve decisions sit
    close to their thresholds, so FP32 rounding of the projections may flip
    a late one: the two step sequences must agree over the first 30 of the 60
    iterations (they run to iteration 39 on the B200 today), the retry counts
    must be equal and the final images within 1e-3."""
    from oracle import bhc_loop_oracle as LO
    g, Ts, x_true, k, I_true, m = setup_problem()
    pr = ct.Projector(g)
    model = bhc.BHCModel(pr, k, Ts)
    dx = torch.full((g.n, g.n), 1.0, device="cuda")
    dI = torch.from_numpy(np.full(20, 1.0 / 20)).cuda()
    dm = torch.from_numpy(m).cuda()
    kw = dict(iterations=60, x_step=1e-3, method="pg", proximal="tviso", u=0.1, max_inner=3, skip_spectrum=True)
    st = model.reconstruct(dx, dI, dm, **kw)
    fw = lambda x: oracle.forward(g, x)
    bw = lambda y: oracle.backward(g, y.reshape(g.np, g.prjWidth))
    xo, Io, so = LO.reconstruct(fw, bw, k, Ts, np.ones((g.n, g.n)), np.full(20, 1.0 / 20),
                                m.astype(np.float64), **kw)
    sg, sO = np.array(st["x_step"]), np.array(so["x_step"])
    same = np.isclose(sg, sO, rtol=1e-12, atol=0)
    n_same = int(np.argmin(same)) if not same.all() else same.size
    print("TV retries: gpu %d, oracle %d; inner %d / %d; steps agree over the first %d iterations; x rel %.2e"
          % (st["prox_retries"], so["prox_retries"], st["inner_iterations"], so["inner_iterations"], n_same,
             rel(dx.cpu().numpy(), xo)))
    assert so["prox_retries"] >= 1
    assert st["prox_retries"] == so["prox_retries"]
    # the inner stopping rule compares relative changes of D with
    # admmTol * difAlpha, small enough here that FP32 rounding of D can move
    # the iteration at which five small changes in a row are first seen
    assert abs(st["inner_iterations"] - so["inner_iterations"]) <= 0.15 * so["inner_iterations"]
    assert n_same >= 30
    assert rel(dx.cpu().numpy(), xo) < 1e-3


def test_tv_loop_options_without_restart_or_step_growth():
    """opt.restart = false, opt.adaptiveStep = false, opt.admmTol = 1e-3 and
    skipIe, as the reference's TV examples set them: the GPU loop follows the
    FP64 loop step for step."""
    from oracle import bhc_loop_oracle as LO
    g, Ts, x_true, k, I_true, m = setup_problem()
    pr = ct.Projector(g)
    model = bhc.BHCModel(pr, k, Ts)
    dx = torch.full((g.n, g.n), 1.0, device="cuda")
    dx[:4] = -0.5                                     # clamped to 0 before the first step
    dI = torch.from_numpy(np.full(20, 1.0 / 20)).cuda()
    dm = torch.from_numpy(m).cuda()
    kw = dict(iterations=15, x_step=1e-3, method="npg", proximal="tviso", u=1e-2, admm_tol=1e-3,
              restart=False, adaptive_step=False, skip_spectrum=True)
    st = model.reconstruct(dx, dI, dm, **kw)
    x0 = np.ones((g.n, g.n))
    x0[:4] = -0.5
    fw = lambda x: oracle.forward(g, x)
    bw = lambda y: oracle.backward(g, y.reshape(g.np, g.prjWidth))
    xo, Io, so = LO.reconstruct(fw, bw, k, Ts, x0, np.full(20, 1.0 / 20), m.astype(np.float64), **kw)
    steps_equal = np.allclose(st["x_step"], so["x_step"], rtol=1e-12, atol=0)
    c, co = np.array(st["cost"]), np.array(so["cost"])
    print("TV loop, no restart / adaptive step: same steps %s, restarts %d, max cost rel %.2e, x rel %.2e" % (
        steps_equal, st["restarts"], float(np.max(np.abs(c - co) / np.abs(co))), rel(dx.cpu().numpy(), xo)))
    assert steps_equal
    assert st["restarts"] == 0
    assert abs(st["inner_iterations"] - so["inner_iterations"]) <= 0.15 * so["inner_iterations"]
    assert float(np.max(np.abs(c - co) / np.abs(co))) < 1e-3
    assert rel(dx.cpu().numpy(), xo) < 1e-3


def test_tv_map_at_512_matches_the_fp64_fgp():
    """A 512^2 image (16 x 16 tiles of the pipelined kernel, several tiles per
    persistent block): 40 fixed iterations against the FP64 FGP."""
    X = noisy_image(512, 512, seed=11)
    D, it = gpu_denoise(X, 0.1, kind="iso", max_iter=40, eps=0.0)
    Do, ito = TVO.tv_denoise(X.astype(np.float64), 0.1, tv="iso", max_iter=40, eps=0.0)
    e = rel(D, Do)
    print("FGP 512^2: rel %.2e" % e)
    assert it == ito == 40
    assert e < 2e-4


def test_tv_loop_with_bb_start_and_l1_tracks_the_oracle():
    """PG with 'tvl1' and the reference's default initial step rule ('BB')."""
    from oracle import bhc_loop_oracle as LO
    g, Ts, x_true, k, I_true, m = setup_problem()
    pr = ct.Projector(g)
    model = bhc.BHCModel(pr, k, Ts)
    dx = torch.full((g.n, g.n), 1.0, device="cuda")
    dI = torch.from_numpy(np.full(20, 1.0 / 20)).cuda()
    dm = torch.from_numpy(m).cuda()
    kw = dict(x_step=1e-3, method="pg", proximal="tvl1", u=1e-2, init_step="bb")
    st = model.reconstruct(dx, dI, dm, iterations=10, **kw)
    fw = lambda x: oracle.forward(g, x)
    bw = lambda y: oracle.backward(g, y.reshape(g.np, g.prjWidth))
    xo, Io, so = LO.reconstruct(fw, bw, k, Ts, np.ones((g.n, g.n)), np.full(20, 1.0 / 20),
                                m.astype(np.float64), 10, **kw)
    c, co = np.array(st["cost"]), np.array(so["cost"])
    steps_equal = np.allclose(st["x_step"], so["x_step"], rtol=1e-5, atol=0)
    print("TV loop bb/l1: max cost rel %.2e, x rel %.2e, steps equal %s" % (
        float(np.max(np.abs(c - co) / np.abs(co))), rel(dx.cpu().numpy(), xo), steps_equal))
    assert steps_equal
    assert float(np.max(np.abs(c - co) / np.abs(co))) < 1e-3
    assert rel(dx.cpu().numpy(), xo) < 1e-3

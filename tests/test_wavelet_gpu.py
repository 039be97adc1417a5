"""The wavelet transform and the ADMM wavelet proximal map on the GPU
(include/ctprj_wavelet.h) against the reference's compiled rwt cores
(tests/golden/rwt_golden.npz) and the FP64 restatement of npg/admm.m
(oracle/wavelet_oracle.py)."""
import os

import numpy as np
import pytest

from oracle import wavelet_oracle as W

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

import imgrecsrc_b200 as ct  # noqa: E402
from imgrecsrc_b200 import wavelet  # noqa: E402
from imgrecsrc_b200._lib import CtprjError  # noqa: E402

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "rwt_golden.npz")
MASKS = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "wvltmask_golden.npz")


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


def rel(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def dev(x):
    return torch.from_numpy(np.ascontiguousarray(x, np.float32)).cuda()


def test_transforms_match_the_compiled_reference():
    """Every golden case (Haar to 12 taps, 2 to 6 levels, filters longer than
    the coarsest block): FP32 transforms within 1e-6 of the reference's
    double-precision MDWT / MIDWT."""
    g = np.load(GOLDEN)
    i = 0
    while "case%d_meta" % i in g:
        daub, m, n, L = (int(v) for v in g["case%d_meta" % i])
        h = g["case%d_h" % i]
        x = dev(g["case%d_x" % i])
        y = wavelet.mdwt(x, h, L).cpu().numpy()
        xi = wavelet.midwt(x, h, L).cpu().numpy()
        e1, e2 = rel(y, g["case%d_mdwt" % i]), rel(xi, g["case%d_midwt" % i])
        print("rwt case %d (daub %d, %dx%d, L %d): mdwt %.2e midwt %.2e" % (i, daub, m, n, L, e1, e2))
        assert e1 < 1e-6 and e2 < 1e-6
        i += 1
    assert i >= 7


@pytest.mark.parametrize("daub,shape,L", [(2, (1024, 1024), 6), (4, (512, 768), 5), (8, (256, 128), 4)])
def test_large_transforms_and_inverse(daub, shape, L):
    rng = np.random.default_rng(daub)
    X = rng.standard_normal(shape)
    h = W.daubcqf(daub)
    y = wavelet.mdwt(dev(X), h, L)
    e = rel(y.cpu().numpy(), W.mdwt(X, h, L))
    xi = wavelet.midwt(y, h, L).cpu().numpy()
    print("daub %d %s L %d: mdwt rel %.2e, round trip %.2e" % (daub, shape, L, e, rel(xi, X)))
    assert e < 1e-6
    assert rel(xi, X) < 2e-6


def test_transposed_layout_gives_the_matlab_coefficients():
    """A column-major (MATLAB) array passed as it lies, rows and columns
    swapped: the result read column-major is MATLAB's mdwt."""
    rng = np.random.default_rng(5)
    X = rng.standard_normal((64, 32))                 # MATLAB 64 x 32
    h = W.daubcqf(4)
    mem = dev(X.T)                                    # its memory, row-major 32 x 64
    y = wavelet.mdwt(mem, h, 3).cpu().numpy().T
    assert rel(y, W.mdwt(X, h, 3)) < 1e-6


@pytest.mark.parametrize("daub", [2, 6])
def test_l1_penalty(daub):
    rng = np.random.default_rng(6)
    X = rng.standard_normal((128, 64))
    h = W.daubcqf(daub)
    v = wavelet.l1(dev(X), h, 4)
    vo = W.l1_penalty(X.astype(np.float32).astype(np.float64), h, 4)
    assert abs(v - vo) / vo < 1e-6


def phantomish(n, seed):
    rng = np.random.default_rng(seed)
    yy, xx = np.mgrid[0:n, 0:n]
    img = ((xx - n / 2) ** 2 + (yy - n / 2) ** 2 < (n / 3) ** 2).astype(np.float64)
    img += 0.7 * ((xx > n / 5) & (xx < n / 2) & (yy > n / 4) & (yy < n / 2))
    return img + 0.1 * rng.standard_normal((n, n))


@pytest.mark.parametrize("daub,u", [(2, 0.5), (4, 0.2)])
def test_admm_fixed_iterations_match_the_fp64_restatement(daub, u):
    """relativeTol = 0: both run maxItr + 1 iterations of the same ADMM
    (including rho adaptations after 20 iterations); alpha agrees to FP32
    accuracy."""
    a = phantomish(64, daub) - 0.2
    init = np.maximum(phantomish(64, daub + 1), 0.0)
    h = W.daubcqf(daub)
    al, it = wavelet.admm(dev(a), u, h, 5, relative_tol=0.0, max_itr=60, init=dev(init))
    alo, ito = W.admm(a.astype(np.float32).astype(np.float64), u, h, 5, rel_tol=0.0, max_itr=60,
                      init=init.astype(np.float32).astype(np.float64))
    e = rel(al.cpu().numpy(), alo)
    print("ADMM daub %d u %g: %d / %d iterations, alpha rel %.2e" % (daub, u, it, ito, e))
    assert it == ito == 61
    assert e < 1e-4
    assert al.min().item() >= 0.0


def test_admm_stopping_rule_and_objective():
    """With the tolerances the density step passes (1e-3 down), the FP32
    iteration stops within a few iterations of the FP64 one and reaches the
    same objective 1/2 |alpha - a|^2 + u |W alpha|_1 to 1e-5."""
    a = phantomish(128, 9) - 0.1
    h = W.daubcqf(2)
    for tol in (1e-3, 1e-5):
        al, it = wavelet.admm(dev(a), 0.3, h, 6, relative_tol=tol, max_itr=1000)
        a64 = a.astype(np.float32).astype(np.float64)
        alo, ito = W.admm(a64, 0.3, h, 6, rel_tol=tol, max_itr=1000)
        f = W.admm_objective(al.cpu().numpy().astype(np.float64), a64, 0.3, h, 6)
        fo = W.admm_objective(alo, a64, 0.3, h, 6)
        print("ADMM tol %g: gpu %d iterations, oracle %d; objective rel %.2e" % (tol, it, ito, abs(f - fo) / fo))
        assert abs(it - ito) <= max(3, 0.1 * ito)
        assert abs(f - fo) / fo < 1e-5


@pytest.mark.parametrize("L,shape", [(6, (256, 192)), (3, (40, 64)), (1, (6, 10))])
def test_fused_two_tap_iteration_matches_the_level_passes(L, shape, monkeypatch):
    """The fused per-tile iteration (two-tap filters, up to 6 levels) against
    the level-by-level passes (CTPRJ_WVLT_KERNEL=levels) and the FP64
    restatement: the same arithmetic, so the same iterations and alpha to
    rounding of the FP64 partial sums' order."""
    rng = np.random.default_rng(L)
    a = rng.standard_normal(shape) + 0.3
    init = np.maximum(rng.standard_normal(shape), 0.0)
    h = W.daubcqf(2)
    fa, it_f = wavelet.admm(dev(a), 0.4, h, L, relative_tol=0.0, max_itr=45, init=dev(init))
    monkeypatch.setenv("CTPRJ_WVLT_KERNEL", "levels")
    la, it_l = wavelet.admm(dev(a), 0.4, h, L, relative_tol=0.0, max_itr=45, init=dev(init))
    monkeypatch.delenv("CTPRJ_WVLT_KERNEL")
    alo, ito = W.admm(a.astype(np.float32).astype(np.float64), 0.4, h, L, rel_tol=0.0, max_itr=45,
                      init=init.astype(np.float32).astype(np.float64))
    e_fl = rel(fa.cpu().numpy(), la.cpu().numpy())
    e_fo = rel(fa.cpu().numpy(), alo)
    print("fused vs levels (L %d, %s): %d / %d / %d iterations, rel %.2e, vs FP64 %.2e" % (
        L, shape, it_f, it_l, ito, e_fl, e_fo))
    assert it_f == it_l == ito == 46
    assert e_fl < 1e-6
    assert e_fo < 1e-4


def test_admm_zero_input_and_errors():
    z = torch.zeros(32, 32, device="cuda")
    out, it = wavelet.admm(z, 0.1, W.daubcqf(2), 3)
    assert it == 0 and not out.any().item()
    x = torch.zeros(24, 24, device="cuda")
    with pytest.raises(CtprjError):
        wavelet.mdwt(x, W.daubcqf(2), 4)               # 24 not divisible by 16
    with pytest.raises(CtprjError):
        wavelet.mdwt(x, np.ones(3), 1)                # odd filter
    with pytest.raises(CtprjError):
        wavelet.admm(x, -1.0, W.daubcqf(2), 2)        # negative weight


def setup_problem(J=20, seed=4):
    import oracle
    from oracle import bhc_oracle as BO
    from imgrecsrc_b200 import phantom
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


@pytest.mark.parametrize("method,daub", [("npg", 2), ("pg", 2), ("npg", 4)])
def test_wvlt_loop_tracks_the_fp64_oracle_loop(method, daub):
    """12 alternating iterations with the reference's default regulariser
    ('wvltADMM', u = 1e-2, 5 levels): the GPU loop and the FP64 loop take the
    same density steps and agree in cost, density and spectrum."""
    import oracle
    from oracle import bhc_loop_oracle as LO
    from imgrecsrc_b200 import bhc
    g, Ts, x_true, k, I_true, m = setup_problem()
    h = W.daubcqf(daub)
    pr = ct.Projector(g)
    model = bhc.BHCModel(pr, k, Ts)
    dx = torch.full((g.n, g.n), 1.0, device="cuda")
    dI = torch.from_numpy(np.full(20, 1.0 / 20)).cuda()
    dm = torch.from_numpy(m).cuda()
    st = model.reconstruct(dx, dI, dm, iterations=12, x_step=1e-3, method=method, proximal="wvltADMM", u=1e-2,
                           wvlt_filter=h, wvlt_levels=5)
    fw = lambda x: oracle.forward(g, x)
    bw = lambda y: oracle.backward(g, y.reshape(g.np, g.prjWidth))
    xo, Io, so = LO.reconstruct(fw, bw, k, Ts, np.ones((g.n, g.n)), np.full(20, 1.0 / 20),
                                m.astype(np.float64), 12, x_step=1e-3, method=method, proximal="wvltADMM",
                                u=1e-2, wvlt_h=h, wvlt_levels=5)
    c, co = np.array(st["cost"]), np.array(so["cost"])
    ex = rel(dx.cpu().numpy(), xo)
    eI = rel(dI.cpu().numpy(), Io)
    ec = float(np.max(np.abs(c - co) / np.abs(co)))
    steps_equal = np.allclose(st["x_step"], so["x_step"], rtol=1e-12, atol=0)
    print("wvlt loop vs FP64 oracle (%s, daub %d): max cost rel %.2e, x rel %.2e, Ie rel %.2e, same steps %s, "
          "inner %d / %d, retries %d / %d" % (method, daub, ec, ex, eI, steps_equal, st["inner_iterations"],
                                              so["inner_iterations"], st["prox_retries"], so["prox_retries"]))
    assert steps_equal
    assert ec < 1e-3
    assert ex < 1e-3
    assert eI < 1e-2
    assert abs(st["inner_iterations"] - so["inner_iterations"]) <= 0.15 * so["inner_iterations"]
    assert st["penalty"] > 0 and abs(st["penalty"] - so["penalty"]) / so["penalty"] < 1e-3


def test_wvlt_loop_rejects_indivisible_image():
    from imgrecsrc_b200 import bhc
    g, Ts, x_true, k, I_true, m = setup_problem()
    model = bhc.BHCModel(ct.Projector(g), k, Ts)
    dx = torch.full((g.n, g.n), 1.0, device="cuda")
    dI = torch.from_numpy(np.full(20, 1.0 / 20)).cuda()
    with pytest.raises(CtprjError):   # 96 is not divisible by 2^6
        model.reconstruct(dx, dI, torch.from_numpy(m).cuda(), iterations=2, proximal="wvltADMM", u=1e-2)


def disc(n, r):
    yy, xx = np.mgrid[0:n, 0:n]
    return (xx - (n - 1) / 2) ** 2 + (yy - (n - 1) / 2) ** 2 < r ** 2


@pytest.mark.parametrize("daub,L", [(2, 4), (4, 3)])
def test_wvlt_mask_matches_utils_wvltmask(daub, L):
    """ctprj_wvlt_mask against the literal restatement of utils/wvltMask.m
    (the union over the mask's pixels of the transform's nonzeros)."""
    m = disc(64, 25)
    h = W.daubcqf(daub)
    g = wavelet.wvlt_mask(torch.from_numpy(m).cuda(), h, L).cpu().numpy().astype(bool)
    assert np.array_equal(g, W.wvlt_mask(m, h, L))


def test_wvlt_mask_matches_every_reference_mask():
    """ctprj_wvlt_mask on Utils.getCircularMask(n) against all 19 coefficient
    masks the reference ships (utils/MaskWvlt<n>CircleL<L>D<D>.mat, outputs of
    its utils/wvltMask.m; n = 64 ... 1024, 1 to 9 levels, Haar and the 6-tap
    filter), bit for bit."""
    z = np.load(MASKS)
    keys = sorted(k for k in z.files if not k.endswith("_count"))
    assert len(keys) == 19
    for key in keys:
        n, L, D = (int(p[1:]) for p in key.split("_"))
        ref = np.unpackbits(z[key], count=n * n).reshape((n, n), order="F").astype(bool)
        assert ref.sum() == int(z[key + "_count"])
        m = torch.from_numpy(W.circular_mask(n).astype(np.uint8)).cuda()
        got = wavelet.wvlt_mask(m, W.daubcqf(D), L).cpu().numpy().astype(bool)
        assert np.array_equal(got, ref), (key, int((got != ref).sum()))


@pytest.mark.parametrize("method,proximal,daub", [("npg", "wvltADMM", 2), ("pg", "wvltADMM", 4),
                                                  ("npg", "tviso", 2)])
def test_masked_loop_tracks_the_fp64_oracle_loop(method, proximal, daub):
    """The loop with the reference's reconstruction mask (opt.mask, a disc):
    the density stays on the mask, gradients and proximal maps are the masked
    ones (maskk derived as utils/wvltMask.m does), and the GPU loop takes the
    FP64 loop's steps."""
    import oracle
    from oracle import bhc_loop_oracle as LO
    from imgrecsrc_b200 import bhc
    g, Ts, x_true, k, I_true, m = setup_problem()
    mk = disc(g.n, 0.45 * g.n)
    h = W.daubcqf(daub)
    pr = ct.Projector(g)
    model = bhc.BHCModel(pr, k, Ts)
    dx = torch.full((g.n, g.n), 1.0, device="cuda")
    dI = torch.from_numpy(np.full(20, 1.0 / 20)).cuda()
    dm = torch.from_numpy(m).cuda()
    st = model.reconstruct(dx, dI, dm, iterations=10, x_step=1e-3, method=method, proximal=proximal, u=1e-2,
                           wvlt_filter=h, wvlt_levels=5, mask=torch.from_numpy(mk).cuda())
    fw = lambda x: oracle.forward(g, x)
    bw = lambda y: oracle.backward(g, y.reshape(g.np, g.prjWidth))
    xo, Io, so = LO.reconstruct(fw, bw, k, Ts, np.ones((g.n, g.n)), np.full(20, 1.0 / 20),
                                m.astype(np.float64), 10, x_step=1e-3, method=method, proximal=proximal,
                                u=1e-2, wvlt_h=h, wvlt_levels=5, mask=mk)
    x = dx.cpu().numpy()
    c, co = np.array(st["cost"]), np.array(so["cost"])
    ec = float(np.max(np.abs(c - co) / np.abs(co)))
    steps_equal = np.allclose(st["x_step"], so["x_step"], rtol=1e-12, atol=0)
    print("masked loop (%s, %s, daub %d): max cost rel %.2e, x rel %.2e, same steps %s, inner %d / %d" % (
        method, proximal, daub, ec, rel(x, xo), steps_equal, st["inner_iterations"], so["inner_iterations"]))
    assert not x[~mk].any()
    assert steps_equal
    assert ec < 1e-3
    assert rel(x, xo) < 1e-3
    assert abs(st["inner_iterations"] - so["inner_iterations"]) <= 0.15 * so["inner_iterations"]


def test_admm_at_512_matches_the_fp64_restatement():
    """A 512^2 image, Haar, 6 levels (the fused per-tile iteration over 64
    tiles): 30 fixed iterations against the FP64 ADMM."""
    a = phantomish(512, 3) - 0.2
    h = W.daubcqf(2)
    al, it = wavelet.admm(dev(a), 0.3, h, 6, relative_tol=0.0, max_itr=29)
    alo, ito = W.admm(a.astype(np.float32).astype(np.float64), 0.3, h, 6, rel_tol=0.0, max_itr=29)
    e = rel(al.cpu().numpy(), alo)
    print("ADMM 512^2: %d / %d iterations, alpha rel %.2e" % (it, ito, e))
    assert it == ito == 30
    assert e < 1e-4


def test_wvlt_loop_gaussian_noise_tracks_the_oracle():
    """'wvltADMM' with the Gaussian (log-domain least squares) model."""
    import oracle
    from oracle import bhc_loop_oracle as LO
    from imgrecsrc_b200 import bhc
    g, Ts, x_true, k, I_true, m = setup_problem()
    pr = ct.Projector(g)
    model = bhc.BHCModel(pr, k, Ts)
    model.set_noise("gaussian")
    dx = torch.full((g.n, g.n), 1.0, device="cuda")
    dI = torch.from_numpy(np.full(20, 1.0 / 20)).cuda()
    dm = torch.from_numpy(m).cuda()
    kw = dict(x_step=1e-3, method="npg", proximal="wvltADMM", u=1e-3, wvlt_levels=5)
    st = model.reconstruct(dx, dI, dm, iterations=10, **kw)
    fw = lambda x: oracle.forward(g, x)
    bw = lambda y: oracle.backward(g, y.reshape(g.np, g.prjWidth))
    xo, Io, so = LO.reconstruct(fw, bw, k, Ts, np.ones((g.n, g.n)), np.full(20, 1.0 / 20),
                                m.astype(np.float64), 10, noise="gaussian", **kw)
    c, co = np.array(st["cost"]), np.array(so["cost"])
    steps_equal = np.allclose(st["x_step"], so["x_step"], rtol=1e-12, atol=0)
    print("wvlt loop gaussian: max cost rel %.2e, x rel %.2e, steps equal %s" % (
        float(np.max(np.abs(c - co) / np.abs(co))), rel(dx.cpu().numpy(), xo), steps_equal))
    assert steps_equal
    assert float(np.max(np.abs(c - co) / np.abs(co))) < 1e-3
    assert rel(dx.cpu().numpy(), xo) < 1e-3

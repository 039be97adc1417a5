"""GPU parity of the polychromatic model: the fused forward (projection with
the per-ray spline epilogue) and its hand-written adjoint, through the C ABI,
against the FP64 oracle (oracle/bhc_oracle.py over the FP64 projector
restatement), the unfused path and central finite differences.

Tolerances: f within 1e-6 relative of the FP64 oracle (FP32 projections, FP64
everything after); df/dx and df/dIe within 1e-5 relative L2.  df/dIe_j sums
b_j(s_i) (1 - m_i/BL_i) over rays where 1 - m/BL is a difference of nearly
equal numbers at high counts, so the FP32 projection's 1e-7 error reaches its
smallest components at ~1e-4 relative while the vector stays near 1e-6."""
import numpy as np
import pytest

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


def problem(g, J=20, seed=0, I0=1e5):
    """Two-material phantom, spectrum bump, Poisson counts at I0 per ray."""
    Ts = 2.0 / g.n                        # a 2 cm field of view
    x = phantom.two_material_phantom(g.n, seed=seed)
    k = BO.kappa_nodes(J)
    Ie = BO.spectrum_bump(J, seed)
    s = Ts * oracle.forward(g, x.astype(np.float64))
    BL, _, _ = BO.b1_iout(k, s.ravel(), Ie)
    rng = np.random.default_rng(seed + 100)
    m = (rng.poisson(I0 * BL) / I0).reshape(g.np, g.prjWidth)
    return x, k, Ie, m, Ts


def oracle_eval(g, x, k, Ie, m, Ts):
    s = Ts * oracle.forward(g, x.astype(np.float64))
    Bm, D, _ = BO.b1_basis(k, s.ravel())
    BL, sBL = Bm @ Ie, D @ Ie
    f = BO.poisson_terms(BL, m.ravel()).sum()
    r = 1 - m.ravel() / BL
    gx = Ts * oracle.backward(g, (r * sBL).reshape(g.np, g.prjWidth))
    gI = Bm.T @ r
    return f, gx, gI


GEOMS = {"fan": ct.Geometry(96, 136, 72, 72, 1.0, 1.0, 400.0),
         "par": ct.Geometry(97, 139, 60, 120, 1.0, 1.0, 0.0)}


@pytest.mark.parametrize("name", sorted(GEOMS))
def test_fused_forward_and_adjoint_match_fp64_oracle(name):
    g = GEOMS[name]
    x, k, Ie, m, Ts = problem(g)
    pr = ct.Projector(g)
    model = bhc.BHCModel(pr, k, Ts)
    dx = torch.from_numpy(x).cuda()
    dI = torch.from_numpy(Ie).cuda()
    dm = torch.from_numpy(m.astype(np.float32)).cuda()
    f = model.forward(dx, dI, dm).item()
    gx, gI = model.backward()
    fo, gxo, gIo = oracle_eval(g, x, k, Ie, m.astype(np.float32).astype(np.float64), Ts)
    assert abs(f - fo) <= 1e-6 * abs(fo)
    assert rel(gx.cpu().numpy(), gxo) < 1e-5
    assert rel(gI.cpu().numpy(), gIo) < 1e-5
    print("bhc %s: f rel %.2e, grad_x rel %.2e, grad_Ie rel %.2e" % (
        name, abs(f - fo) / abs(fo), rel(gx.cpu().numpy(), gxo), rel(gI.cpu().numpy(), gIo)))


def test_fused_forward_and_adjoint_match_fp64_oracle_at_the_1024_configuration():
    """The polychromatic model's own configuration: fan 1024^2, 720 views over
    [0, 2 pi), 1024 detectors, source 2048 px from the isocentre, J = 20,
    two-material phantom, Poisson counts at I0 = 1e5 of the FP64 oracle's
    intensity, against the FP64 oracle (the FP64 projector restatement and
    oracle/bhc_oracle.py; bhc/poissLAlpha.m:1-19, bhc/poissLI.m:1-27).

    f within 1e-6 and df/dx within 1e-5 relative L2.  df/dIe_j sums
    b_j(s_i) (1 - m_i / BL_i) over 7.4e5 rays near the likelihood's optimum,
    where the terms nearly cancel: a projection bias of 3e-8 (half a float32
    unit) shared by all rays moves it by 6e-5 relative (the oracle's own
    sensitivity, |sum_i |b_ij| |dBL/ds| s_i / BL_i| / |df/dIe|, is about
    1900).  So df/dIe is checked twice: the FP64 epilogue on the GPU's own
    float32 projections must agree with the oracle's epilogue on the same
    projections to 1e-9, and against the all-FP64 oracle the error must stay
    below what a common projection bias of 1e-7 would cause."""
    g = ct.Geometry(1024, 1024, 720, 720, 1.0, 1.0, 2048.0)
    x, k, Ie, m, Ts = problem(g, J=20, seed=4)
    pr = ct.Projector(g)
    model = bhc.BHCModel(pr, k, Ts)
    dx = torch.from_numpy(x).cuda()
    dI = torch.from_numpy(Ie).cuda()
    m32 = m.astype(np.float32)
    dm = torch.from_numpy(m32).cuda()
    f = model.forward(dx, dI, dm).item()
    gx, gI = model.backward()
    gI = gI.cpu().numpy()
    mo = m32.astype(np.float64).ravel()
    fo, gxo, gIo = oracle_eval(g, x, k, Ie, m32.astype(np.float64), Ts)
    ef, ex, eI = abs(f - fo) / abs(fo), rel(gx.cpu().numpy(), gxo), rel(gI, gIo)
    # the oracle's epilogue on the GPU's own float32 projections
    s_gpu = Ts * pr.forward(dx).double().cpu().numpy().ravel()
    Bm, D, _ = BO.b1_basis(k, s_gpu)
    BL = Bm @ Ie
    eI_same = rel(gI, Bm.T @ (1 - mo / BL))
    # sensitivity of df/dIe to a relative projection bias shared by all rays
    s_o = Ts * oracle.forward(g, x.astype(np.float64)).ravel()
    Bo, Do, _ = BO.b1_basis(k, s_o)
    BLo = Bo @ Ie
    amp = np.linalg.norm(np.abs(Bo.T) @ (np.abs(Do @ Ie) / BLo * s_o)) / np.linalg.norm(gIo)
    print("bhc fan 1024^2 / 720 views: f rel %.2e, grad_x rel %.2e, grad_Ie rel %.2e (same projections "
          "%.2e; sensitivity %.0f: equivalent projection bias %.1e)" % (ef, ex, eI, eI_same, amp, eI / amp))
    assert ef <= 1e-6
    assert ex < 1e-5
    assert eI_same < 1e-9
    assert eI < 1e-7 * amp


def test_fused_equals_unfused_and_recompute_equals_store():
    g = GEOMS["fan"]
    x, k, Ie, m, Ts = problem(g, J=30, seed=2)
    pr = ct.Projector(g)
    model = bhc.BHCModel(pr, k, Ts)
    dx = torch.from_numpy(x).cuda()
    dI = torch.from_numpy(Ie).cuda()
    dm = torch.from_numpy(m.astype(np.float32)).cuda()
    f1 = model.forward(dx, dI, dm, save=True).item()
    gx1, gI1 = model.backward()
    sino = pr.forward(dx)
    f2 = model.terms(sino, dI, dm, save=True).item()
    gx2, gI2 = model.backward()
    assert abs(f1 - f2) <= 1e-12 * abs(f1)
    assert torch.equal(gx1, gx2)
    assert rel(gI1.cpu().numpy(), gI2.cpu().numpy()) < 1e-13
    f3 = model.forward(dx, dI, dm, save=False).item()
    gx3, gI3 = model.backward(dx, dI, dm)
    assert f3 == f1
    assert torch.equal(gx3, gx1)
    assert rel(gI3.cpu().numpy(), gI1.cpu().numpy()) < 1e-13


def test_central_finite_differences():
    """32 seeded directions, step h = 1e-3 relative (density) and 1e-4
    relative per coefficient (spectrum: direction d_j = Ie_j z_j, z ~ N(0,1),
    so that the near-zero tail coefficients are not pushed through zero)."""
    g = GEOMS["fan"]
    x, k, Ie, m, Ts = problem(g, seed=3)
    pr = ct.Projector(g)
    model = bhc.BHCModel(pr, k, Ts)
    dx = torch.from_numpy(x).cuda()
    dI = torch.from_numpy(Ie).cuda()
    dm = torch.from_numpy(m.astype(np.float32)).cuda()
    model.forward(dx, dI, dm)
    gx, gI = model.backward()
    gx = gx.double()
    rng = np.random.default_rng(9)
    f = lambda xx, II: model.forward(xx, II, dm, save=False).item()
    errs = []
    for _ in range(32):
        d = torch.from_numpy(rng.standard_normal((g.n, g.n)).astype(np.float32)).cuda()
        h = 1e-3 * (torch.linalg.norm(dx) / torch.linalg.norm(d)).item()
        fd = (f(dx + h * d, dI) - f(dx - h * d, dI)) / (2 * h)
        an = (gx * d.double()).sum().item()
        errs.append(abs(fd - an) / (torch.linalg.norm(gx) * torch.linalg.norm(d.double())).item())
    assert max(errs) < 2e-3, max(errs)
    errI = []
    for _ in range(32):
        d = dI * torch.from_numpy(rng.standard_normal(Ie.size)).cuda()
        h = 1e-4
        fd = (f(dx, dI + h * d) - f(dx, dI - h * d)) / (2 * h)
        an = (gI * d).sum().item()
        errI.append(abs(fd - an) / (torch.linalg.norm(gI) * torch.linalg.norm(d)).item())
    assert max(errI) < 1e-5, max(errI)
    print("bhc finite differences: max rel err density %.2e, spectrum %.2e" % (max(errs), max(errI)))


def test_basis_matrix_and_reference_call_structure():
    """The materialised basis matrix (Spline.b1Iout with I empty) matches the
    oracle, and the spectrum gradient formed the reference's way,
    A^T (1 - m / (A Ie)) (bhc/poissLI.m:2-6), equals the fused one."""
    g = GEOMS["fan"]
    x, k, Ie, m, Ts = problem(g, J=30, seed=5)
    pr = ct.Projector(g)
    model = bhc.BHCModel(pr, k, Ts)
    dx = torch.from_numpy(x).cuda()
    dI = torch.from_numpy(Ie).cuda()
    dm = torch.from_numpy(m.astype(np.float32)).cuda()
    sino = pr.forward(dx)
    A = model.basis(sino)
    s = Ts * sino.double().cpu().numpy().ravel()
    Bo, _, _ = BO.b1_basis(k, s)
    assert rel(A.cpu().numpy(), Bo) < 1e-12
    Ir = A @ dI
    gI_ref = A.t() @ (1 - dm.double().ravel() / Ir)
    model.forward(dx, dI, dm)
    _, gI = model.backward(grad_x=False)
    assert rel(gI.cpu().numpy(), gI_ref.cpu().numpy()) < 1e-6


def test_finite_differences_at_the_1024_configuration():
    """The polychromatic model's own configuration (fan 1024^2, 720 views over
    [0, 2 pi), 1024 detectors, J = 20, Poisson counts at I0 = 1e5): f and both
    gradients against central differences on 32 seeded directions, h = 1e-3
    relative for the density, 1e-6 relative per coefficient for the spectrum:
    with 7.4e5 rays the third derivative in Ie grows with the ray count while
    the gradient, a sum of residuals, grows with its square root, so at 1e-4
    the truncation alone is ~1e-4 of the gradient (3e-5 for the FP64 oracle on
    the same problem); at 1e-6 it is far below FP64 rounding of f."""
    g = ct.Geometry(1024, 1024, 720, 720, 1.0, 1.0, 2048.0)
    Ts = 2.0 / g.n
    x = phantom.two_material_phantom(g.n, seed=7)
    k = BO.kappa_nodes(20)
    Ie = BO.spectrum_bump(20, 7)
    pr = ct.Projector(g)
    model = bhc.BHCModel(pr, k, Ts)
    dx = torch.from_numpy(x).cuda()
    dI = torch.from_numpy(Ie).cuda()
    A = model.basis(pr.forward(dx))
    BL = (A @ dI).reshape(g.np, g.prjWidth)
    gen = torch.Generator(device="cuda").manual_seed(11)
    dm = (torch.poisson(1e5 * BL, generator=gen) / 1e5).float().contiguous()
    del A, BL
    model.forward(dx, dI, dm)
    gx, gI = model.backward()
    gx = gx.double()
    rng = np.random.default_rng(12)
    f = lambda xx, II: model.forward(xx, II, dm, save=False).item()
    errs, errI = [], []
    for _ in range(32):
        d = torch.from_numpy(rng.standard_normal((g.n, g.n)).astype(np.float32)).cuda()
        h = 1e-3 * (torch.linalg.norm(dx) / torch.linalg.norm(d)).item()
        fd = (f(dx + h * d, dI) - f(dx - h * d, dI)) / (2 * h)
        errs.append(abs(fd - (gx * d.double()).sum().item())
                    / (torch.linalg.norm(gx) * torch.linalg.norm(d.double())).item())
        dd = dI * torch.from_numpy(rng.standard_normal(Ie.size)).cuda()
        fdI = (f(dx, dI + 1e-6 * dd) - f(dx, dI - 1e-6 * dd)) / 2e-6
        errI.append(abs(fdI - (gI * dd).sum().item()) / (torch.linalg.norm(gI) * torch.linalg.norm(dd)).item())
    print("bhc finite differences at 1024^2: max rel err density %.2e, spectrum %.2e" % (max(errs), max(errI)))
    assert max(errs) < 5e-3
    assert max(errI) < 1e-5

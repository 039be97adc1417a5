"""The projector in MATLAB's layout with ConfigCT's mask on the device
(include/ctprj_masked.h): the operators of tomography/ConfigCT.m:122-135
against the same composition done on the host around the gateway mirror
(utils/maskFunc.m + prj/mPrj.c conventions), bit for bit, plus adjointness and
the FP64 oracle."""
import numpy as np
import pytest

import oracle

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

import imgrecsrc_b200 as ct  # noqa: E402
from imgrecsrc_b200 import mex  # noqa: E402


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


def conf_of(g):
    return {"n": g.n, "prjWidth": g.prjWidth, "np": g.np, "prjFull": g.prjFull,
            "dSize": g.dSize, "effectiveRate": g.effectiveRate, "d": g.d}


def disc_mask(n):
    r = np.arange(n) - (n - 1) / 2
    return (r[:, None] ** 2 + r[None, :] ** 2 <= (0.45 * n) ** 2).astype(np.uint8)


@pytest.mark.parametrize("g", [ct.Geometry(96, 136, 72, 72, 1.0, 1.0, 400.0),
                               ct.Geometry(81, 117, 46, 92, 1.0, 1.0, 0.0)])
@pytest.mark.parametrize("masked", [False, True])
def test_device_operators_equal_the_host_composition(g, masked):
    Ts = 0.0125
    rng = np.random.default_rng(5)
    pr = ct.Projector(g)
    mask = disc_mask(g.n) if masked else None
    Phi, Phit, FBP = mex.gpuFanParOps(pr, mask, Ts)
    idx = (np.flatnonzero(mask.ravel(order="F")) if masked else np.arange(g.n * g.n))
    s = rng.standard_normal(idx.size)
    y = rng.standard_normal(g.np * g.prjWidth)
    dev = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
    phi = Phi(dev(s)).cpu().numpy()
    phit = Phit(dev(y)).cpu().numpy()
    fbp = FBP(dev(y)).cpu().numpy()
    # the host composition: maskFunc then the gateway, as ConfigCT does
    mex.gpuPrj(0, conf_of(g), "config")
    x = np.zeros(g.n * g.n)
    x[idx] = s                                   # x(maskIdx) = s, column-major
    ref_phi = mex.gpuPrj(x, 0, "forward") * Ts
    ref_phit = mex.gpuPrj(y, 0, "backward")[idx] * Ts
    ref_fbp = mex.gpuPrj(y, 0, "FBP")[idx] / Ts
    assert np.array_equal(phi, ref_phi)
    assert np.array_equal(phit, ref_phit)
    assert np.array_equal(fbp, ref_fbp)
    # adjoint pair, and the FP64 oracle on the scattered image
    lhs, rhs = phi @ y, s @ phit
    assert abs(lhs - rhs) <= 1e-6 * np.linalg.norm(phi) * np.linalg.norm(y)
    img = x.reshape(g.n, g.n, order="F").astype(np.float32).astype(np.float64)
    so = Ts * oracle.forward(g, img).ravel()
    assert np.linalg.norm(phi - so) / np.linalg.norm(so) < 1e-5


def test_bad_arguments_are_rejected():
    g = ct.Geometry(64, 91, 30, 60, 1.0, 1.0, 0.0)
    pr = ct.Projector(g)
    L = ct.lib()
    buf = torch.zeros(g.n * g.n, dtype=torch.float64, device="cuda")
    y = torch.zeros(g.np * g.prjWidth, dtype=torch.float64, device="cuda")
    import ctypes
    st = L.ctprj_masked_forward(pr._plan, None, g.n * g.n - 1, ctypes.c_void_p(buf.data_ptr()), 1.0,
                                ctypes.c_void_p(y.data_ptr()), None)
    assert st == 1   # CTPRJ_EINVAL: without a mask npix must be n*n

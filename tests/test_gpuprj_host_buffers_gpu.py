"""The reference-compatible gpuPrj() with pageable host buffers (what the
reference's MATLAB gateway passes, prj/mPrj.c:70-73) and with pinned ones:
the results are equal bit for bit in both directions, and equal the device
path's."""
import ctypes

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

import imgrecsrc_b200 as ct  # noqa: E402
from imgrecsrc_b200 import phantom  # noqa: E402


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


def test_pageable_equals_pinned():
    L = ct.lib()
    n, W, npv = 1800, 1999, 1440                    # 13.0 MB image, 11.5 MB sinogram
    L.setup(n, W, npv, npv, 1.0, 1.0, 7000.0)
    rng = np.random.default_rng(4)
    img_u = phantom.ellipse_phantom(n, seed=4)
    sino_u = np.empty((npv, W), np.float32)
    y_u = rng.standard_normal((npv, W)).astype(np.float32)
    back_u = np.empty((n, n), np.float32)
    img_p = torch.from_numpy(img_u).pin_memory()
    sino_p = torch.empty(npv, W).pin_memory()
    y_p = torch.from_numpy(y_u).pin_memory()
    back_p = torch.empty(n, n).pin_memory()
    c = lambda a: ctypes.c_void_p(a.ctypes.data if isinstance(a, np.ndarray) else a.data_ptr())
    ct.check(L.gpuPrj(c(img_u), c(sino_u), bytes([ct.FWD_BIT])))
    ct.check(L.gpuPrj(c(img_p), c(sino_p), bytes([ct.FWD_BIT])))
    assert np.array_equal(sino_u, sino_p.numpy())
    ct.check(L.gpuPrj(c(back_u), c(y_u), bytes([ct.BWD_BIT])))
    ct.check(L.gpuPrj(c(back_p), c(y_p), bytes([ct.BWD_BIT])))
    assert np.array_equal(back_u, back_p.numpy())
    # and the device path agrees
    pr = ct.Projector(ct.Geometry(n, W, npv, npv, 1.0, 1.0, 7000.0))
    assert np.array_equal(pr.forward(torch.from_numpy(img_u).cuda()).cpu().numpy(), sino_u)

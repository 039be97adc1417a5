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


def _ptr(a):
    return ctypes.c_void_p(a.ctypes.data if isinstance(a, np.ndarray) else a.data_ptr())


def test_mixed_buffers_fbp_and_a_new_setup():
    """Pageable input with a pinned result and the other way round, FBP, and
    a second setup() with larger buffers (the staging buffer of pageable calls
    grows with it): every combination gives the pinned path's bits."""
    L = ct.lib()
    rng = np.random.default_rng(9)
    for n, W, npv, d in ((300, 431, 240, 900.0), (1100, 1500, 720, 4000.0)):
        L.setup(n, W, npv, npv, 1.0, 1.0, d)
        img_u = phantom.ellipse_phantom(n, seed=n)
        y_u = rng.standard_normal((npv, W)).astype(np.float32)
        img_p, y_p = torch.from_numpy(img_u).pin_memory(), torch.from_numpy(y_u).pin_memory()
        ref_s, ref_b, ref_f = torch.empty(npv, W).pin_memory(), torch.empty(n, n).pin_memory(), torch.empty(n, n).pin_memory()
        ct.check(L.gpuPrj(_ptr(img_p), _ptr(ref_s), bytes([ct.FWD_BIT])))
        ct.check(L.gpuPrj(_ptr(ref_b), _ptr(y_p), bytes([ct.BWD_BIT])))
        ct.check(L.gpuPrj(_ptr(ref_f), _ptr(y_p), bytes([ct.FBP_BIT])))
        for src_img, src_y in ((img_u, y_p), (img_p, y_u), (img_u, y_u)):
            for pinned_out in (False, True):
                s_out = torch.empty(npv, W).pin_memory() if pinned_out else np.full((npv, W), np.nan, np.float32)
                b_out = torch.empty(n, n).pin_memory() if pinned_out else np.full((n, n), np.nan, np.float32)
                f_out = torch.empty(n, n).pin_memory() if pinned_out else np.full((n, n), np.nan, np.float32)
                ct.check(L.gpuPrj(_ptr(src_img), _ptr(s_out), bytes([ct.FWD_BIT])))
                ct.check(L.gpuPrj(_ptr(b_out), _ptr(src_y), bytes([ct.BWD_BIT])))
                ct.check(L.gpuPrj(_ptr(f_out), _ptr(src_y), bytes([ct.FBP_BIT])))
                as_np = lambda a: a.numpy() if isinstance(a, torch.Tensor) else a
                assert np.array_equal(as_np(s_out), ref_s.numpy()), (n, pinned_out)
                assert np.array_equal(as_np(b_out), ref_b.numpy()), (n, pinned_out)
                assert np.array_equal(as_np(f_out), ref_f.numpy()), (n, pinned_out)

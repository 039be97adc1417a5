"""The wavelet regulariser over torch tensors (include/ctprj_wavelet.h): the
GPU counterparts of the Rice Wavelet Toolbox transforms mdwt / midwt that the
reference vendors (rwt/), its Daubechies filter design daubcqf, and the ADMM
proximal map npg/admm.m behind the reference's default density-step
regulariser ('wvltADMM', bhc/beamhardenSpline.m:205-209).

Images are 2-D float32 CUDA tensors indexed [row, column] like the MATLAB
matrices the reference transforms; rows and columns must be divisible by
2^L.
"""
import ctypes
import math

import numpy as np

from ._lib import check, lib
from .projector import _stream_handle


def daubcqf(N):
    """Minimum-phase Daubechies scaling filter of even length N, normalised to
    sum sqrt(2) (rwt/daubcqf.m with TYPE 'min'): the binomial half-band
    polynomial's factor from its N/2 - 1 roots of smallest modulus."""
    if N < 2 or N % 2:
        raise ValueError("Daubechies filters have even length >= 2")
    K = N // 2
    a, h0, p, q = 1.0, np.array([1.0, 1.0]), np.array([1.0]), np.array([1.0])
    for j in range(1, K):
        a = -a * 0.25 * (j + K - 1) / j
        h0 = np.append(0.0, h0) + np.append(h0, 0.0)
        p = np.append(0.0, -p) + np.append(p, 0.0)
        p = np.append(0.0, -p) + np.append(p, 0.0)
        q = np.concatenate(([0.0], q, [0.0])) + a * p
    if K > 1:
        roots = sorted(np.roots(q), key=lambda z: (abs(z), np.angle(z)))
        h0 = np.convolve(h0, np.real(np.poly(roots[:K - 1])))
    return math.sqrt(2.0) * h0 / h0.sum()


def _img(x):
    import torch
    if not (isinstance(x, torch.Tensor) and x.is_cuda and x.dtype == torch.float32 and x.is_contiguous()
            and x.dim() == 2):
        raise TypeError("expected a contiguous 2-D CUDA float32 tensor")
    return x


def _filt(h):
    h = np.ascontiguousarray(h, np.float64)
    return h, h.ctypes.data, len(h)


def _vp(t):
    return ctypes.c_void_p(t.data_ptr())


def mdwt(x, h, L, stream=None):
    """y = mdwt(x, h, L)."""
    import torch
    x = _img(x)
    hh, hp, lh = _filt(h)
    y = torch.empty_like(x)
    check(lib().ctprj_dwt(_vp(x), x.shape[0], x.shape[1], hp, lh, int(L), _vp(y),
                          _stream_handle(stream, x.device.index)))
    return y


def midwt(y, h, L, stream=None):
    """x = midwt(y, h, L)."""
    import torch
    y = _img(y)
    hh, hp, lh = _filt(h)
    x = torch.empty_like(y)
    check(lib().ctprj_idwt(_vp(y), y.shape[0], y.shape[1], hp, lh, int(L), _vp(x),
                           _stream_handle(stream, y.device.index)))
    return x


def l1(x, h, L, stream=None):
    """pNorm(Psit(x), 1) in FP64."""
    import torch
    x = _img(x)
    hh, hp, lh = _filt(h)
    out = torch.zeros(1, dtype=torch.float64, device=x.device)
    check(lib().ctprj_wvlt_l1(_vp(x), x.shape[0], x.shape[1], hp, lh, int(L), _vp(out),
                              _stream_handle(stream, x.device.index)))
    return float(out.item())


def admm(a, u, h, L, relative_tol=1e-6, max_itr=1000, init=None, stream=None):
    """[alpha, pppp] = admm(Psi, Psit, a, u, relativeTol, maxItr, false, init)
    (npg/admm.m) with Psi / Psit the L-level transforms of filter h.
    Returns (alpha, iterations)."""
    import torch
    a = _img(a)
    if init is not None:
        init = _img(init)
    hh, hp, lh = _filt(h)
    out = torch.empty_like(a)
    it = ctypes.c_int(0)
    check(lib().ctprj_wvlt_admm(_vp(a), a.shape[0], a.shape[1], hp, lh, int(L), float(u), float(relative_tol),
                                int(max_itr), _vp(init) if init is not None else None, _vp(out),
                                ctypes.byref(it), _stream_handle(stream, a.device.index)))
    return out, it.value


def get_psi_psit(daub, L):
    """(Psi, Psit) = Utils.getPsiPsit(daub, dwt_L) without masks
    (utils/Utils.m:445-469): Psi = midwt(., daubcqf(daub), L), Psit = mdwt."""
    h = daubcqf(daub)
    return (lambda s: midwt(s, h, L)), (lambda x: mdwt(x, h, L))


def wvlt_mask(mask, h, L, stream=None):
    """maskk = wvltMask(mask, L, daub) (utils/wvltMask.m): the coefficients of
    the L-level transform of filter h that a pixel of mask reaches, as a
    uint8 CUDA tensor of the mask's shape."""
    import torch
    m = (mask != 0).to(torch.uint8).contiguous()
    if not m.is_cuda or m.dim() != 2:
        raise TypeError("expected a 2-D CUDA mask")
    hh, hp, lh = _filt(h)
    out = torch.empty_like(m)
    check(lib().ctprj_wvlt_mask(_vp(m), m.shape[0], m.shape[1], hp, lh, int(L), _vp(out),
                                _stream_handle(stream, m.device.index)))
    return out

"""The total-variation proximal map over torch tensors (include/ctprj_tv.h),
the GPU counterpart of the reference's TV.denoise (utils/TV.m:56-80, through
utils/denoise_bound_mod.m) and tlv (utils/tlv.m).

The reference calls them on MATLAB arrays, column-major: a vector x of
nRow * nCol values (or of the pixels of a mask) reshaped to nRow x nCol.
The same memory read row-major is nCol x nRow, and the iteration treats both
axes alike, so the vectors here are passed to the kernels as they lie.
"""
import ctypes
import math

from ._lib import check, lib
from .projector import _stream_handle

TV_TYPES = {"iso": 0, "l1": 1}


def _flat_f32(x):
    import torch
    if not (isinstance(x, torch.Tensor) and x.is_cuda and x.dtype == torch.float32 and x.is_contiguous()):
        raise TypeError("expected a contiguous CUDA float32 tensor")
    return x


def denoise(x, u, inner_thresh=1e-4, max_inner_itr=100, mask=None, tv_type="iso", lb=0.0, ub=math.inf,
            n_row=None, n_col=None, stream=None):
    """[newX, innerSearch] = TV.denoise(x, u, innerThresh, maxInnerItr, maskmt,
    tvType, init, lb, ub, nRow, nCol): argmin_X ||X - x||^2 + 2 u TV(X) over
    lb <= X <= ub, X of the shape of x.  mask: None, or a boolean CUDA tensor
    whose column-major nonzeros (MATLAB's find(maskmt ~= 0)) are the pixels
    of the vector x; the pixels outside it enter as zeros, as maskFunc makes
    them.  Returns (newX, iterations)."""
    import torch
    x = _flat_f32(x)
    if mask is not None:
        mt = mask.t().contiguous().reshape(-1) != 0        # column-major order of the mask
        idx = torch.nonzero(mt).squeeze(1)
        if idx.numel() != x.numel():
            raise ValueError("x has %d values, the mask %d pixels" % (x.numel(), idx.numel()))
        n_col, n_row = mask.shape[1], mask.shape[0]
        img = torch.zeros(n_row * n_col, dtype=torch.float32, device=x.device)
        img[idx] = x.reshape(-1)
    else:
        img = x.reshape(-1)
        if n_row is None:
            n_row = int(round(math.sqrt(img.numel())))
        if n_col is None:
            n_col = img.numel() // n_row
        if n_row * n_col != img.numel():
            raise ValueError("nRow * nCol = %d, x has %d values" % (n_row * n_col, img.numel()))
    out = torch.empty_like(img)
    it = ctypes.c_int(0)
    # column-major nRow x nCol = row-major nCol x nRow
    check(lib().ctprj_tv_denoise(ctypes.c_void_p(img.data_ptr()), int(n_col), int(n_row), float(u), float(lb),
                                 float(ub), TV_TYPES[tv_type], int(max_inner_itr), float(inner_thresh),
                                 ctypes.c_void_p(out.data_ptr()), ctypes.byref(it),
                                 _stream_handle(stream, x.device.index)))
    if mask is not None:
        return out[idx].reshape(x.shape), it.value
    return out.reshape(x.shape), it.value


def tlv(x, tv_type="iso", n_row=None, n_col=None, stream=None):
    """tlv(X, type) of a 2-D image (or a vector read as column-major
    nRow x nCol), in FP64."""
    import torch
    x = _flat_f32(x)
    if x.dim() == 2 and n_row is None:
        rows, cols = x.shape                      # row-major 2-D tensor as it is
    else:
        n = x.numel()
        n_row = n_row or int(round(math.sqrt(n)))
        n_col = n_col or n // n_row
        rows, cols = n_col, n_row
    out = torch.zeros(1, dtype=torch.float64, device=x.device)
    check(lib().ctprj_tv_value(ctypes.c_void_p(x.data_ptr()), int(rows), int(cols), TV_TYPES[tv_type],
                               ctypes.c_void_p(out.data_ptr()), _stream_handle(stream, x.device.index)))
    return float(out.item())

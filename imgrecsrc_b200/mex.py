"""Host mirror of the reference's MATLAB operator interface.

``gpuPrj(x, conf, cmd)`` follows the MEX gateway prj/mPrj.c:37-173 (built by
the reference as gpuPrj.mex): ``cmd`` is 'config' (conf carries the fields n,
prjWidth, np, prjFull, dSize, effectiveRate, d), 'forward', 'backward', 'FBP',
or anything else to print the configuration.  Arrays are taken and returned
with MATLAB's meaning: an image argument is the n x n matrix (rows are y),
passed as a 2-D array or as its column-major vector; a sinogram is the
prjWidth*np vector, view after view.  Results are float64 vectors, as the MEX
function returns, in MATLAB's column-major order.  The work runs through the C
ABI's setup()/gpuPrj() on the GPU; there is no CPU path.
"""
import ctypes

import numpy as np

from ._lib import BWD_BIT, FBP_BIT, FWD_BIT, ParConf, check, lib

_conf = None


def _field(conf, name):
    return conf[name] if isinstance(conf, dict) else getattr(conf, name)


def _image_in(x, n):
    a = np.asarray(x)
    if a.ndim == 2:
        return np.ascontiguousarray(a, dtype=np.float32)
    # a MATLAB column-major vector of the n x n matrix (prj/mPrj.c:82-84)
    return np.ascontiguousarray(a.reshape(n, n, order="F"), dtype=np.float32)


def gpuPrj(x, conf, cmd):
    global _conf
    L = lib()
    if cmd == "config":
        vals = [_field(conf, k) for k in ("n", "prjWidth", "np", "prjFull", "dSize",
                                          "effectiveRate", "d")]
        L.setup(int(vals[0]), int(vals[1]), int(vals[2]), int(vals[3]), float(vals[4]),
                float(vals[5]), float(vals[6]))
        _conf = dict(zip(("n", "prjWidth", "np", "prjFull", "dSize", "effectiveRate", "d"), vals))
        return None
    if _conf is None:
        raise RuntimeError("gpuPrj: call with 'config' first")
    n, W, npv = int(_conf["n"]), int(_conf["prjWidth"]), int(_conf["np"])
    if cmd == "forward":
        img = _image_in(x, n)
        sino = np.zeros((npv, W), np.float32)
        check(L.gpuPrj(img.ctypes.data, sino.ctypes.data, bytes([FWD_BIT])))
        return sino.astype(np.float64).ravel()
    if cmd in ("backward", "FBP"):
        sino = np.ascontiguousarray(np.asarray(x, dtype=np.float32).ravel())
        if sino.size != npv * W:
            raise ValueError("expected a sinogram of %d values" % (npv * W))
        img = np.zeros((n, n), np.float32)
        bit = BWD_BIT if cmd == "backward" else FBP_BIT
        check(L.gpuPrj(img.ctypes.data, sino.ctypes.data, bytes([bit])))
        # column-major vector of the image matrix (prj/mPrj.c:134-136)
        return img.astype(np.float64).ravel(order="F")
    L.showSetup()
    return None


def mParPrj(x, maskIdx, conf, cmd):
    """The MEX function mParPrj(x, maskIdx, conf, cmd) of prj/mParPrj.c:26-74:
    the double-precision parallel-beam operator over the angles conf.theta
    (degrees) and the 0-based column-major pixel indices maskIdx of an
    conf.nr x conf.nc image, beam width conf.bw, conf.prjWidth detectors.
    'forward' maps one value per mask entry to np*prjWidth values; any other
    command is the backprojection.  Returns a float64 vector."""
    theta = np.ascontiguousarray(_field(conf, "theta"), np.float64).ravel()
    mask = np.ascontiguousarray(maskIdx, np.float64).ravel()
    x = np.ascontiguousarray(x, np.float64).ravel()
    W = int(_field(conf, "prjWidth"))
    fwd = cmd == "forward"
    pc = ParConf(float(_field(conf, "bw")), int(_field(conf, "nc")), int(_field(conf, "nr")),
                 theta.size, W, theta.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                 1 if fwd else 0)
    if fwd:
        img, prj = x, np.zeros(theta.size * W, np.float64)     # mxCreateDoubleMatrix zeros
        out = prj
    else:
        if x.size != theta.size * W:
            raise ValueError("expected %d sinogram values" % (theta.size * W))
        img, prj = np.zeros(mask.size, np.float64), x.copy()
        out = img
    L = lib()
    check(L.parPrjConf(img.ctypes.data, prj.ctypes.data, mask.ctypes.data, ctypes.byref(pc),
                       mask.size))
    check(L.parPrjThread())
    return out


def gpuFanParOps(projector, mask=None, Ts=1.0):
    """Phi, Phit and FBP of ConfigCT.gpuFanParOps (tomography/ConfigCT.m:122-135)
    with its mask (utils/maskFunc.m), as device operators on float64 torch
    tensors in MATLAB's layout:
      Phi(s)  = Ts * gpuPrj(maskFunc(s, maskIdx, [n n]), 0, 'forward')
      Phit(y) = Ts * maskFunc(gpuPrj(y, 0, 'backward'), maskIdx)
      FBP(y)  = maskFunc(gpuPrj(y, 0, 'FBP'), maskIdx) / Ts
    mask: an n x n array (nonzero = reconstructed pixel, MATLAB's rows and
    columns) or None for the whole image.  s is the vector of masked pixels in
    column-major order, y the view-major sinogram vector.  The scatter, gather,
    transposes and casts run as kernels (include/ctprj_masked.h)."""
    import torch

    from ._lib import lib as _l
    g = projector.geometry
    dev = torch.device("cuda", projector.device)
    if mask is None:
        d_mask, npix = None, g.n * g.n
    else:
        m = np.asarray(mask)
        idx = np.flatnonzero(m.ravel(order="F")).astype(np.int32)   # find(mask ~= 0) - 1
        d_mask = torch.from_numpy(idx).to(dev)
        npix = int(idx.size)
    nsino = g.np * g.prjWidth
    mptr = None if d_mask is None else ctypes.c_void_p(d_mask.data_ptr())

    def _vec(t, size):
        if t.dtype != torch.float64 or t.device != dev or t.numel() != size or not t.is_contiguous():
            raise ValueError("expected a contiguous float64 CUDA vector of %d values" % size)
        return ctypes.c_void_p(t.data_ptr())

    def _stream():
        return ctypes.c_void_p(torch.cuda.current_stream(dev).cuda_stream)

    def Phi(s):
        y = torch.empty(nsino, dtype=torch.float64, device=dev)
        check(_l().ctprj_masked_forward(projector._plan, mptr, npix, _vec(s, npix), float(Ts),
                                        _vec(y, nsino), _stream()))
        return y

    def Phit(y):
        s = torch.empty(npix, dtype=torch.float64, device=dev)
        check(_l().ctprj_masked_backward(projector._plan, mptr, npix, _vec(y, nsino), float(Ts),
                                         _vec(s, npix), _stream()))
        return s

    def FBP(y):
        s = torch.empty(npix, dtype=torch.float64, device=dev)
        check(_l().ctprj_masked_fbp(projector._plan, mptr, npix, _vec(y, nsino), 1.0 / float(Ts),
                                    _vec(s, npix), _stream()))
        return s

    Phi.mask = d_mask
    return Phi, Phit, FBP

"""The oracle -- TEST INFRASTRUCTURE ONLY.

CPU restatements of the reference (anindyabijoydas/imgRecSrc) hot path, used as
the checker by ``tests/``, ``__graft_entry__.smoke()`` and the ``cpu_baseline``
leg of ``bench.py``.  The product package ``imgrecsrc_b200`` never imports this
package.

* ``ctprj_oracle.c``  projector restatement of prj/cpuPrj.c + prj/utils.h (FP64
  and FP32 builds), loaded here through ctypes.
* ``parprj_oracle.c`` restatement of prj/parPrj.c (mParPrj operator, FP64).
* ``bhc_oracle.py``   FP64 NumPy restatement of bhc/Spline.m (b1Iout),
  bhc/poissLAlpha.m and bhc/poissLI.m.
* ``ref``             the reference's own prj/cpuPrj.c and prj/parPrj.c,
  compiled unchanged into ``oracle/_ref`` when the reference sources are
  present (``make -C oracle ref REF=<reference>/prj``; the build functions
  below find the reference through the environment variable
  IMGRECSRC_REFERENCE); used to pin the restatements.

Geometry arguments are any object with the attributes of the reference's
``struct prjConf`` (prj/prj.h:42-57): n, prjWidth, np, prjFull, dSize,
effectiveRate, d.
"""
import ctypes
import os
import subprocess
import threading

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
BUILD = os.path.join(HERE, "_build")
REFDIR = os.path.join(HERE, "_ref")
_lock = threading.Lock()
_libs = {}


class _Geom(ctypes.Structure):
    _fields_ = [("n", ctypes.c_int), ("prjWidth", ctypes.c_int), ("np", ctypes.c_int),
                ("prjFull", ctypes.c_int), ("dSize", ctypes.c_double),
                ("effectiveRate", ctypes.c_double), ("d", ctypes.c_double),
                ("fbp", ctypes.c_int)]


class _ParConf(ctypes.Structure):
    _fields_ = [("bw", ctypes.c_double), ("nc", ctypes.c_int), ("nr", ctypes.c_int),
                ("np", ctypes.c_int), ("prjWidth", ctypes.c_int),
                ("theta", ctypes.POINTER(ctypes.c_double))]


def build():
    """Compiles the restatements (and, when the reference is present, its own
    sources) with oracle/Makefile."""
    subprocess.run(["make", "-s", "-C", HERE, "oracle"], check=True)


def reference_dir(sub):
    """<reference>/<sub> where the environment variable IMGRECSRC_REFERENCE
    names the reference project's root, else None."""
    root = os.environ.get("IMGRECSRC_REFERENCE")
    return os.path.join(root, sub) if root else None


def build_ref(ref_prj_dir=None):
    """The reference's own projector sources (<reference>/prj), compiled
    unchanged into oracle/_ref; False when they are not there."""
    ref_prj_dir = ref_prj_dir or reference_dir("prj")
    if not ref_prj_dir or not os.path.isdir(ref_prj_dir):
        return False
    subprocess.run(["make", "-s", "-C", HERE, "ref", "REF=" + ref_prj_dir], check=True)
    return True


def build_rwt(ref_rwt_dir=None):
    """The reference's vendored wavelet transform cores (rwt/mdwt_r.c,
    rwt/midwt_r.c), compiled unchanged into oracle/_ref/libref_rwt.so."""
    ref_rwt_dir = ref_rwt_dir or reference_dir("rwt")
    if not ref_rwt_dir or not os.path.isdir(ref_rwt_dir):
        return False
    subprocess.run(["make", "-s", "-C", HERE, "rwt", "RWT=" + ref_rwt_dir], check=True)
    return True


def build_gateways(ref_prj_dir=None):
    """The reference's own MEX gateways compiled against the engine library
    (oracle/Makefile target `gateways`), for the boundary tests."""
    ref_prj_dir = ref_prj_dir or reference_dir("prj")
    if not ref_prj_dir or not os.path.isdir(ref_prj_dir):
        return False
    subprocess.run(["make", "-s", "-C", HERE, "gateways", "REF=" + ref_prj_dir], check=True)
    return True


def _load(name, builder):
    with _lock:
        if name in _libs:
            return _libs[name]
        path = os.path.join(BUILD if name.startswith("liboracle") else REFDIR, name + ".so")
        if not os.path.exists(path):
            builder()
        lib = ctypes.CDLL(path)
        _libs[name] = lib
        return lib


def _olib(prec):
    lib = _load("liboracle_f%d" % prec, build)
    real = ctypes.c_double if prec == 64 else ctypes.c_float
    P = ctypes.c_void_p
    lib.ora_forward.argtypes = [ctypes.POINTER(_Geom), P, P, ctypes.c_int]
    lib.ora_backward.argtypes = [ctypes.POINTER(_Geom), P, P, ctypes.c_int]
    lib.ora_forward_nnz.argtypes = [ctypes.POINTER(_Geom), ctypes.c_int]
    lib.ora_forward_nnz.restype = ctypes.c_longlong
    lib.ora_backward_nnz.argtypes = [ctypes.POINTER(_Geom), ctypes.c_int]
    lib.ora_backward_nnz.restype = ctypes.c_longlong
    lib.ora_weight.argtypes = [real] * 4
    lib.ora_weight.restype = real
    lib.ora_par_forward.argtypes = [ctypes.POINTER(_ParConf), P, P, ctypes.c_longlong, P, ctypes.c_int]
    lib.ora_par_backward.argtypes = [ctypes.POINTER(_ParConf), P, P, ctypes.c_longlong, P, ctypes.c_int]
    return lib


def _geom(g, fbp=False):
    return _Geom(int(g.n), int(g.prjWidth), int(g.np), int(g.prjFull), float(g.dSize),
                 float(g.effectiveRate), float(g.d), 1 if fbp else 0)


def _dtype(prec):
    return np.float64 if prec == 64 else np.float32


def forward(g, img, prec=64, threads=0):
    """Sinogram (np, prjWidth) of the n x n image ``img`` (row-major, C order)."""
    dt = _dtype(prec)
    img = np.ascontiguousarray(img, dtype=dt).reshape(g.n, g.n)
    sino = np.zeros((g.np, g.prjWidth), dt)
    G = _geom(g)
    if _olib(prec).ora_forward(ctypes.byref(G), img.ctypes.data, sino.ctypes.data, threads):
        raise ValueError("invalid geometry")
    return sino


def backward(g, sino, prec=64, threads=0, fbp_weighting=False):
    """Backprojection (n, n) of the sinogram ``sino`` (np, prjWidth).  With
    ``fbp_weighting`` the FBP distance weights and scale are applied (the
    backprojection stage of FBP, without the filter)."""
    dt = _dtype(prec)
    sino = np.ascontiguousarray(sino, dtype=dt).reshape(g.np, g.prjWidth)
    img = np.zeros((g.n, g.n), dt)
    G = _geom(g, fbp_weighting)
    if _olib(prec).ora_backward(ctypes.byref(G), sino.ctypes.data, img.ctypes.data, threads):
        raise ValueError("invalid geometry")
    return img


def forward_nnz(g, threads=0):
    """Exact number of nonzero forward-operator entries (ray-pixel updates)."""
    G = _geom(g)
    return int(_olib(64).ora_forward_nnz(ctypes.byref(G), threads))


def backward_nnz(g, threads=0):
    G = _geom(g)
    return int(_olib(64).ora_backward_nnz(ctypes.byref(G), threads))


def weight(dist, bw, c, s, prec=64):
    return float(_olib(prec).ora_weight(dist, bw, c, s))


def _parconf(conf):
    theta = np.ascontiguousarray(conf["theta"], dtype=np.float64).ravel()
    pc = _ParConf(float(conf["bw"]), int(conf["nc"]), int(conf["nr"]), int(theta.size),
                  int(conf["prjWidth"]),
                  theta.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
    return pc, theta


def par_forward(x, mask_idx, conf, threads=0):
    """mParPrj(x, maskIdx, conf, 'forward') (prj/mParPrj.c): x has one value per
    0-based column-major mask index; returns np*prjWidth values (view-major)."""
    pc, theta = _parconf(conf)
    x = np.ascontiguousarray(x, dtype=np.float64).ravel()
    m = np.ascontiguousarray(mask_idx, dtype=np.float64).ravel()
    out = np.zeros(theta.size * int(conf["prjWidth"]), np.float64)
    _olib(64).ora_par_forward(ctypes.byref(pc), x.ctypes.data, m.ctypes.data, m.size,
                              out.ctypes.data, threads)
    return out


def par_backward(y, mask_idx, conf, threads=0):
    pc, theta = _parconf(conf)
    y = np.ascontiguousarray(y, dtype=np.float64).ravel()
    m = np.ascontiguousarray(mask_idx, dtype=np.float64).ravel()
    out = np.zeros(m.size, np.float64)
    _olib(64).ora_par_backward(ctypes.byref(pc), y.ctypes.data, m.ctypes.data, m.size,
                               out.ctypes.data, threads)
    return out


from . import ref  # noqa: E402,F401


_PI_F = np.float32(3.14159265359)


def ramp_filter_rows(sino_rows):
    """prj/utils.h:94-151 (rampFilter) applied to every row, in FP64: each row
    of W samples is zero padded to N = 2W, multiplied in the DFT domain by the
    real part of the DFT of the spatial ramp (0.25 at 0, -1/(pi^2 i^2) at odd
    lags, formed in float as the reference does) times a Hann window
    0.5 + 0.5 cos(2 pi i / N) (argument formed in float), and the first W
    samples of the inverse DFT are kept."""
    s = np.asarray(sino_rows, np.float64)
    W = s.shape[-1]
    N = 2 * W
    ramp = np.zeros(N, np.float64)
    ramp[0] = 0.25
    for i in range(1, N):
        if i % 2 == 0:
            continue
        m = i if i < N // 2 else N - i
        r = np.float32(-1.0) / _PI_F
        r = r / _PI_F
        r = r / np.float32(m)
        r = r / np.float32(m)
        ramp[i] = float(r)
    i = np.arange(N)
    arg = ((np.float32(2.0) * _PI_F) * i.astype(np.float32)) / np.float32(N)
    hann = 0.5 + 0.5 * np.cos(arg.astype(np.float64))
    G = np.fft.fft(ramp).real * hann
    pad = np.zeros(s.shape[:-1] + (N,), np.float64)
    pad[..., :W] = s
    return np.fft.ifft(np.fft.fft(pad, axis=-1) * G, axis=-1).real[..., :W]


def fbp(g, sino, prec=64, threads=0):
    """prj/cpuPrj.c:718-784 (cmd FBP_BIT): fan-beam cosine pre-weight
    d / sqrt(d^2 + (j dSize)^2) at detector offset j, ramp filter per view,
    then the FBP-weighted backprojection."""
    s = np.asarray(sino, np.float64).reshape(g.np, g.prjWidth).copy()
    if g.d > 0:
        j = np.abs(np.arange(g.prjWidth) - g.prjWidth // 2).astype(np.float64)
        d = float(g.d)
        s *= d / np.sqrt(d * d + j * j * float(g.dSize) * float(g.dSize))
    return backward(g, ramp_filter_rows(s), prec=prec, threads=threads, fbp_weighting=True)

"""The reference's own CPU projector, compiled unchanged -- TEST INFRASTRUCTURE.

Drives ``oracle/_ref/libref_prj{32,64}.so`` (prj/cpuPrj.c, as shipped and with
its scalar widened to double) and ``libref_parprj.so`` (prj/parPrj.c) through
their C entry points ``setup``/``cpuPrj`` (prj/prj.h:62-67) and
``parPrjConf``/``parPrjThread`` (prj/parPrj.h:18-20).  These libraries exist
only where the reference sources were present at build time; callers check
``available()`` first.  The reference keeps its configuration in process-global
state, so every call here is serialised.
"""
import ctypes
import os
import threading

import numpy as np

from . import REFDIR

FWD_BIT, BWD_BIT, FBP_BIT = 1 << 1, 1 << 2, 1 << 3   # prj/prj.h:30-32
_lock = threading.Lock()
_libs = {}


class _ParConf(ctypes.Structure):   # prj/parPrj.h:9-16
    _fields_ = [("bw", ctypes.c_double), ("nc", ctypes.c_int), ("nr", ctypes.c_int),
                ("np", ctypes.c_int), ("prjWidth", ctypes.c_int),
                ("theta", ctypes.POINTER(ctypes.c_double)), ("fwd", ctypes.c_int)]


def path(name):
    return os.path.join(REFDIR, name + ".so")


def available(name="libref_prj64"):
    return os.path.exists(path(name))


def _lib(prec):
    name = "libref_prj%d" % prec
    if name not in _libs:
        lib = ctypes.CDLL(path(name))
        real = ctypes.c_double if prec == 64 else ctypes.c_float
        lib.setup.argtypes = [ctypes.c_int] * 4 + [real] * 3
        lib.setup.restype = None
        lib.cpuPrj.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_char]
        lib.cpuPrj.restype = ctypes.c_int
        _libs[name] = lib
    return _libs[name]


def _run(g, prec, cmd, img, sino):
    lib = _lib(prec)
    with _lock:
        lib.setup(int(g.n), int(g.prjWidth), int(g.np), int(g.prjFull),
                  float(g.dSize), float(g.effectiveRate), float(g.d))
        lib.cpuPrj(img.ctypes.data, sino.ctypes.data, bytes([cmd]))


def forward(g, img, prec=64):
    dt = np.float64 if prec == 64 else np.float32
    img = np.ascontiguousarray(img, dtype=dt).reshape(g.n, g.n)
    sino = np.zeros((g.np, g.prjWidth), dt)
    _run(g, prec, FWD_BIT, img, sino)
    return sino


def backward(g, sino, prec=64):
    dt = np.float64 if prec == 64 else np.float32
    sino = np.ascontiguousarray(sino, dtype=dt).reshape(g.np, g.prjWidth)
    img = np.zeros((g.n, g.n), dt)
    _run(g, prec, BWD_BIT, img, sino)
    return img


def fbp(g, sino, prec=64):
    dt = np.float64 if prec == 64 else np.float32
    sino = np.ascontiguousarray(sino, dtype=dt).reshape(g.np, g.prjWidth)
    img = np.zeros((g.n, g.n), dt)
    _run(g, prec, FBP_BIT, img, sino)
    return img


def weight(dist, bw, c, s, prec=64):
    lib = _lib(prec)
    real = ctypes.c_double if prec == 64 else ctypes.c_float
    lib.getWeight.argtypes = [real] * 4
    lib.getWeight.restype = real
    return float(lib.getWeight(dist, bw, c, s))


def _parlib():
    if "par" not in _libs:
        lib = ctypes.CDLL(path("libref_parprj"))
        lib.parPrjConf.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                   ctypes.POINTER(_ParConf), ctypes.c_size_t]
        lib.parPrjThread.argtypes = []
        _libs["par"] = lib
    return _libs["par"]


def _par(x, mask_idx, conf, fwd):
    theta = np.ascontiguousarray(conf["theta"], dtype=np.float64).ravel()
    m = np.ascontiguousarray(mask_idx, dtype=np.float64).ravel()
    pc = _ParConf(float(conf["bw"]), int(conf["nc"]), int(conf["nr"]), theta.size,
                  int(conf["prjWidth"]), theta.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                  1 if fwd else 0)
    x = np.ascontiguousarray(x, dtype=np.float64).ravel()
    if fwd:
        img, out = x, np.zeros(theta.size * int(conf["prjWidth"]), np.float64)
        args = (img, out)
    else:
        out, prj = np.zeros(m.size, np.float64), x
        args = (out, prj)
    lib = _parlib()
    with _lock:
        lib.parPrjConf(args[0].ctypes.data, args[1].ctypes.data, m.ctypes.data,
                       ctypes.byref(pc), m.size)
        lib.parPrjThread()
    return out


def par_forward(x, mask_idx, conf):
    return _par(x, mask_idx, conf, True)


def par_backward(y, mask_idx, conf):
    return _par(y, mask_idx, conf, False)

"""Batches of slices with different geometries (include/ctprj_batch.h) over
torch tensors: one persistent launch per direction, optional CUDA-graph
capture, launch shapes chosen by the library's tuner."""
import ctypes

import numpy as np

from ._lib import CTPRJ_OK, CTPRJ_ETIMEOUT, Geometry, check, lib
from .projector import _stream_handle


def cfg4_geometries(count=64, seed=0):
    """Seeded slices of the mixed-size batch workload: n uniform over
    {128, 256, 384, 512, 768, 1024}, views over {90, 180, 360, 720}, half
    parallel beam over [0, pi) (prjFull = 2 views) and half fan beam over
    [0, 2 pi) (prjFull = views; the reference needs prjFull % 4 == 0, so 90
    fan views become 92), prjWidth = ceil(1.42 n), source at 4 n px."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(count):
        n = int(rng.choice([128, 256, 384, 512, 768, 1024]))
        v = int(rng.choice([90, 180, 360, 720]))
        W = int(np.ceil(1.42 * n))
        if rng.uniform() < 0.5:
            out.append(Geometry(n, W, v, 2 * v, 1.0, 1.0, 0.0))
        else:
            v = v if v % 4 == 0 else v + 2
            out.append(Geometry(n, W, v, v, 1.0, 1.0, 4.0 * n))
    return out


def _ptrs(ts):
    if ts is None:
        return None
    return (ctypes.c_void_p * len(ts))(*[ctypes.c_void_p(t.data_ptr()) for t in ts])


class Batch:
    def __init__(self, geometries, device=None):
        import torch
        self.geometries = [g if isinstance(g, Geometry) else Geometry(*g) for g in geometries]
        self.device = torch.cuda.current_device() if device is None else int(device)
        arr = (Geometry * len(self.geometries))(*self.geometries)
        self._b = ctypes.c_void_p()
        check(lib().ctprj_batch_create(arr, len(self.geometries), self.device, ctypes.byref(self._b)))
        self._keep = None

    def close(self):
        if self._b:
            lib().ctprj_batch_destroy(self._b)
            self._b = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def bind(self, imgs=None, sinos=None, bsinos=None, bimgs=None):
        for ts, shape in ((imgs, "img"), (sinos, "sino"), (bsinos, "sino"), (bimgs, "img")):
            if ts is None:
                continue
            for g, t in zip(self.geometries, ts):
                n = g.n * g.n if shape == "img" else g.np * g.prjWidth
                if not (t.is_cuda and t.is_contiguous() and t.numel() == n):
                    raise ValueError("buffer does not match its slice")
        self._keep = (imgs, sinos, bsinos, bimgs)
        check(lib().ctprj_batch_bind(self._b, _ptrs(imgs), _ptrs(sinos), _ptrs(bsinos), _ptrs(bimgs)))

    def forward(self, stream=None):
        check(lib().ctprj_batch_forward(self._b, _stream_handle(stream, self.device)))

    def backward(self, stream=None):
        check(lib().ctprj_batch_backward(self._b, _stream_handle(stream, self.device)))

    def capture(self, stream=None):
        import torch
        s = torch.cuda.Stream(self.device) if stream is None else stream
        torch.cuda.current_stream(self.device).synchronize()
        check(lib().ctprj_batch_capture(self._b, _stream_handle(s, self.device)))
        s.synchronize()

    def autotune(self, cache_path=None, stream=None):
        check(lib().ctprj_batch_autotune(self._b, _stream_handle(stream, self.device),
                                         cache_path.encode() if cache_path else None))
        return self.config()

    def config(self):
        buf = ctypes.create_string_buffer(256)
        check(lib().ctprj_batch_config(self._b, buf, 256))
        return buf.value.decode()


class StreamFlags:
    """Host-mapped publication flags for ctprj_batch_stream_backward: set
    flag i once slice i's sinogram is on the device."""

    def __init__(self, n):
        self._h = ctypes.c_void_p()
        self._d = ctypes.c_void_p()
        check(lib().ctprj_stream_flags_create(int(n), ctypes.byref(self._h), ctypes.byref(self._d)))
        self.n = int(n)
        self.flags = np.ctypeslib.as_array(ctypes.cast(self._h, ctypes.POINTER(ctypes.c_int)), shape=(self.n,))

    def publish(self, i):
        self.flags[i] = 1

    def close(self):
        if self._h:
            lib().ctprj_stream_flags_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def stream_backward(b, flags, timeout_s, stream=None):
    """Streaming backprojection of a bound Batch; returns (status code,
    per-slice timed-out flags).  CTPRJ_ETIMEOUT is returned, not raised."""
    st = (ctypes.c_int * len(b.geometries))()
    code = lib().ctprj_batch_stream_backward(b._b, flags._d, float(timeout_s), st,
                                             _stream_handle(stream, b.device))
    if code not in (CTPRJ_OK, CTPRJ_ETIMEOUT):
        check(code)
    return code, list(st)

"""Device-pointer projector: the plan API of include/ctprj.h over torch tensors.

Tensors are float32, contiguous and on the plan's CUDA device; every call is
enqueued on the current torch stream (or the stream given) and returns without
synchronising.  Shapes follow the reference (prj/cpuPrj.c): images (n, n)
row-major, sinograms (np, prjWidth) view-major.
"""
import ctypes

from ._lib import Geometry, check, lib


def _stream_handle(stream, device):
    import torch
    s = stream if stream is not None else torch.cuda.current_stream(device)
    return ctypes.c_void_p(s.cuda_stream)


def _dev_ptr(t, shape, device):
    import torch
    if not (isinstance(t, torch.Tensor) and t.is_cuda):
        raise TypeError("expected a CUDA tensor")
    if t.dtype != torch.float32 or not t.is_contiguous():
        raise TypeError("expected a contiguous float32 tensor")
    if t.numel() != shape[0] * shape[1]:
        raise ValueError("expected %d elements, got %d" % (shape[0] * shape[1], t.numel()))
    if t.device.index != device:
        raise ValueError("tensor on cuda:%d, plan on cuda:%d" % (t.device.index, device))
    return ctypes.c_void_p(t.data_ptr())


class Projector:
    """Forward projector A, backprojector A^T and FBP for one geometry."""

    def __init__(self, geometry, device=None):
        import torch
        self.geometry = geometry if isinstance(geometry, Geometry) else Geometry(*geometry)
        self.device = torch.cuda.current_device() if device is None else int(device)
        self._plan = ctypes.c_void_p()
        check(lib().ctprj_plan_create(ctypes.byref(self.geometry), self.device,
                                      ctypes.byref(self._plan)))
        g = self.geometry
        self.img_shape = (g.n, g.n)
        self.sino_shape = (g.np, g.prjWidth)

    def close(self):
        if self._plan:
            lib().ctprj_plan_destroy(self._plan)
            self._plan = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _new(self, shape):
        import torch
        return torch.empty(shape, dtype=torch.float32, device="cuda:%d" % self.device)

    def forward(self, img, out=None, stream=None):
        out = self._new(self.sino_shape) if out is None else out
        check(lib().ctprj_forward(self._plan, _dev_ptr(img, self.img_shape, self.device),
                                  _dev_ptr(out, self.sino_shape, self.device),
                                  _stream_handle(stream, self.device)))
        return out

    def backward(self, sino, out=None, stream=None):
        out = self._new(self.img_shape) if out is None else out
        check(lib().ctprj_backward(self._plan, _dev_ptr(sino, self.sino_shape, self.device),
                                   _dev_ptr(out, self.img_shape, self.device),
                                   _stream_handle(stream, self.device)))
        return out

    def fbp(self, sino, out=None, stream=None):
        out = self._new(self.img_shape) if out is None else out
        check(lib().ctprj_fbp(self._plan, _dev_ptr(sino, self.sino_shape, self.device),
                              _dev_ptr(out, self.img_shape, self.device),
                              _stream_handle(stream, self.device)))
        return out

    def count_updates(self, stream=None):
        """(forward, backward) ray-pixel updates per call: the exact number of
        nonzero operator entries each pass visits."""
        f, b = ctypes.c_longlong(), ctypes.c_longlong()
        check(lib().ctprj_count_updates(self._plan, ctypes.byref(f), ctypes.byref(b),
                                        _stream_handle(stream, self.device)))
        return f.value, b.value

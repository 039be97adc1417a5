"""The allocation-free forward projection (include/ctprj_noalloc.h).

Callers that cannot call cudaMalloc -- code inside another framework's memory
pool, real-time loops, embedders that reserved the whole GPU -- use
ctprj_forward_noalloc, whose scratch lives in file-scope device arrays.  This
test calls it through the C ABI twice in a row, on two different geometries,
and checks each result against the plan-based ctprj_forward (the tolerance of
the projector tests, 1e-5 relative L2; the two share their kernels, so the
results are expected to be identical).  The file is named to be collected last.
"""
import ctypes

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

import imgrecsrc_b200 as ct  # noqa: E402
from imgrecsrc_b200 import phantom  # noqa: E402

TOL = 1e-5


def noalloc():
    f = ct.lib().ctprj_forward_noalloc
    f.argtypes = [ctypes.POINTER(ct.Geometry), ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
    f.restype = ctypes.c_int
    return f


def rel(a, b):
    return (torch.linalg.norm((a - b).double()) / torch.linalg.norm(b.double())).item()


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


def test_two_calls_in_a_row_match_plan_forward():
    f = noalloc()
    stream = torch.cuda.current_stream()
    geoms = [ct.Geometry(512, 1024, 360, 360, 1.0, 1.0, 2048.0),
             ct.Geometry(255, 363, 180, 360, 1.0, 1.0, 0.0)]
    for call, g in enumerate(geoms):
        x = torch.from_numpy(phantom.ellipse_phantom(g.n, seed=call + 1)).cuda()
        x = x + 0.1 * torch.randn_like(x)
        out = torch.full((g.np, g.prjWidth), float("nan"), device="cuda")
        st = f(ctypes.byref(g), ctypes.c_void_p(x.data_ptr()), ctypes.c_void_p(out.data_ptr()),
               ctypes.c_void_p(stream.cuda_stream))
        assert st == 0, ct.lib().ctprj_last_error()
        ref = ct.Projector(g).forward(x)
        torch.cuda.synchronize()
        assert torch.isfinite(out).all()
        assert rel(out, ref) < TOL


def test_sizes_beyond_the_limit_are_rejected():
    f = noalloc()
    g = ct.Geometry(1025, 1448, 90, 180, 1.0, 1.0, 0.0)
    x = torch.zeros(1025 * 1025, device="cuda")
    y = torch.zeros(90 * 1448, device="cuda")
    st = f(ctypes.byref(g), ctypes.c_void_p(x.data_ptr()), ctypes.c_void_p(y.data_ptr()), None)
    assert st == ct._lib.CTPRJ_ERANGE
    assert b"1024" in ct.lib().ctprj_last_error()


def _call(f, g, x, out, stream):
    return f(ctypes.byref(g), ctypes.c_void_p(x.data_ptr()), ctypes.c_void_p(out.data_ptr()),
             ctypes.c_void_p(stream.cuda_stream))


@pytest.mark.parametrize("g", [
    ct.Geometry(1024, 4096, 8192, 8192, 1.0, 1.0, 4096.0),   # every static array at capacity
    ct.Geometry(301, 430, 364, 364, 1.0, 1.0, 900.0),       # prjFull % 8 == 4
    ct.Geometry(300, 427, 180, 364, 1.0, 1.0, 0.0),         # parallel, np < prjFull
], ids=["limits", "fan364", "par364"])
def test_limits_and_ragged_view_counts_match_plan_forward(g):
    f = noalloc()
    stream = torch.cuda.current_stream()
    x = torch.from_numpy(phantom.ellipse_phantom(g.n, seed=7)).cuda()
    x = x + 0.1 * torch.randn_like(x)
    # the plan-based forward first, then the allocation-free one on the same input
    ref = ct.Projector(g).forward(x)
    out = torch.full((g.np, g.prjWidth), float("nan"), device="cuda")
    assert _call(f, g, x, out, stream) == 0, ct.lib().ctprj_last_error()
    torch.cuda.synchronize()
    assert torch.isfinite(out).all()
    assert rel(out, ref) < TOL
    assert torch.equal(out, ref)


def test_call_on_a_capturing_stream_is_refused():
    f = noalloc()
    g = ct.Geometry(64, 91, 30, 60, 1.0, 1.0, 0.0)
    x = torch.rand(64, 64, device="cuda")
    out = torch.zeros(30, 91, device="cuda")
    side = torch.cuda.Stream()
    torch.cuda.synchronize()
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph, stream=side):
        out.add_(0.0)
        st = _call(f, g, x, out, side)
    assert st == ct._lib.CTPRJ_EINVAL
    assert b"captured" in ct.lib().ctprj_last_error()
    del graph
    # outside the capture the same call runs
    assert _call(f, g, x, out, torch.cuda.current_stream()) == 0
    torch.cuda.synchronize()
    assert rel(out, ct.Projector(g).forward(x)) < TOL

"""The reference's own MEX gateways, compiled unchanged against libctprj.so.

prj/mPrj.c (the gpuPrj MEX function, -DGPU=1) and prj/mParPrj.c are built by
`make -C oracle gateways` against a minimal MEX API (oracle/mexmock, MATLAB is
not installed) and linked to this engine's library.  Driving their mexFunction
exercises the drop-in boundary exactly as MATLAB would: 'config', 'forward',
'backward', 'FBP' for gpuPrj; 'forward'/'backward' for mParPrj.  The compiled
gateways exist only where the reference sources were present at build time.
"""
import ctypes
import os

import numpy as np
import pytest

import oracle

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

import imgrecsrc_b200 as ct  # noqa: E402,F401  (loads libctprj.so first)

VP = ctypes.c_void_p


def gateway(name):
    path = os.path.join(oracle.REFDIR, name + ".so")
    if not os.path.exists(path):
        pytest.skip("gateway %s not built (reference sources absent at build time)" % name)
    L = ctypes.CDLL(path)
    L.mexFunction.argtypes = [ctypes.c_int, ctypes.POINTER(VP), ctypes.c_int, ctypes.POINTER(VP)]
    L.mock_numeric.argtypes = [ctypes.c_size_t, ctypes.c_size_t, ctypes.c_int, VP]
    L.mock_numeric.restype = VP
    L.mock_string.argtypes = [ctypes.c_char_p]
    L.mock_string.restype = VP
    L.mock_struct.argtypes = [ctypes.c_int, ctypes.POINTER(ctypes.c_char_p), ctypes.POINTER(VP)]
    L.mock_struct.restype = VP
    L.mock_destroy.argtypes = [VP]
    L.mxGetPr.argtypes = [VP]
    L.mxGetPr.restype = ctypes.POINTER(ctypes.c_double)
    L.mxGetNumberOfElements.argtypes = [VP]
    L.mxGetNumberOfElements.restype = ctypes.c_size_t
    return L


def matrix(L, a, single=False):
    """A MATLAB matrix holding the 2-D array a (stored column-major)."""
    a = np.asarray(a, np.float32 if single else np.float64)
    if a.ndim == 1:
        a = a[:, None]
    f = np.asfortranarray(a)
    return L.mock_numeric(a.shape[0], a.shape[1], 1 if single else 0, f.ctypes.data)


def struct(L, fields):
    names = (ctypes.c_char_p * len(fields))(*[k.encode() for k in fields])
    vals = (VP * len(fields))(*[matrix(L, np.atleast_1d(v)) for v in fields.values()])
    return L.mock_struct(len(fields), names, vals)


def call(L, nlhs, args):
    prhs = (VP * len(args))(*args)
    plhs = (VP * max(nlhs, 1))()
    L.mexFunction(nlhs, plhs, len(args), prhs)
    if nlhs == 0:
        return None
    n = L.mxGetNumberOfElements(plhs[0])
    out = np.ctypeslib.as_array(L.mxGetPr(plhs[0]), shape=(n,)).copy()
    L.mock_destroy(plhs[0])
    return out


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


def rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def test_reference_mprj_gateway_on_the_engine():
    L = gateway("libref_mprj_gpu")
    import types
    g = types.SimpleNamespace(n=129, prjWidth=183, np=50, prjFull=120, dSize=0.9,
                              effectiveRate=0.8, d=400.0)
    conf = struct(L, dict(n=g.n, prjWidth=g.prjWidth, np=g.np, prjFull=g.prjFull,
                          dSize=g.dSize, effectiveRate=g.effectiveRate, d=g.d))
    call(L, 0, [matrix(L, [[0.0]]), conf, L.mock_string(b"config")])
    rng = np.random.default_rng(0)
    img = rng.standard_normal((g.n, g.n))       # MATLAB matrix: rows are y
    sino = rng.standard_normal(g.np * g.prjWidth)
    fwd = call(L, 1, [matrix(L, img), matrix(L, [[0.0]]), L.mock_string(b"forward")])
    assert rel(fwd, oracle.forward(g, img.astype(np.float32).astype(np.float64)).ravel()) < 1e-5
    fwd1 = call(L, 1, [matrix(L, img, single=True), matrix(L, [[0.0]]), L.mock_string(b"forward")])
    assert np.array_equal(fwd, fwd1)
    bwd = call(L, 1, [matrix(L, sino), matrix(L, [[0.0]]), L.mock_string(b"backward")])
    ob = oracle.backward(g, sino.astype(np.float32).astype(np.float64).reshape(g.np, g.prjWidth))
    assert rel(bwd, ob.ravel(order="F")) < 1e-5
    fb = call(L, 1, [matrix(L, sino), matrix(L, [[0.0]]), L.mock_string(b"FBP")])
    of = oracle.fbp(g, sino.astype(np.float32).astype(np.float64))
    assert rel(fb, of.ravel(order="F")) < 1e-4


def test_reference_mparprj_gateway_on_the_engine():
    L = gateway("libref_mparprj_gpu")
    z = np.load("tests/golden/parprj_golden.npz")
    for case in range(int(z["ncases"])):
        bw, nc, nr, W = z["p%d_conf" % case]
        theta = z["p%d_theta" % case]
        m = z["p%d_mask" % case]

        def conf():
            return struct(L, dict(bw=bw, nc=nc, nr=nr, prjWidth=W, theta=theta))
        fwd = call(L, 1, [matrix(L, z["p%d_x" % case]), matrix(L, m), conf(),
                          L.mock_string(b"forward")])
        bwd = call(L, 1, [matrix(L, z["p%d_y" % case]), matrix(L, m), conf(),
                          L.mock_string(b"backward")])
        assert rel(fwd, z["p%d_fwd" % case]) < 1e-12
        assert rel(bwd, z["p%d_bwd" % case]) < 1e-12

"""Pins the oracle restatement to the reference (CPU only).

The FP64 and FP32 restatements in oracle/ are compared with fixtures that the
reference's own prj/cpuPrj.c and prj/parPrj.c produced (tests/golden/, made by
make_golden.py), and, where the compiled reference is present in oracle/_ref,
with live runs of it on the parallel 256^2 / 180-view and fan 512^2 /
360-view geometries.
"""
import types

import numpy as np
import pytest

import oracle
from oracle import ref

GOLD = "tests/golden/projector_golden.npz"
PGOLD = "tests/golden/parprj_golden.npz"


def rel(a, b):
    return float(np.linalg.norm(np.asarray(a, np.float64) - b) / max(np.linalg.norm(b), 1e-300))


def geom(v):
    n, W, npv, P, ds, er, d = v
    return types.SimpleNamespace(n=int(n), prjWidth=int(W), np=int(npv), prjFull=int(P),
                                 dSize=float(ds), effectiveRate=float(er), d=float(d))


def golden_cases():
    z = np.load(GOLD)
    return [(z, i) for i in range(int(z["ncases"]))]


@pytest.mark.parametrize("case", range(10))
def test_fp64_restatement_matches_reference_fixtures(case):
    z = np.load(GOLD)
    if case >= int(z["ncases"]):
        pytest.skip("no such fixture")
    g = geom(z["c%d_geom" % case])
    f = oracle.forward(g, z["c%d_img" % case])
    b = oracle.backward(g, z["c%d_sino" % case])
    assert rel(f, z["c%d_fwd64" % case]) < 1e-13
    assert rel(b, z["c%d_bwd64" % case]) < 1e-13
    # structural zeros: detector 0 for even prjWidth, row/col 0 for even n
    if g.prjWidth % 2 == 0:
        assert np.all(f[:, 0] == 0)
    if g.n % 2 == 0:
        assert np.all(b[0, :] == 0) and np.all(b[:, 0] == 0)


@pytest.mark.parametrize("case", range(10))
def test_fbp_restatement_matches_reference_fixtures(case):
    z = np.load(GOLD)
    if case >= int(z["ncases"]):
        pytest.skip("no such fixture")
    g = geom(z["c%d_geom" % case])
    assert rel(oracle.fbp(g, z["c%d_sino" % case]), z["c%d_fbp64" % case]) < 1e-12


@pytest.mark.parametrize("case", range(10))
def test_fp32_restatement_matches_reference_fixtures(case):
    z = np.load(GOLD)
    if case >= int(z["ncases"]):
        pytest.skip("no such fixture")
    g = geom(z["c%d_geom" % case])
    f = oracle.forward(g, z["c%d_img" % case].astype(np.float32), prec=32)
    b = oracle.backward(g, z["c%d_sino" % case].astype(np.float32), prec=32)
    assert rel(f, z["c%d_fwd32" % case]) < 5e-6
    assert rel(b, z["c%d_bwd32" % case]) < 5e-6


@pytest.mark.parametrize("case", range(4))
def test_parprj_restatement_matches_reference_fixtures(case):
    z = np.load(PGOLD)
    bw, nc, nr, W = z["p%d_conf" % case]
    conf = dict(bw=bw, nc=int(nc), nr=int(nr), prjWidth=int(W), theta=z["p%d_theta" % case])
    m = z["p%d_mask" % case]
    assert rel(oracle.par_forward(z["p%d_x" % case], m, conf), z["p%d_fwd" % case]) < 1e-13
    assert rel(oracle.par_backward(z["p%d_y" % case], m, conf), z["p%d_bwd" % case]) < 1e-13


def test_weight_matches_reference_getweight():
    if not ref.available():
        pytest.skip("compiled reference not present")
    rng = np.random.default_rng(5)
    cases = [(0.3, 1.0, 1.0, 0.0), (0.5, 1.0, 0.0, 1.0), (-0.2, 0.4, 0.6, 0.8),
             (0.0, 2.5, 0.7071, 0.7071), (1.1, 1.0, 0.9, 0.1), (0.75, 0.5, 1.0, 0.0)]
    for _ in range(2000):
        th = rng.uniform(0, 2 * np.pi)
        cases.append((rng.uniform(-2, 2), rng.uniform(0.05, 3), np.cos(th), np.sin(th)))
    for c in cases:
        assert abs(oracle.weight(*c) - ref.weight(*c)) < 1e-13


def test_fp64_restatement_matches_live_reference_par256_fan512():
    if not ref.available():
        pytest.skip("compiled reference not present")
    rng = np.random.default_rng(7)
    for g in [geom((256, 363, 180, 360, 1, 1, 0)), geom((512, 1024, 360, 360, 1, 1, 2048))]:
        x = rng.standard_normal((g.n, g.n))
        y = rng.standard_normal((g.np, g.prjWidth))
        assert rel(oracle.forward(g, x), ref.forward(g, x)) < 1e-13
        assert rel(oracle.backward(g, y), ref.backward(g, y)) < 1e-13


def test_oracle_pair_is_adjoint():
    """<A x, y> = <x, A^T y> to the reference's own level (norm-normalised)."""
    rng = np.random.default_rng(11)
    for g in [geom((64, 91, 30, 60, 1, 1, 0)), geom((64, 90, 48, 48, 1, 1, 200))]:
        x = rng.standard_normal((g.n, g.n))
        y = rng.standard_normal((g.np, g.prjWidth))
        Ax = oracle.forward(g, x)
        Aty = oracle.backward(g, y)
        if g.prjWidth % 2 == 0:
            y[:, 0] = 0
        if g.n % 2 == 0:
            x[0, :] = 0
            x[:, 0] = 0
        err = abs((Ax * y).sum() - (x * Aty).sum()) / (np.linalg.norm(Ax) * np.linalg.norm(y))
        assert err < 1e-5


def test_nnz_counts_are_consistent():
    g = geom((64, 91, 30, 60, 1, 1, 0))
    f, b = oracle.forward_nnz(g), oracle.backward_nnz(g)
    assert 2.0 < f / (g.n ** 2 * g.np) < 2.6
    assert abs(f - b) / f < 0.02


def test_invalid_geometry_rejected():
    with pytest.raises(ValueError):
        oracle.forward(geom((32, 45, 16, 18, 1, 1, 0)), np.zeros((32, 32)))


@pytest.mark.parametrize("case", [0, 1])
def test_fp64_restatement_matches_reference_rows_at_full_size(case):
    """The restatement on full-size fan workloads against the selected rows of
    the reference's own FP64 output (tests/golden/fullsize_rows.npz)."""
    from imgrecsrc_b200 import phantom
    z = np.load("tests/golden/fullsize_rows.npz")
    g = geom(z["c%d_geom" % case])
    x = phantom.ellipse_phantom(g.n, seed=1).astype(np.float32).astype(np.float64)
    y = np.random.default_rng(int(z["sino_seed"])).standard_normal((g.np, g.prjWidth)).astype(np.float32)
    assert rel(oracle.forward(g, x)[z["c%d_views" % case]], z["c%d_fwd" % case]) < 1e-6
    assert rel(oracle.backward(g, y.astype(np.float64))[z["c%d_rows" % case]], z["c%d_bwd" % case]) < 1e-6

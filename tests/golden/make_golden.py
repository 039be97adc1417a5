"""Generates the golden fixtures in this directory from the reference itself.

Runs the reference's own prj/cpuPrj.c (FP64-widened and as-shipped FP32:
forward, backward and FBP) and prj/parPrj.c, compiled unchanged from the reference sources into oracle/_ref
(``make -C oracle ref``), on small seeded inputs, and stores inputs and outputs
in ``projector_golden.npz`` / ``parprj_golden.npz``.  The tests compare the
oracle restatement and the GPU path against these files, so they need neither
the reference sources nor the compiled reference at test time.

Usage:  python tests/golden/make_golden.py [reference_prj_dir]
"""
import os
import sys
import types

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

import oracle  # noqa: E402
from oracle import ref  # noqa: E402

# (n, prjWidth, np, prjFull, dSize, effectiveRate, d): parallel and fan, odd and
# even image / detector counts, partial view sets, non-unit detector pitch and
# beam fraction, and prjFull not divisible by 8.
PROJECTOR_CASES = [
    (32, 45, 16, 16, 1.0, 1.0, 0.0),
    (33, 46, 20, 40, 1.0, 1.0, 0.0),
    (32, 46, 24, 24, 0.8, 0.9, 100.0),
    (33, 45, 36, 36, 1.2, 1.0, 60.0),
    (64, 91, 30, 60, 1.0, 1.0, 0.0),
    (64, 90, 7, 60, 1.0, 1.3, 200.0),
    (48, 68, 12, 12, 1.0, 1.0, 150.0),
    (17, 25, 4, 4, 1.0, 1.0, 0.0),
    (1, 3, 4, 8, 1.0, 1.0, 0.0),
    (2, 4, 8, 8, 1.0, 1.0, 40.0),
]

PARPRJ_CASES = [
    (32, 45, 16, 32, 1.0, 0.7),
    (33, 50, 20, 40, 1.0, 1.0),
    (64, 91, 30, 60, 0.7, 0.5),
    (40, 60, 10, 37, 1.0, 1.0),
]


def main():
    refdir = sys.argv[1] if len(sys.argv) > 1 else oracle.reference_dir("prj")
    if not refdir or not oracle.build_ref(refdir):
        raise SystemExit("reference sources not found: pass <reference>/prj or set IMGRECSRC_REFERENCE")
    rng = np.random.default_rng(20240601)
    out = {}
    for ci, (n, W, npv, P, ds, er, d) in enumerate(PROJECTOR_CASES):
        g = types.SimpleNamespace(n=n, prjWidth=W, np=npv, prjFull=P, dSize=ds,
                                  effectiveRate=er, d=d)
        x = rng.standard_normal((n, n))
        y = rng.standard_normal((npv, W))
        out["c%d_geom" % ci] = np.array([n, W, npv, P, ds, er, d], np.float64)
        out["c%d_img" % ci] = x
        out["c%d_sino" % ci] = y
        out["c%d_fwd64" % ci] = ref.forward(g, x, 64)
        out["c%d_bwd64" % ci] = ref.backward(g, y, 64)
        out["c%d_fwd32" % ci] = ref.forward(g, x.astype(np.float32), 32)
        out["c%d_bwd32" % ci] = ref.backward(g, y.astype(np.float32), 32)
        out["c%d_fbp64" % ci] = ref.fbp(g, y, 64)
    out["ncases"] = np.array(len(PROJECTOR_CASES))
    np.savez_compressed(os.path.join(os.path.dirname(__file__), "projector_golden.npz"), **out)

    out = {}
    for ci, (n, W, npv, P, bw, keep) in enumerate(PARPRJ_CASES):
        theta = np.arange(npv) * 360.0 / P
        conf = dict(bw=bw, nc=n, nr=n, prjWidth=W, theta=theta)
        mask = np.flatnonzero(rng.random(n * n) < keep).astype(np.float64)
        x = rng.standard_normal(mask.size)
        y = rng.standard_normal(npv * W)
        out["p%d_conf" % ci] = np.array([bw, n, n, W], np.float64)
        out["p%d_theta" % ci] = theta
        out["p%d_mask" % ci] = mask
        out["p%d_x" % ci] = x
        out["p%d_y" % ci] = y
        out["p%d_fwd" % ci] = ref.par_forward(x, mask, conf)
        out["p%d_bwd" % ci] = ref.par_backward(y, mask, conf)
    out["ncases"] = np.array(len(PARPRJ_CASES))
    np.savez_compressed(os.path.join(os.path.dirname(__file__), "parprj_golden.npz"), **out)
    print("wrote fixtures")


if __name__ == "__main__":
    main()

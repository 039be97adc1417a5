"""Generates ``fullsize_rows.npz``: selected rows of the reference's own
prj/cpuPrj.c (FP64-widened, compiled unchanged into oracle/_ref by
``make -C oracle ref``) on two full-size fan workloads -- case 0: 2048^2,
1440 views over [0, 2 pi), 2048 detectors of unit pitch, source 8192 px from
the isocentre; case 1: 1024^2, 720 views, 1024 detectors, source 2048 px --
for the seeded ellipse phantom (forward) and a seeded N(0, 1) sinogram
(backprojection).  The full outputs (up to 12 and 17 MB) are too large to
commit; the rows cover octant-boundary views and interior ones, and image
rows near the centre, the axes and the edges.  The tests regenerate the same
inputs from the seeds.

Usage:  python tests/golden/make_fullsize_golden.py
"""
import os
import sys
import time
import types

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from oracle import ref  # noqa: E402
from imgrecsrc_b200 import phantom  # noqa: E402

CASES = [
    ((2048, 2048, 1440, 1440, 1.0, 1.0, 8192.0), [0, 1, 90, 179, 180, 181, 359, 360, 500, 719, 720, 1081, 1439],
     [0, 1, 2, 511, 1023, 1024, 1025, 1536, 2046, 2047]),
    ((1024, 1024, 720, 720, 1.0, 1.0, 2048.0), [0, 1, 45, 89, 90, 91, 179, 180, 250, 359, 360, 541, 719],
     [0, 1, 2, 255, 511, 512, 513, 768, 1022, 1023]),
]
SINO_SEED = 17


def main():
    if not ref.available():
        sys.exit("the compiled reference is missing: make -C oracle ref")
    arrays = {"ncases": len(CASES), "sino_seed": SINO_SEED}
    for c, (geom, views, rows) in enumerate(CASES):
        n, W, npv, P, ds, er, d = geom
        g = types.SimpleNamespace(n=n, prjWidth=W, np=npv, prjFull=P, dSize=ds, effectiveRate=er, d=d)
        x = phantom.ellipse_phantom(n, seed=1).astype(np.float32)
        y = np.random.default_rng(SINO_SEED).standard_normal((npv, W)).astype(np.float32)
        t = time.time()
        f = ref.forward(g, x.astype(np.float64), prec=64)
        b = ref.backward(g, y.astype(np.float64), prec=64)
        print("case %d: reference FP64 forward + backward %.1f s" % (c, time.time() - t))
        arrays.update({"c%d_geom" % c: np.array(geom), "c%d_views" % c: np.array(views),
                       "c%d_rows" % c: np.array(rows), "c%d_fwd" % c: f[views].astype(np.float32),
                       "c%d_bwd" % c: b[rows].astype(np.float32)})
    out = os.path.join(os.path.dirname(os.path.abspath(__file__)), "fullsize_rows.npz")
    np.savez_compressed(out, **arrays)
    print("wrote", out, os.path.getsize(out), "bytes")


if __name__ == "__main__":
    main()

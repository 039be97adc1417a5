"""Generates ``fullsize_rows.npz``: selected rows of the reference's own
prj/cpuPrj.c (FP64-widened, compiled unchanged into oracle/_ref by
``make -C oracle ref``) on the full 2048^2 fan workload -- 1440 views over
[0, 2 pi), 2048 detectors of unit pitch, source 8192 px from the isocentre --
for the seeded ellipse phantom (forward) and a seeded N(0, 1) sinogram
(backprojection).  The full outputs (12 and 17 MB) are too large to commit;
the rows below cover both octant-boundary views and interior ones, and image
rows near the centre, the axes and the edges.  The GPU test regenerates the
same inputs from the seeds.

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

GEOM = (2048, 2048, 1440, 1440, 1.0, 1.0, 8192.0)
VIEWS = [0, 1, 90, 179, 180, 181, 359, 360, 500, 719, 720, 1081, 1439]
ROWS = [0, 1, 2, 511, 1023, 1024, 1025, 1536, 2046, 2047]
SINO_SEED = 17


def inputs():
    n, W, npv = GEOM[0], GEOM[1], GEOM[2]
    x = phantom.ellipse_phantom(n, seed=1).astype(np.float32)
    y = np.random.default_rng(SINO_SEED).standard_normal((npv, W)).astype(np.float32)
    return x, y


def main():
    if not ref.available():
        sys.exit("the compiled reference is missing: make -C oracle ref")
    g = types.SimpleNamespace(n=GEOM[0], prjWidth=GEOM[1], np=GEOM[2], prjFull=GEOM[3], dSize=GEOM[4],
                              effectiveRate=GEOM[5], d=GEOM[6])
    x, y = inputs()
    t = time.time()
    f = ref.forward(g, x.astype(np.float64), prec=64)
    b = ref.backward(g, y.astype(np.float64), prec=64)
    print("reference FP64 forward + backward: %.1f s" % (time.time() - t))
    out = os.path.join(os.path.dirname(os.path.abspath(__file__)), "fullsize_rows.npz")
    np.savez_compressed(out, geom=np.array(GEOM), views=np.array(VIEWS), rows=np.array(ROWS),
                        sino_seed=SINO_SEED, fwd=f[VIEWS].astype(np.float32), bwd=b[ROWS].astype(np.float32),
                        fwd_norm=np.linalg.norm(f), bwd_norm=np.linalg.norm(b))
    print("wrote", out, os.path.getsize(out), "bytes")


if __name__ == "__main__":
    main()

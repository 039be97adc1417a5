"""Generates rwt_golden.npz in this directory from the reference itself.

Runs the reference's vendored Rice Wavelet Toolbox cores (rwt/mdwt_r.c MDWT,
rwt/midwt_r.c MIDWT), compiled unchanged into oracle/_ref/libref_rwt.so
(``make -C oracle rwt``), on small seeded column-major images for several
Daubechies filters (the filters themselves from the oracle's restatement of
rwt/daubcqf.m) and level counts, and stores filters, inputs and outputs.  The
tests compare the oracle restatement and the GPU transform against this file,
so they need neither the reference sources nor the compiled reference.

Usage:  python tests/golden/make_rwt_golden.py [reference_rwt_dir]
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

import oracle  # noqa: E402
from oracle import wavelet_oracle as W  # noqa: E402

# (daub, rows, cols, levels): Haar as the BHC examples use it (6 levels),
# longer filters, non-square images, filters longer than the coarsest block
CASES = [
    (2, 64, 64, 6),
    (2, 16, 48, 4),
    (4, 32, 32, 3),
    (4, 16, 40, 3),
    (6, 32, 16, 4),
    (8, 24, 16, 3),
    (12, 16, 16, 2),
]


def main():
    rwt = sys.argv[1] if len(sys.argv) > 1 else oracle.reference_dir("rwt")
    if not rwt or not oracle.build_rwt(rwt):
        sys.exit("reference rwt sources not found: pass <reference>/rwt or set IMGRECSRC_REFERENCE")
    rng = np.random.default_rng(20240611)
    out = {}
    for i, (daub, m, n, L) in enumerate(CASES):
        h = W.daubcqf(daub)
        x = rng.standard_normal((m, n))
        out["case%d_meta" % i] = np.array([daub, m, n, L])
        out["case%d_h" % i] = h
        out["case%d_x" % i] = x                          # input of both transforms
        out["case%d_mdwt" % i] = W.ref_mdwt(x, h, L)
        out["case%d_midwt" % i] = W.ref_midwt(x, h, L)
    np.savez_compressed(os.path.join(os.path.dirname(os.path.abspath(__file__)), "rwt_golden.npz"), **out)
    print("wrote %d cases" % len(CASES))


if __name__ == "__main__":
    main()

"""Generates wvltmask_golden.npz in this directory from the reference itself.

The reference ships the wavelet-coefficient masks its BHC drivers load
(bhc/doBHC.m:45-52, bhcEx/load*.m): utils/MaskWvlt<n>CircleL<L>D<D>.mat, each
the output of its own utils/wvltMask.m for the reconstruction mask
Utils.getCircularMask(n) (utils/Utils.m:438-444), an L-level transform and the
Daubechies filter daubcqf(D).  This script copies every one of them, as packed
bits in MATLAB's element order, into one compressed fixture, so that the tests
compare the oracle restatement and the GPU's ctprj_wvlt_mask against reference
outputs without the reference being present.

Usage:  python tests/golden/make_wvltmask_golden.py [reference_utils_dir]
"""
import glob
import os
import re
import sys

import numpy as np
import scipy.io as sio

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

import oracle  # noqa: E402


def main():
    utils = sys.argv[1] if len(sys.argv) > 1 else oracle.reference_dir("utils")
    if not utils or not os.path.isdir(utils):
        sys.exit("reference utils/ not found: pass <reference>/utils or set IMGRECSRC_REFERENCE")
    out = {}
    for f in sorted(glob.glob(os.path.join(utils, "MaskWvlt*Circle*.mat"))):
        mt = re.fullmatch(r"MaskWvlt(\d+)CircleL(\d+)D(\d+)\.mat", os.path.basename(f))
        if not mt:
            continue
        n, L, D = map(int, mt.groups())
        maskk = sio.loadmat(f)["maskk"] != 0
        assert maskk.shape == (n, n), (f, maskk.shape)
        key = "n%d_L%d_D%d" % (n, L, D)
        out[key] = np.packbits(maskk.ravel(order="F"))
        out[key + "_count"] = np.array(int(maskk.sum()))
    np.savez_compressed(os.path.join(os.path.dirname(os.path.abspath(__file__)), "wvltmask_golden.npz"), **out)
    print("wrote %d masks" % (len(out) // 2))


if __name__ == "__main__":
    main()

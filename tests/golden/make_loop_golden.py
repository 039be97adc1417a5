"""Writes tests/golden/loop_fan2048_pg50.npz: the FP64 oracle's run of the
alternating beam-hardening loop at full size, the record the GPU loop is
checked against (tests/test_loop_fullsize_gpu.py).

Problem (the polychromatic loop at scale): fan beam, 2048^2 image, 1440 views
over [0, 2 pi), 2048 detectors, source 8192 px from the isocentre; two-material
phantom (seed 2); J = 30 b1 spectrum coefficients on kappa log-spaced over
[1e-2, 1e2] cm^2/g, truth = the seeded bump (seed 2); pixel size 2 cm / 2048.
Measurement: Poisson counts at I0 = 1e5 per ray of the FP64 oracle's
noise-free intensity, drawn by numpy (seed 7), divided by I0 and stored as
float32 -- regenerated by the GPU test, which checks this file's digest of it.
Loop: 50 iterations of the projected-gradient density step (npg/PG.m, initial
step 1e-3, projection on x >= 0) and the FP64 spectrum step (two Newton steps
on Ie >= 0), from x = 1 g/cm^3 and a uniform spectrum
(bhc/beamhardenSpline.m:340-570), run by oracle/bhc_loop_oracle.py over the
FP64 projector restatement.  About 90 minutes on an 8-core host.

Stored: the cost and accepted step of every iteration, the final spectrum, the
final density at 65536 seeded pixels with the full image's L2 norm (the test
estimates the relative L2 error from those pixels), the oracle's own error
against the phantom, and the measurement's digest.

  python tests/golden/make_loop_golden.py [ITERATIONS]
"""
import hashlib
import os
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

GEOM = dict(n=2048, prjWidth=2048, np=1440, prjFull=1440, dSize=1.0, effectiveRate=1.0, d=8192.0)
J, I0, SEED_X, SEED_I, SEED_M = 30, 1e5, 2, 2, 7
SAMPLE, SAMPLE_SEED = 65536, 11
OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "loop_fan2048_pg50.npz")


def geometry():
    import types
    return types.SimpleNamespace(**GEOM)


def measurement(g):
    """Noise-free FP64 intensity of the phantom through the oracle, then seeded
    Poisson counts; returns (x_true, Ie_true, imea float32, digest)."""
    import oracle
    from imgrecsrc_b200 import phantom
    from oracle import bhc_oracle as BO
    x_true = phantom.two_material_phantom(g.n, seed=SEED_X)
    I_true = phantom.spectrum_bump(J, seed=SEED_I)
    Ts = 2.0 / g.n
    s = Ts * oracle.forward(g, x_true.astype(np.float64)).ravel()
    BL, _, _ = BO.b1_iout(BO.kappa_nodes(J), s, I_true)
    rng = np.random.default_rng(SEED_M)
    imea = (rng.poisson(I0 * BL) / I0).astype(np.float32).reshape(g.np, g.prjWidth)
    return x_true, I_true, imea, digest(imea)


def digest(a):
    return hashlib.sha256(np.ascontiguousarray(a, np.float32).tobytes()).hexdigest()


def sample_index(n):
    return np.sort(np.random.default_rng(SAMPLE_SEED).choice(n * n, SAMPLE, replace=False))


def main(iters=50):
    import oracle
    from oracle import bhc_loop_oracle as LO
    from oracle import bhc_oracle as BO
    g = geometry()
    t0 = time.time()
    x_true, I_true, imea, dg = measurement(g)
    print("measurement: %.0f s, digest %s" % (time.time() - t0, dg), flush=True)
    Ts = 2.0 / g.n
    t0 = time.time()
    x, Ie, st = LO.reconstruct(lambda v: oracle.forward(g, v),
                               lambda y: oracle.backward(g, y.reshape(g.np, g.prjWidth)),
                               BO.kappa_nodes(J), Ts, np.ones((g.n, g.n)), np.full(J, 1.0 / J),
                               imea.astype(np.float64), iters, x_step=1e-3, method="pg")
    secs = time.time() - t0
    idx = sample_index(g.n)
    rel_truth = float(np.linalg.norm(x - x_true) / np.linalg.norm(x_true))
    np.savez_compressed(OUT, iterations=iters, cost=np.array(st["cost"]), x_step=np.array(st["x_step"]),
                        Ie=Ie, x_norm=float(np.linalg.norm(x)), x_sample_index=idx.astype(np.int32),
                        x_sample=x.ravel()[idx], rel_err_vs_truth=rel_truth, imea_digest=dg,
                        imea_sum=float(imea.astype(np.float64).sum()), oracle_seconds=secs)
    print("oracle loop: %d iterations in %.0f s, final cost %.12g, rel err vs phantom %.6g"
          % (iters, secs, st["cost"][-1], rel_truth))


if __name__ == "__main__":
    main(int(sys.argv[1]) if len(sys.argv) > 1 else 50)

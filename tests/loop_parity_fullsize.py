"""The BHC loop at config 5's full size against the FP64 oracle loop (not a
pytest module: the FP64 side takes about 40 minutes of host time).

  python tests/loop_parity_fullsize.py gpu OUTDIR [ITERS]      # on a B200
  python tests/loop_parity_fullsize.py oracle OUTDIR [ITERS]   # on any host

The GPU step builds the bench's problem (fan 2048^2, 1440 views, 2048 bins,
d = 8192 px, two-material phantom, J = 30, Poisson counts at I0 = 1e5), runs
ITERS (default 20) PG iterations of ctprj_bhc_reconstruct and saves the
measurement and the results in OUTDIR; the oracle step runs the same loop in
FP64 (oracle/bhc_loop_oracle.py over the FP64 projector) on that measurement
and prints how the two compare.
"""
import os
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

GEOM = (2048, 2048, 1440, 1440, 1.0, 1.0, 8192.0)
J, I0 = 30, 1e5


def run_gpu(out, iters):
    import torch

    import imgrecsrc_b200 as ct
    from imgrecsrc_b200 import bhc, phantom
    g = ct.Geometry(*GEOM)
    pr = ct.Projector(g)
    Ts = 2.0 / g.n
    x_true = torch.from_numpy(phantom.two_material_phantom(g.n, seed=2)).cuda()
    model = bhc.BHCModel(pr, bhc.kappa_nodes(J), Ts)
    I_true = torch.from_numpy(phantom.spectrum_bump(J, seed=2)).cuda()
    BL = (model.basis(pr.forward(x_true)) @ I_true).reshape(g.np, g.prjWidth)
    gen = torch.Generator(device="cuda").manual_seed(7)
    imea = (torch.poisson(I0 * BL, generator=gen) / I0).float().contiguous()
    x = torch.full((g.n, g.n), 1.0, device="cuda")
    Ie = torch.full((J,), 1.0 / J, dtype=torch.float64, device="cuda")
    st = model.reconstruct(x, Ie, imea, iterations=iters, x_step=1e-3, method="pg")
    np.savez(os.path.join(out, "loop_parity_gpu.npz"), imea=imea.cpu().numpy(), x=x.cpu().numpy(),
             Ie=Ie.cpu().numpy(), cost=np.array(st["cost"]), step=np.array(st["x_step"]))
    print("gpu: %d iterations, final cost %.10g, %d evaluations" % (st["iterations"], st["final_cost"],
                                                                    st["evaluations"]))


def run_oracle(out, iters):
    import imgrecsrc_b200 as ct
    import oracle
    from imgrecsrc_b200 import phantom
    from oracle import bhc_loop_oracle as LO
    from oracle import bhc_oracle as BO
    d = np.load(os.path.join(out, "loop_parity_gpu.npz"))
    g = ct.Geometry(*GEOM)
    Ts = 2.0 / g.n
    t0 = time.time()
    xo, Io, so = LO.reconstruct(lambda x: oracle.forward(g, x),
                                lambda y: oracle.backward(g, y.reshape(g.np, g.prjWidth)),
                                BO.kappa_nodes(J), Ts, np.ones((g.n, g.n)), np.full(J, 1.0 / J),
                                d["imea"].astype(np.float64), iters, x_step=1e-3, method="pg")
    cg, sg = d["cost"][:iters], d["step"][:iters]
    co, sto = np.array(so["cost"]), np.array(so["x_step"])
    rel = lambda a, b: float(np.linalg.norm(a - b) / np.linalg.norm(b))
    x_true = phantom.two_material_phantom(g.n, seed=2).astype(np.float64)
    print("oracle: %.0f s" % (time.time() - t0))
    print("identical steps:", bool(np.array_equal(sg, sto)))
    print("max cost rel %.3g (final %.10g vs %.10g)" % (float(np.max(np.abs(cg - co) / np.abs(co))), cg[-1], co[-1]))
    print("x rel %.3g, Ie rel %.3g" % (rel(d["x"].astype(np.float64), xo), rel(d["Ie"], Io)))
    print("vs truth: gpu %.6g, oracle %.6g" % (rel(d["x"].astype(np.float64), x_true), rel(xo, x_true)))


if __name__ == "__main__":
    mode, outdir = sys.argv[1], sys.argv[2]
    n_it = int(sys.argv[3]) if len(sys.argv) > 3 else 20
    (run_gpu if mode == "gpu" else run_oracle)(outdir, n_it)

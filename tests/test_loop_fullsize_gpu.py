"""The alternating beam-hardening loop at full size against the FP64 oracle's
run of it (tests/golden/loop_fan2048_pg50.npz, written by
tests/golden/make_loop_golden.py; reference loop bhc/beamhardenSpline.m:340-570
with the npg/PG.m density step).

Fan beam 2048^2, 1440 views, 2048 detectors, source 8192 px from the
isocentre, J = 30, Poisson counts at I0 = 1e5: the measurement is regenerated
here exactly as the golden's generator drew it (its digest must match), then
50 iterations of ctprj_bhc_reconstruct (projected-gradient density step with
initial step 1e-3, two FP64 Newton spectrum steps) run on the GPU.

Checked against the oracle's record: the same accepted density step in every
iteration (the line search took the same decisions), the cost of every
iteration within 1e-5 relative, the final spectrum within 1e-5 relative L2 and
the final density within 1e-5 relative L2, estimated from 65536 seeded
pixels (the oracle's image is too large to keep).  The cost is a sum of
2.9e6 per-ray terms of order one that cancel to about 220, so the FP32
projections' rounding reaches it amplified (3e-6 at worst over the 50
iterations on the B200, 7e-7 at the end)."""
import importlib.util
import os

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

import imgrecsrc_b200 as ct  # noqa: E402
from imgrecsrc_b200 import bhc  # noqa: E402

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = os.path.join(HERE, "golden", "loop_fan2048_pg50.npz")


def generator():
    spec = importlib.util.spec_from_file_location("make_loop_golden",
                                                  os.path.join(HERE, "golden", "make_loop_golden.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


def test_fifty_iterations_track_the_fp64_oracle_loop():
    gold = np.load(GOLDEN)
    gen = generator()
    gm = gen.geometry()
    _, _, imea, dg = gen.measurement(gm)
    assert dg == str(gold["imea_digest"]), "the measurement was not regenerated bit for bit"
    iters = int(gold["iterations"])

    g = ct.Geometry(gm.n, gm.prjWidth, gm.np, gm.prjFull, gm.dSize, gm.effectiveRate, gm.d)
    pr = ct.Projector(g)
    Ts = 2.0 / g.n
    model = bhc.BHCModel(pr, bhc.kappa_nodes(gen.J), Ts)
    x = torch.full((g.n, g.n), 1.0, device="cuda")
    Ie = torch.full((gen.J,), 1.0 / gen.J, dtype=torch.float64, device="cuda")
    st = model.reconstruct(x, Ie, torch.from_numpy(imea).cuda(), iterations=iters, x_step=1e-3,
                           method="pg")
    assert st["iterations"] == iters
    steps, cost = np.array(st["x_step"]), np.array(st["cost"])
    np.testing.assert_allclose(steps, gold["x_step"], rtol=1e-12, atol=0)
    cost_rel = np.abs(cost - gold["cost"]) / np.abs(gold["cost"])
    Ie_rel = float(np.linalg.norm(Ie.cpu().numpy() - gold["Ie"]) / np.linalg.norm(gold["Ie"]))
    idx = gold["x_sample_index"].astype(np.int64)
    xs = x.cpu().numpy().ravel()[idx].astype(np.float64)
    # sum of squares over the sample, scaled to the whole image
    x_rel = float(np.sqrt(np.sum((xs - gold["x_sample"]) ** 2) * (g.n * g.n / idx.size))
                  / gold["x_norm"])
    print("loop fan 2048^2, %d iterations: steps identical, max cost rel %.2e (final %.10g vs %.10g), "
          "Ie rel %.2e, x rel %.2e (sampled)" % (iters, cost_rel.max(), cost[-1], gold["cost"][-1],
                                                  Ie_rel, x_rel))
    assert cost_rel.max() <= 1e-5
    assert Ie_rel <= 1e-5
    assert x_rel <= 1e-5
    model.close()
    pr.close()

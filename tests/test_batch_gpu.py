"""Batched persistent launches (include/ctprj_batch.h): every slice of a
mixed batch must come out bit for bit as the per-slice ctprj_forward /
ctprj_backward give it (same block bodies), directly, from a captured CUDA
graph, and after the tuner changed the launch shapes."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

import imgrecsrc_b200 as ct  # noqa: E402
from imgrecsrc_b200 import batch, phantom  # noqa: E402


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


def small_batch():
    geoms = [ct.Geometry(128, 182, 90, 180, 1.0, 1.0, 0.0),
             ct.Geometry(256, 364, 180, 180, 1.0, 1.0, 1024.0),
             ct.Geometry(127, 181, 92, 92, 1.0, 1.0, 508.0),
             ct.Geometry(384, 546, 90, 180, 1.0, 1.0, 0.0),
             ct.Geometry(96, 137, 60, 120, 0.9, 0.8, 0.0),
             ct.Geometry(200, 284, 120, 120, 1.1, 1.0, 300.0),
             ct.Geometry(64, 91, 33, 60, 1.0, 1.0, 0.0),
             ct.Geometry(33, 45, 36, 36, 1.2, 1.0, 60.0)]   # strongly magnified fan
    return geoms


def run(geoms, tune_path=None):
    rng = np.random.default_rng(0)
    imgs = [torch.from_numpy(phantom.ellipse_phantom(g.n, seed=i)).cuda() for i, g in enumerate(geoms)]
    bsinos = [torch.from_numpy(rng.standard_normal((g.np, g.prjWidth)).astype(np.float32)).cuda()
              for g in geoms]
    sinos = [torch.full((g.np, g.prjWidth), float("nan"), device="cuda") for g in geoms]
    bimgs = [torch.full((g.n, g.n), float("nan"), device="cuda") for g in geoms]
    b = batch.Batch(geoms)
    b.bind(imgs, sinos, bsinos, bimgs)
    refs_f = [ct.Projector(g).forward(x) for g, x in zip(geoms, imgs)]
    refs_b = [ct.Projector(g).backward(y) for g, y in zip(geoms, bsinos)]

    def check_all():
        torch.cuda.synchronize()
        for i in range(len(geoms)):
            assert torch.equal(sinos[i], refs_f[i]), i
            assert torch.equal(bimgs[i], refs_b[i]), i

    b.forward()
    b.backward()
    check_all()
    for t in sinos + bimgs:
        t.fill_(float("nan"))
    b.capture()
    b.forward()
    b.backward()
    check_all()
    if tune_path:
        cfg = b.autotune(tune_path)
        for t in sinos + bimgs:
            t.fill_(float("nan"))
        b.forward()
        b.backward()
        check_all()
        return cfg
    return b.config()


def test_batch_matches_per_slice_bitwise(tmp_path):
    cfg = run(small_batch(), str(tmp_path / "tune.txt"))
    assert "fwd_views" in cfg
    # the cache is reused on a second tuning of the same batch
    assert open(tmp_path / "tune.txt").read().count("\n") == 1
    cfg2 = run(small_batch(), str(tmp_path / "tune.txt"))
    assert cfg2 == cfg
    assert open(tmp_path / "tune.txt").read().count("\n") == 1


def test_cfg4_batch_matches_per_slice():
    """All 64 slices of the mixed batch the bench times (image sizes drawn from
    {128, ..., 1024}^2, 90 to 720 views, half parallel and half fan), each bit
    for bit equal to its per-slice forward and backprojection."""
    geoms = batch.cfg4_geometries(64, seed=0)
    assert len(geoms) == 64
    run(geoms)

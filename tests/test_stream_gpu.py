"""Streaming backprojection with bounded device-side waits (failure
detection without a GPU fault): the persistent kernel waits for slices the
host publishes through host-mapped flags, gives up on a slice after the
timeout, reports CTPRJ_ETIMEOUT with per-slice status, and leaves the device
usable.  Published slices come out exactly as the plain backprojection."""
import threading
import time

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

import imgrecsrc_b200 as ct  # noqa: E402
from imgrecsrc_b200 import batch  # noqa: E402


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


def make():
    geoms = [ct.Geometry(128, 182, 90, 180, 1.0, 1.0, 0.0), ct.Geometry(96, 137, 60, 60, 1.0, 1.0, 400.0),
             ct.Geometry(160, 228, 72, 144, 1.0, 1.0, 0.0), ct.Geometry(64, 91, 48, 48, 1.0, 1.0, 256.0),
             ct.Geometry(200, 284, 40, 80, 1.0, 1.0, 0.0), ct.Geometry(100, 142, 36, 36, 1.0, 1.0, 500.0)]
    rng = np.random.default_rng(0)
    sinos = [torch.from_numpy(rng.standard_normal((g.np, g.prjWidth)).astype(np.float32)).cuda() for g in geoms]
    outs = [torch.full((g.n, g.n), float("nan"), device="cuda") for g in geoms]
    b = batch.Batch(geoms)
    b.bind(None, None, sinos, outs)
    refs = [ct.Projector(g).backward(y) for g, y in zip(geoms, sinos)]
    return geoms, b, outs, refs


def test_unpublished_slices_time_out_and_the_device_stays_usable():
    geoms, b, outs, refs = make()
    flags = batch.StreamFlags(len(geoms))
    for i in (0, 2, 4):
        flags.publish(i)
    t0 = time.time()
    code, status = batch.stream_backward(b, flags, timeout_s=0.2)
    took = time.time() - t0
    assert code == ct._lib.CTPRJ_ETIMEOUT
    assert status == [0, 1, 0, 1, 0, 1]
    assert b"not published" in ct.lib().ctprj_last_error()
    assert took < 10
    torch.cuda.synchronize()
    for i in (0, 2, 4):
        assert torch.equal(outs[i], refs[i])
    for i in (1, 3, 5):
        assert torch.isnan(outs[i]).all()
    # the context is intact: the regular batched launch works afterwards
    b.backward()
    torch.cuda.synchronize()
    for i in range(len(geoms)):
        assert torch.equal(outs[i], refs[i])
    flags.close()


def test_publication_while_the_kernel_runs():
    geoms, b, outs, refs = make()
    flags = batch.StreamFlags(len(geoms))

    def publisher():
        for i in reversed(range(len(geoms))):
            time.sleep(0.02)
            flags.publish(i)
    th = threading.Thread(target=publisher)
    th.start()
    code, status = batch.stream_backward(b, flags, timeout_s=5.0)
    th.join()
    assert code == ct._lib.CTPRJ_OK and status == [0] * len(geoms)
    torch.cuda.synchronize()
    for i in range(len(geoms)):
        assert torch.equal(outs[i], refs[i])
    flags.close()

"""The wavelet oracle (oracle/wavelet_oracle.py) pinned to the reference: the
worked examples of rwt's own help texts (rwt/daubcqf.m, rwt/mdwt.m,
rwt/midwt.m), the golden outputs of the reference's compiled rwt cores
(tests/golden/rwt_golden.npz, made by tests/golden/make_rwt_golden.py), and
the ADMM restatement of npg/admm.m against an independent primal-dual solve
of the same proximal problem."""
import math
import os

import numpy as np
import pytest

from oracle import wavelet_oracle as W

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "rwt_golden.npz")
MASKS = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "wvltmask_golden.npz")


def reference_mask(z, key):
    """(n, L, daub) and the mask of golden entry `key` (MATLAB's element order)."""
    n, L, D = (int(p[1:]) for p in key.split("_"))
    m = np.unpackbits(z[key], count=n * n).reshape((n, n), order="F").astype(bool)
    assert m.sum() == int(z[key + "_count"])
    return n, L, D, m


def test_daubechies_filters():
    """daubcqf(4) as printed in rwt/daubcqf.m's example, and its closed form;
    every filter orthonormal (sum h^2 = 1, sum h = sqrt 2)."""
    h4 = W.daubcqf(4)
    assert np.allclose(h4, [0.4830, 0.8365, 0.2241, -0.1294], atol=5e-5)
    s3 = math.sqrt(3.0)
    assert np.allclose(h4, np.array([1 + s3, 3 + s3, 3 - s3, 1 - s3]) / (4 * math.sqrt(2.0)), atol=1e-14)
    assert np.allclose(W.daubcqf(2), [2 ** -0.5, 2 ** -0.5], atol=0)
    for N in (2, 4, 6, 8, 12, 20):
        h = W.daubcqf(N)
        assert len(h) == N
        assert abs((h * h).sum() - 1.0) < 1e-10
        assert abs(h.sum() - math.sqrt(2.0)) < 1e-12
        for k in range(1, N // 2):   # orthogonal to its even shifts
            assert abs((h[2 * k:] * h[:N - 2 * k]).sum()) < 1e-10


def test_help_text_examples():
    """mdwt(makesig('LinChirp', 8), daubcqf(4), 2) and midwt(mdwt(x, h, 1),
    h, 1) as printed in rwt/mdwt.m and rwt/midwt.m."""
    t = np.arange(1, 9) / 8.0
    x = np.sin(np.pi * t * ((8 * 0.125) * t))          # rwt/makesig.m 'LinChirp'
    h = W.daubcqf(4)
    y = W.mdwt(x, h, 2)
    assert np.allclose(y, [1.1097, 0.8767, 0.8204, -0.5201, -0.0339, 0.1001, 0.2201, -0.1401], atol=5e-5)
    xi = W.midwt(W.mdwt(x, h, 1), h, 1)
    assert np.allclose(xi, [0.0491, 0.1951, 0.4276, 0.7071, 0.9415, 0.9808, 0.6716, 0.0000], atol=5e-5)


def test_against_the_compiled_reference_golden():
    g = np.load(GOLDEN)
    i = 0
    while "case%d_meta" % i in g:
        daub, m, n, L = (int(v) for v in g["case%d_meta" % i])
        h = g["case%d_h" % i]
        assert np.allclose(h, W.daubcqf(daub), atol=1e-14, rtol=0)
        x = g["case%d_x" % i]
        assert x.shape == (m, n)
        assert np.abs(W.mdwt(x, h, L) - g["case%d_mdwt" % i]).max() < 1e-13, (daub, m, n, L)
        assert np.abs(W.midwt(x, h, L) - g["case%d_midwt" % i]).max() < 1e-13, (daub, m, n, L)
        i += 1
    assert i >= 7


@pytest.mark.skipif(not W.ref_available(), reason="reference rwt not compiled here")
def test_against_the_compiled_reference_live():
    rng = np.random.default_rng(1)
    for daub, (m, n, L) in ((2, (32, 64, 5)), (4, (48, 16, 3)), (10, (16, 32, 2))):
        h = W.daubcqf(daub)
        x = rng.standard_normal((m, n))
        assert np.abs(W.mdwt(x, h, L) - W.ref_mdwt(x, h, L)).max() < 1e-13
        assert np.abs(W.midwt(x, h, L) - W.ref_midwt(x, h, L)).max() < 1e-13


def test_transform_is_orthogonal():
    rng = np.random.default_rng(2)
    for daub in (2, 4, 8):
        h = W.daubcqf(daub)
        x = rng.standard_normal((32, 16))
        y = rng.standard_normal((32, 16))
        assert abs((W.mdwt(x, h, 3) * y).sum() - (x * W.midwt(y, h, 3)).sum()) < 1e-11
        assert np.abs(W.midwt(W.mdwt(x, h, 3), h, 3) - x).max() < 1e-12


def chambolle_pock(a, u, h, L, iters=4000):
    """min 1/2 |x - a|^2 + I(x >= 0) + u |W x|_1 by the primal-dual method of
    Chambolle and Pock (tau = sigma = 1, |W| = 1)."""
    x = np.maximum(a, 0.0)
    xb = x.copy()
    y = np.zeros_like(a)
    for _ in range(iters):
        y = np.clip(y + W.mdwt(xb, h, L), -u, u)
        xn = np.maximum((x - W.midwt(y, h, L) + a) / 2.0, 0.0)
        xb = 2 * xn - x
        x = xn
    return x


@pytest.mark.parametrize("daub,u", [(2, 0.3), (4, 0.1)])
def test_admm_solves_the_proximal_problem(daub, u):
    rng = np.random.default_rng(3)
    a = rng.standard_normal((16, 16)) + 0.5
    h = W.daubcqf(daub)
    al, it = W.admm(a, u, h, 2, rel_tol=1e-9, max_itr=5000)
    cp = chambolle_pock(a, u, h, 2)
    fa = W.admm_objective(al, a, u, h, 2)
    fc = W.admm_objective(cp, a, u, h, 2)
    assert al.min() >= 0.0
    assert abs(fa - fc) / abs(fc) < 1e-6
    assert np.linalg.norm(al - cp) / np.linalg.norm(cp) < 1e-3
    assert it < 5000


def test_admm_iteration_count_and_zero_input():
    """relativeTol = 0 never stops early: maxItr + 1 iterations, as npg/admm.m
    breaks after its counter exceeds maxItr; a = 0 returns 0 at once."""
    rng = np.random.default_rng(4)
    a = rng.standard_normal((8, 8))
    _, it = W.admm(a, 0.1, W.daubcqf(2), 3, rel_tol=0.0, max_itr=7)
    assert it == 8
    z, it0 = W.admm(np.zeros((8, 8)), 0.1, W.daubcqf(2), 3)
    assert it0 == 0 and not z.any()


def test_wavelet_mask_is_the_reach_of_the_pixels():
    """utils/wvltMask.m: the union of Wt(e_i) != 0 over the mask's pixels.  A
    single pixel reaches one coefficient per quadrant and level with the
    two-tap filter (3 L + 1), more with longer filters; the full image
    reaches every coefficient."""
    h2, h4 = W.daubcqf(2), W.daubcqf(4)
    one = np.zeros((32, 32), bool)
    one[13, 6] = True
    assert W.wvlt_mask(one, h2, 4).sum() == 3 * 4 + 1
    assert W.wvlt_mask(one, h4, 3).sum() > 3 * 3 + 1
    assert W.wvlt_mask(np.ones((16, 16), bool), h4, 2).all()


def test_masked_admm_keeps_the_masks():
    """With masks the ADMM's alpha is zero outside the pixel mask and equals
    the solution of the masked problem (Chambolle-Pock on the masked
    operators)."""
    rng = np.random.default_rng(8)
    yy, xx = np.mgrid[0:16, 0:16]
    mask = ((xx - 7.5) ** 2 + (yy - 7.5) ** 2 < 6.5 ** 2).astype(float)
    h = W.daubcqf(2)
    maskk = W.wvlt_mask(mask, h, 2).astype(float)
    a = (rng.standard_normal((16, 16)) + 0.5) * mask
    al, it = W.admm(a, 0.2, h, 2, rel_tol=1e-9, max_itr=5000, mask=mask, maskk=maskk)
    assert not al[mask == 0].any()
    x = np.maximum(a, 0.0)
    xb = x.copy()
    y = np.zeros_like(a)
    for _ in range(6000):   # the same problem over the masked operators
        y = np.clip(y + W.mdwt(xb * mask, h, 2) * maskk, -0.2, 0.2)
        xn = np.maximum((x - W.midwt(y * maskk, h, 2) * mask + a) / 2.0, 0.0) * mask
        xb = 2 * xn - x
        x = xn
    assert np.linalg.norm(al - x) / np.linalg.norm(x) < 1e-3


@pytest.mark.parametrize("key", ["n64_L3_D2", "n128_L2_D2", "n128_L6_D6"])
def test_wavelet_mask_matches_the_reference_masks(key):
    """The reference ships the coefficient masks its BHC drivers load
    (utils/MaskWvlt<n>CircleL<L>D<D>.mat, written by its own utils/wvltMask.m
    for Utils.getCircularMask(n); copied into tests/golden/wvltmask_golden.npz
    by make_wvltmask_golden.py): the oracle's restatement of both reproduces
    them bit for bit, the 6-tap filter included."""
    z = np.load(MASKS)
    n, L, D, ref = reference_mask(z, key)
    assert np.array_equal(W.wvlt_mask(W.circular_mask(n), W.daubcqf(D), L), ref)

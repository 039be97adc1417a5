"""The fixed windows of the projection kernels hold every run of the
reference's range rules (host-side check of the bounds the kernels rely on;
no GPU).

Forward (k_forward): a ray whose run across a row (prj/cpuPrj.c:365-369
parallel, :514-536 fan) is always narrower than 1.95 (2.95) pixels has, in
every row, its run [round(xl), round(xr)] inside the three pixels centred on
round(xc) (the four from floor(xc) - 1), xc = (xl + xr) / 2, after both are
clamped to the image.  Backward (k_backward_tiled): where the plan's bound on
a pixel shadow is at most 1.9 detectors, the reference's detector range of a
pixel [round(tlo), round(thi)] (its exact corner shadows, prj/cpuPrj.c:218-244)
lies inside the three detectors centred on the projection of its centre tc;
where it is at most 2.85, inside the four from floor(tc) - 1."""
import numpy as np
import pytest

PI_F = np.float32(3.14159265359)
GEOMS = [(2048, 2048, 1440, 8192.0, 1.0, 1.0), (512, 1024, 360, 2048.0, 1.0, 1.0),
         (256, 363, 360, 0.0, 1.0, 1.0), (1024, 1024, 720, 2048.0, 1.0, 1.0),
         (97, 139, 120, 0.0, 0.8, 1.0), (64, 91, 60, 0.0, 0.5, 0.7), (33, 45, 36, 60.0, 1.2, 1.2)]


def view_angles(b, P):
    th = (np.float32(2) * b.astype(np.float32) * PI_F) / np.float32(P)
    return th.astype(np.float64)


@pytest.mark.parametrize("n, W, P, d, bw, dS", GEOMS)
def test_forward_windows_hold_every_run(n, W, P, d, bw, dS):
    half = (n - 1) // 2
    pC = W // 2
    nb = min(P, P // 8 + 1)
    th = view_angles(np.arange(nb), P)
    cT, sT = np.cos(th)[:, None], np.sin(th)[:, None]
    k0 = 1 if W % 2 == 0 else 0
    nk = (W - 1 if W % 2 == 0 else W) if d > 0 else (W // 2 if W % 2 == 0 else (W + 1) // 2)
    t = (k0 + np.arange(nk) - pC) * dS
    tl, tr = t - 0.5 * bw, t + 0.5 * bw
    if d > 0:
        qxl, qyl = tl * cT + d * sT, -tl * sT + d * cT
        qxr, qyr = tr * cT + d * sT, -tr * sT + d * cT
        Al = (d * tl - np.where(qxl > 0, 0.5, -0.5) * qxl) / qyl
        Ar = (d * tr + np.where(qxr > 0, 0.5, -0.5) * qxr) / qyr
        Sl, Sr = qxl / qyl, qxr / qyr
    else:
        Al, Ar = (tl - 0.5 * sT) / cT, (tr + 0.5 * sT) / cT
        Sl = Sr = np.broadcast_to(sT / cT, Al.shape)
    Al, Sl, Ar, Sr = (np.asarray(v, np.float32) for v in (Al, Sl, Ar, Sr))
    wa, ws = Ar - Al, Sr - Sl
    wmax = np.maximum(np.abs(wa - half * ws), np.abs(wa + half * ws))
    code = np.where(wmax < 1.95, 3, np.where(wmax < 2.95, 4, 5))
    for j in range(0, nk, 32):   # the warp takes the widest window its rays need
        code[:, j:j + 32] = code[:, j:j + 32].max(1, keepdims=True)
    Ac, Sc = np.float32(0.5) * (Al + Ar), np.float32(0.5) * (Sl + Sr)
    checked = 0
    for y in range(-half, half + 1, max(1, n // 64)):
        yf = np.float32(y)
        xl, xr, xc = -yf * Sl + Al, -yf * Sr + Ar, -yf * Sc + Ac
        x0, x1 = np.maximum(np.round(xl), -half), np.minimum(np.round(xr), half)
        run = x0 <= x1
        for wn in (3, 4):
            m = (code == wn) & run
            skipped = (xc < -half - 2) | (xc > half + 2)
            assert not (m & skipped).any()
            xs = np.clip((np.round(xc) if wn == 3 else np.floor(xc)) - 1, -half, half - (wn - 1))
            assert not (m & ((x0 < xs) | (x1 > xs + wn - 1))).any()
            checked += m.sum()
    assert checked > 0


@pytest.mark.parametrize("n, W, P, d, bw, dS", [g for g in GEOMS if g[4] <= 1.0])
def test_backward_window_holds_every_shadow(n, W, P, d, bw, dS):
    half = (n - 1) // 2
    R = (half + 1.0) * np.sqrt(2.0)
    if d > 0:
        if not d > 2 * R:
            pytest.skip("source too close for the bound")
        tg = R / (d - R)
        bound = np.sqrt(2.0) * d / (d - R) * (1 + tg * tg) / dS
    else:
        bound = np.sqrt(2.0) / dS
    if bound > 2.85:
        pytest.skip("the plan keeps the per-pixel range here (bound %.2f)" % bound)
    rng = np.random.default_rng(n)
    x = rng.integers(0, half + 1, 400000).astype(np.float64)
    y = rng.integers(0, half + 1, 400000).astype(np.float64)
    keep = y <= x
    x, y = x[keep], y[keep]
    th = view_angles(rng.integers(0, P, x.size), P)
    c, s = np.cos(th), np.sin(th)
    u = x * c + y * s
    if d > 0:
        qe = d - (y * c - x * s)
        ts = np.array([d * ((x + ex) * c + (y + ey) * s) / ((x + ex) * s - (y + ey) * c + d)
                       for ex, ey in ((-.5, -.5), (.5, -.5), (.5, .5), (-.5, .5))])
        tlo, thi, tc = ts.min(0) / dS, ts.max(0) / dS, d * u / qe / dS
    else:
        hw = 0.5 * (np.abs(c) + np.abs(s))
        tlo, thi, tc = (u - hw) / dS, (u + hw) / dS, u / dS
    assert (thi - tlo).max() <= bound * (1 + 1e-9)
    if bound <= 1.9:   # three detectors centred on round(tc)
        k = np.round(tc)
        assert (np.round(tlo) >= k - 1).all() and (np.round(thi) <= k + 1).all()
    else:              # four detectors from floor(tc) - 1
        k = np.floor(tc)
        assert (np.round(tlo) >= k - 1).all() and (np.round(thi) <= k + 2).all()

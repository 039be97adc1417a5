"""Seeded synthetic inputs with the shapes and value distributions of the
reference's workloads (it ships no data for the projector).

ellipse_phantom: 10 ellipses, centres uniform in the unit disc, semi-axes
U(0.05, 0.4), rotation U(0, pi), additive densities U(-0.5, 1.0), clipped at 0;
the unit square [-1, 1]^2 covers the n x n grid.
two_material_phantom: ellipses of aluminium (2.7 g/cm^3) and iron (7.8 g/cm^3)
in air (0), painted in order.
"""
import numpy as np


def _grid(n):
    c = (np.arange(n) - n // 2) / (n / 2.0)     # pixel index -> centred coordinate
    return np.meshgrid(c, c)                    # X varies along columns, Y along rows


def _ellipse_mask(X, Y, cx, cy, a, b, phi):
    cp, sp = np.cos(phi), np.sin(phi)
    u = (X - cx) * cp + (Y - cy) * sp
    v = -(X - cx) * sp + (Y - cy) * cp
    return (u / a) ** 2 + (v / b) ** 2 <= 1.0


def _draw(rng, k):
    r = np.sqrt(rng.uniform(0, 1, k))
    t = rng.uniform(0, 2 * np.pi, k)
    return (r * np.cos(t), r * np.sin(t), rng.uniform(0.05, 0.4, k), rng.uniform(0.05, 0.4, k),
            rng.uniform(0, np.pi, k))


def ellipse_phantom(n, seed=0, count=10):
    rng = np.random.default_rng(seed)
    X, Y = _grid(n)
    img = np.zeros((n, n), np.float64)
    cx, cy, a, b, phi = _draw(rng, count)
    dens = rng.uniform(-0.5, 1.0, count)
    for i in range(count):
        img[_ellipse_mask(X, Y, cx[i], cy[i], a[i], b[i], phi[i])] += dens[i]
    return np.clip(img, 0, None).astype(np.float32)


def two_material_phantom(n, seed=0, count=10, fe_fraction=0.3):
    rng = np.random.default_rng(seed)
    X, Y = _grid(n)
    img = np.zeros((n, n), np.float64)
    # a body of aluminium, then inclusions of either material
    img[_ellipse_mask(X, Y, 0.0, 0.0, rng.uniform(0.6, 0.8), rng.uniform(0.5, 0.7),
                      rng.uniform(0, np.pi))] = 2.7
    cx, cy, a, b, phi = _draw(rng, count - 1)
    fe = rng.uniform(0, 1, count - 1) < fe_fraction
    for i in range(count - 1):
        m = _ellipse_mask(X, Y, 0.6 * cx[i], 0.6 * cy[i], 0.5 * a[i], 0.5 * b[i], phi[i])
        img[m] = 7.8 if fe[i] else 2.7
    return img.astype(np.float32)


def spectrum_bump(J, seed=0):
    """Seeded smooth bump of J non-negative spectrum coefficients, positive
    everywhere and normalised to sum 1."""
    rng = np.random.default_rng(seed)
    mu = rng.uniform(0.35, 0.65) * (J - 1)
    sig = rng.uniform(0.08, 0.15) * J
    I = np.exp(-0.5 * ((np.arange(J) - mu) / sig) ** 2) + 1e-3
    return I / I.sum()

"""FP64 restatement of the reference's polychromatic beam-hardening model --
TEST INFRASTRUCTURE ONLY (the oracle; never imported by the product).

Follows bhc/Spline.m:122-203 (b1Iout: Laplace transforms of the degree-1
B-spline mass-attenuation basis, with their first and second derivatives and
the cubic Taylor branch near s = 0), bhc/poissLAlpha.m:1-19 (Poisson negative
log-likelihood in the density and its gradient through Phi^T),
bhc/poissLI.m:1-27 (the same in the spectrum coefficients, with the Hessian),
the Gaussian (log-domain least-squares) pair bhc/gaussLAlpha.m:1-34 and
bhc/gaussLI.m:1-27, the density Hessians of both (the `hessian` closures of
poissLAlpha / gaussLAlpha) and the kappa grid rule of
bhc/beamhardenSpline.m:137-165.

The reference is MATLAB and cannot run here: parity of this restatement is
unpinned against the reference's own outputs; it is cross-checked against
numerical quadrature of the defining integrals and against central finite
differences (tests/test_bhc_oracle.py).
"""
import numpy as np

TAYLOR_EPS = 1e-6   # bhc/Spline.m:128


def kappa_nodes(J, kmin=1e-2, kmax=1e2):
    """J log-spaced mass-attenuation values on [kmin, kmax] padded with one node
    on each side at the same ratio q = kappa_2 / kappa_1
    (bhc/beamhardenSpline.m:164-165): J + 2 B-spline nodes."""
    kappa = np.logspace(np.log10(kmin), np.log10(kmax), J)
    q = kappa[1] / kappa[0]
    return np.concatenate([[kappa[0] / q], kappa, [kappa[-1] * q]])


def taylor_tables(k):
    """Per basis function j (nodes a, b, c = k[j], k[j+1], k[j+2]): cubic Taylor
    coefficients of b_j, b_j' and b_j'' about s = 0 and the |s| below which the
    reference switches to them (bhc/Spline.m:156-165, :173-181, :189-197)."""
    k = np.asarray(k, np.float64)
    J = k.size - 2
    T = {"B": np.zeros((J, 4)), "D": np.zeros((J, 4)), "DD": np.zeros((J, 4)),
         "thrB": np.zeros(J), "thrD": np.zeros(J), "thrDD": np.zeros(J)}
    for j in range(J):
        a, b, c = k[j], k[j + 1], k[j + 2]
        B = [-a / 2 + c / 2,
             (a ** 3 - b ** 3) / (6 * (a - b)) - (b ** 3 - c ** 3) / (6 * (b - c)),
             -(a ** 4 - b ** 4) / (24 * (a - b)) + (b ** 4 - c ** 4) / (24 * (b - c)),
             (a ** 5 - b ** 5) / (120 * (a - b)) - (b ** 5 - c ** 5) / (120 * (b - c))]
        D = [(a ** 3 - b ** 3) / (6 * (a - b)) - (b ** 3 - c ** 3) / (6 * (b - c)),
             -(a ** 4 - b ** 4) / (12 * (a - b)) + (b ** 4 - c ** 4) / (12 * (b - c)),
             (a ** 5 - b ** 5) / (40 * (a - b)) - (b ** 5 - c ** 5) / (40 * (b - c)),
             -(a ** 6 - b ** 6) / (180 * (a - b)) + (b ** 6 - c ** 6) / (180 * (b - c))]
        DD = [-((a + b) * (a * a + b * b)) / 12 + ((b + c) * (b * b + c * c)) / 12,
              (a ** 4 + a ** 3 * b + a * a * b * b + a * b ** 3 + b ** 4) / 20
              - (b ** 4 + b ** 3 * c + b * b * c * c + b * c ** 3 + c ** 4) / 20,
              -((a + b) * (a * a + a * b + b * b) * (a * a - a * b + b * b)) / 60
              + ((b + c) * (b * b + b * c + c * c) * (b * b - b * c + c * c)) / 60,
              (a ** 6 + a ** 5 * b + a ** 4 * b * b + a ** 3 * b ** 3 + a * a * b ** 4 + a * b ** 5 + b ** 6) / 252
              - (b ** 6 + b ** 5 * c + b ** 4 * c * c + b ** 3 * c ** 3 + b * b * c ** 4 + b * c ** 5 + c ** 6) / 252]
        for name, co, thr in (("B", B, "thrB"), ("D", D, "thrD"), ("DD", DD, "thrDD")):
            T[name][j] = co
            T[thr][j] = abs(TAYLOR_EPS * co[0] / co[3]) ** (1.0 / 3.0)
    return T


def b1_basis(k, s, derivs=2):
    """Columns b_j(s), b_j'(s), b_j''(s) for j = 0..J-1 (bhc/Spline.m:139-203
    with I empty).  s is a vector of projections; returns arrays (len(s), J)."""
    k = np.asarray(k, np.float64)
    s = np.asarray(s, np.float64).ravel()
    J = k.size - 2
    T = taylor_tables(k)
    B = np.zeros((s.size, J))
    D = np.zeros((s.size, J))
    DD = np.zeros((s.size, J))
    s2, s3, s4, abss = s * s, s ** 3, s ** 4, np.abs(s)
    with np.errstate(divide="ignore", invalid="ignore", over="ignore"):
        eC = np.exp(-k[0] * s)
        eR = np.exp(-k[1] * s)
        for j in range(J):
            a, b, c = k[j], k[j + 1], k[j + 2]
            eL, eC, eR = eC, eR, np.exp(-c * s)
            v = -(eL - eC) / (s2 * (a - b)) + (eC - eR) / (s2 * (b - c))
            idx = abss < T["thrB"][j]
            co = T["B"][j]
            v[idx] = co[0] + s[idx] * co[1] + s2[idx] * co[2] + s3[idx] * co[3]
            B[:, j] = v
            if derivs >= 1:
                v = (2 * (eL - eC) / (s3 * (a - b)) + (a * eL - b * eC) / (s2 * (a - b))
                     - 2 * (eC - eR) / (s3 * (b - c)) - (b * eC - c * eR) / (s2 * (b - c)))
                idx = abss < T["thrD"][j]
                co = T["D"][j]
                v[idx] = co[0] + s[idx] * co[1] + s2[idx] * co[2] + s3[idx] * co[3]
                D[:, j] = v
            if derivs >= 2:
                v = (-(6 * eL - 6 * eC + s2 * (a * a * eL - b * b * eC) + s * (4 * a * eL - 4 * b * eC))
                     / (s4 * (a - b))
                     + (6 * eC - 6 * eR + s2 * (b * b * eC - c * c * eR) + s * (4 * b * eC - 4 * c * eR))
                     / (s4 * (b - c)))
                idx = abss < T["thrDD"][j]
                co = T["DD"][j]
                v[idx] = co[0] + s[idx] * co[1] + s2[idx] * co[2] + s3[idx] * co[3]
                DD[:, j] = v
    return B, D, DD


def b1_iout(k, s, I):
    """[BL, sBL, ssBL] = Spline.b1Iout(k, s, I): the spectrum-weighted sums."""
    B, D, DD = b1_basis(k, s)
    I = np.asarray(I, np.float64).ravel()
    return B @ I, D @ I, DD @ I


def poisson_terms(BL, imea):
    """Per-ray f_i = BL_i - m_i - m_i log(BL_i / m_i) (bhc/poissLAlpha.m:10-11),
    with m_i log(BL_i / m_i) taken as 0 where m_i = 0 (zero counts)."""
    BL = np.asarray(BL, np.float64)
    m = np.asarray(imea, np.float64)
    with np.errstate(divide="ignore", invalid="ignore"):
        lg = np.where(m > 0, m * np.log(BL / np.where(m > 0, m, 1.0)), 0.0)
    return BL - m - lg


def poiss_alpha(imea, Ie, s, k, backproject):
    """bhc/poissLAlpha.m for the projections s = Phi(alpha): returns
    (f, grad_alpha, per-ray weight w) with grad = backproject(w),
    w = (1 - m / BL) * sBL."""
    BL, sBL, _ = b1_iout(k, s, Ie)
    m = np.asarray(imea, np.float64).ravel()
    f = poisson_terms(BL, m).sum()
    w = (1 - m / BL) * sBL
    return f, backproject(w), w


def poiss_hessian_weight(imea, Ie, s, k):
    """Per-ray weight of the density Hessian of poissLAlpha
    (bhc/poissLAlpha.m:15): (sBL/BL)^2 m + ssBL (1 - m/BL); the Hessian is
    Phi^T diag(weight) Phi."""
    BL, sBL, ssBL = b1_iout(k, s, Ie)
    m = np.asarray(imea, np.float64).ravel()
    return (sBL / BL) ** 2 * m + ssBL * (1 - m / BL)


def gauss_alpha(imea, Ie, s, k, backproject):
    """bhc/gaussLAlpha.m:1-20: Err = log(BL/m), f = Err'Err/2,
    grad = backproject(Err sBL / BL); returns (f, grad, per-ray weight)."""
    BL, sBL, _ = b1_iout(k, s, Ie)
    m = np.asarray(imea, np.float64).ravel()
    err = np.log(BL / m)
    w = err * sBL / BL
    return 0.5 * err @ err, backproject(w), w


def gauss_hessian_weight(imea, Ie, s, k):
    """bhc/gaussLAlpha.m:18: (1 - Err)(sBL/BL)^2 + Err ssBL/BL."""
    BL, sBL, ssBL = b1_iout(k, s, Ie)
    m = np.asarray(imea, np.float64).ravel()
    err = np.log(BL / m)
    return (1 - err) * (sBL / BL) ** 2 + err * ssBL / BL


def gauss_ie(imea, A, Ie):
    """bhc/gaussLI.m:1-27: Ir = A Ie, Err = log(Ir/m), f = Err'Err/2,
    g = A^T (Err / Ir), H = A^T diag((1 - Err) / Ir^2) A."""
    Ir = A @ np.asarray(Ie, np.float64)
    m = np.asarray(imea, np.float64).ravel()
    err = np.log(Ir / m)
    return 0.5 * err @ err, A.T @ (err / Ir), A.T @ (A * ((1 - err) / Ir ** 2)[:, None])


def poiss_ie(imea, A, Ie):
    """bhc/poissLI.m: f, gradient A^T (1 - m / Ir) and Hessian
    A^T diag(m / Ir^2) A in the spectrum coefficients, with Ir = A Ie."""
    Ir = A @ np.asarray(Ie, np.float64)
    m = np.asarray(imea, np.float64).ravel()
    f = poisson_terms(Ir, m).sum()
    g = A.T @ (1 - m / Ir)
    H = A.T @ (A * (m / Ir ** 2)[:, None])
    return f, g, H


def spectrum_bump(J, seed=0):
    """A smooth seeded bump over the J coefficients, positive everywhere,
    normalised to sum 1."""
    rng = np.random.default_rng(seed)
    mu = rng.uniform(0.35, 0.65) * (J - 1)
    sig = rng.uniform(0.08, 0.15) * J
    I = np.exp(-0.5 * ((np.arange(J) - mu) / sig) ** 2) + 1e-3
    return I / I.sum()

"""The q = 1 weak-identification interval of Kline, Saggio and Solvsten
(2020, Section 6.1 and Appendix C.6), with the curvature-adjusted critical
value of Andrews and Mikusheva (2016).  Host arithmetic on a handful of
scalars; the moments it takes come from the device
(`StandardErrors.weak_moments`).  The reference computes the same interval
(am_interval.py `am_interval`); this module derives it independently:

Critical value.  With xi_1, xi_2 independent standard normals and c =
1/kappa, the statistic is rho = ((xi_1)^2 + (|xi_2| + c)^2)^(1/2) - c, so
rho <= z exactly when (xi_1, |xi_2| + c) lies in the disc of radius R = z + c
about the origin.  Integrating over x = xi_1 first, |xi_2| must lie below
(R^2 - x^2)^(1/2) - c, which needs |x| <= X = (z (z + 2c))^(1/2):

    F(z) = int_{-X}^{X} phi(x) (2 Phi((R^2 - x^2)^(1/2) - c) - 1) dx.

The substitution x = X sin(u) turns R^2 - x^2 into c^2 + X^2 cos(u)^2, so
the integrand becomes analytic on [0, pi/2] (no square-root end point, even as
c -> 0) and a fixed Gauss-Legendre rule integrates it to rounding error.
F'(z), the density of rho, has the same form, so z_{alpha, kappa} = F^{-1}(1 -
alpha) comes from Newton's method kept inside the bracket between the
chi-squared(1) quantile (kappa = 0) and the chi-squared(2) one (kappa ->
infinity).

Extremes.  The interval is the range of lambda_1 b^2 + t over the ellipse
{(b1 - b, theta1 - t) Sigma^-1 (.)' <= z^2}; the objective increases one for
one with t, so the extremes lie on the boundary, (b, t) = (b1, theta1) + z L
(cos u, sin u) with L the Cholesky factor of Sigma.  There the first-order
condition, in (cos u, sin u) = (x, y), is y (A + B x) = C x with A = 2
lambda_1 p b1 + a, B = 2 lambda_1 p^2, C the sine coefficient; squaring with
y^2 = 1 - x^2 gives KSS's quartic (Appendix C.6.2)

    (1 - x^2)(A + B x)^2 - C^2 x^2 = 0,

whose real roots in [-1, 1] give at most four stationary points.  Each is
polished by Newton's method on the angle and the smallest and largest values
of the objective there (and at u = 0, pi) are the interval.
"""

from __future__ import annotations

import math

import numpy as np

# Gauss-Legendre rule on [0, 1], mapped onto the angle range in use
_NODES = 128
_GL_T, _GL_W = np.polynomial.legendre.leggauss(_NODES)
_GL_T, _GL_W = 0.5 * (_GL_T + 1.0), 0.5 * _GL_W
_INV_SQRT_2PI = 1.0 / math.sqrt(2.0 * math.pi)
_X_CUT = 9.0            # phi(9) ~ 1e-18: |x| beyond it adds nothing


def _pdf(x):
    return _INV_SQRT_2PI * np.exp(-0.5 * x * x)


def _rho_cdf_pdf(z: float, c: float):
    """(F(z), F'(z)) of rho for c = 1/kappa > 0: the x-integral over
    [0, min(X, 9)] (twice, by symmetry) after x = X sin(u)."""
    from scipy.special import ndtr
    X = math.sqrt(z * (z + 2.0 * c))
    u_max = 0.5 * math.pi if X <= _X_CUT else math.asin(_X_CUT / X)
    u = u_max * _GL_T
    w = u_max * _GL_W
    cu = np.cos(u)
    xc2 = (X * cu) ** 2
    s = np.sqrt(c * c + xc2)                       # (R^2 - x^2)^(1/2) at x = X sin(u)
    gap = xc2 / (s + c)                            # s - c without cancellation
    jac = X * cu                                   # dx / du
    phi_x = _pdf(X * np.sin(u))
    F = 2.0 * float(np.sum(w * phi_x * (2.0 * ndtr(gap) - 1.0) * jac))
    # d/dz of the inner term: 2 phi(s - c) ds/dz with ds/dz = R / s (the
    # integrand vanishes at x = +-X, so the limits contribute nothing)
    dF = 2.0 * float(np.sum(w * phi_x * 2.0 * _pdf(gap) * ((z + c) / s) * jac))
    return F, dF


def am_cdf(z: float, kappa: float) -> float:
    """P(rho(kappa) <= z)."""
    from scipy.special import ndtr
    if z <= 0.0:
        return 0.0
    if kappa <= 0.0:
        return float(2.0 * ndtr(z) - 1.0)
    return _rho_cdf_pdf(z, 1.0 / kappa)[0]


def am_critical_value(kappa: float, alpha: float = 0.05) -> float:
    """z_{alpha, kappa}: the (1 - alpha) quantile of rho(kappa)."""
    from scipy.special import chdtri
    lo = math.sqrt(float(chdtri(1, alpha)))
    if kappa <= 0.0:
        return lo
    hi = math.sqrt(float(chdtri(2, alpha)))
    c = 1.0 / kappa
    target = 1.0 - alpha
    z = 0.5 * (lo + hi)
    for _ in range(100):
        F, dF = _rho_cdf_pdf(z, c)
        r = F - target
        if r > 0.0:
            hi = min(hi, z)
        else:
            lo = max(lo, z)
        step = r / dF if dF > 0.0 else 0.0
        nz = z - step
        if not lo < nz < hi:                      # keep Newton inside the bracket
            nz = 0.5 * (lo + hi)
        if abs(nz - z) <= 1e-15 * z:
            z = nz
            break
        z = nz
    return float(z)


def curvature(lam1: float, sigma) -> float:
    """kappa = 2 |lambda_1| V[b1] / (V[theta1] (1 - r^2))^(1/2), r the
    correlation of (b1, theta1)."""
    vb, vt, cv = float(sigma[0][0]), float(sigma[1][1]), float(sigma[0][1])
    return 2.0 * abs(lam1) * vb / math.sqrt(vt - cv * cv / vb)


def _stationary_angles(A: float, B: float, C: float):
    """Angles u where sin(u) (A + B cos u) = C cos u, from the quartic in
    x = cos u (plus u = 0 and pi, where the squared form can lose roots)."""
    # (1 - x^2)(A + B x)^2 - C^2 x^2, highest power first
    q = np.array([-B * B, -2.0 * A * B, B * B - A * A - C * C, 2.0 * A * B, A * A])
    nz = np.flatnonzero(np.abs(q) > 0.0)
    angles = [0.0, math.pi]
    if len(nz):
        roots = np.roots(q[nz[0]:]) if len(q) - nz[0] > 1 else []
        for x in roots:
            if abs(x.imag) > 1e-6 or abs(x.real) > 1.0 + 1e-9:
                continue
            x = min(1.0, max(-1.0, float(x.real)))
            y = math.sqrt(max(1.0 - x * x, 0.0))
            angles += [math.atan2(y, x), math.atan2(-y, x)]
    return angles


def am_interval(lam1: float, b1: float, theta1: float, sigma, alpha: float = 0.05):
    """(lower, upper, {"kappa", "z", "rho"}) of the q = 1 interval; sigma
    the positive-definite 2x2 covariance of (b1, theta1)."""
    sigma = np.asarray(sigma, dtype=np.float64)
    kappa = curvature(lam1, sigma)
    z = am_critical_value(kappa, alpha)
    l00 = math.sqrt(sigma[0, 0])
    l10 = sigma[1, 0] / l00
    l11 = math.sqrt(max(sigma[1, 1] - l10 * l10, 0.0))
    p, a, s = z * l00, z * l10, z * l11

    def g(u):
        x = b1 + p * math.cos(u)
        return lam1 * x * x + theta1 + a * math.cos(u) + s * math.sin(u)

    def dg(u):
        return math.sin(u) * (-2.0 * lam1 * p * (b1 + p * math.cos(u)) - a) + s * math.cos(u)

    def d2g(u):
        c, sn = math.cos(u), math.sin(u)
        return (-2.0 * lam1 * p * (c * (b1 + p * c) - p * sn * sn) - a * c - s * sn)

    values = []
    for u in _stationary_angles(2.0 * lam1 * p * b1 + a, 2.0 * lam1 * p * p, s):
        for _ in range(8):                         # the quartic's roots to full precision
            h = d2g(u)
            if h == 0.0:
                break
            du = dg(u) / h
            if abs(du) > 1e-3:                     # not near a root of the unsquared form
                break
            u -= du
            if abs(du) < 1e-16:
                break
        values.append(g(u))
    rho = float(sigma[0, 1] / math.sqrt(sigma[0, 0] * sigma[1, 1]))
    return min(values), max(values), {"kappa": float(kappa), "z": float(z), "rho": rho}

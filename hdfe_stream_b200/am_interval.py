"""The q = 1 weak-identification interval of Kline, Saggio and Solvsten
(2020, Section 6.1), with the Andrews-Mikusheva (2016) curvature-adjusted
critical value (am_interval.py `am_interval`).  Host arithmetic on a handful
of scalars; the moments it takes come from the device
(`StandardErrors.weak_moments`).

The interval is the range of lambda_1 b^2 + t over the ellipse
{(b1 - b, theta1 - t) Sigma^-1 (.)' <= z^2}.  z is the (1 - alpha) quantile
of rho = sqrt(chi_1^2 + (chi_1' + 1/kappa)^2) - 1/kappa for the curvature
kappa = 2 |lambda_1| V[b1] / (V[theta1] (1 - r^2))^(1/2), r the correlation
of (b1, theta1): for two independent half-normals a, b and c = 1/kappa,
rho <= z exactly when a^2 + (b + c)^2 <= (z + c)^2, so

    P(rho <= z) = int_0^z 2 phi(b) (2 Phi(((z - b)(z + b + 2c))^(1/2)) - 1) db,

one quadrature, between the chi-squared(1) quantile (kappa = 0) and the
chi-squared(2) one (kappa -> infinity).  The extremes lie on the ellipse's
boundary (the map moves one for one with t), where the objective is a
trigonometric polynomial of degree two in the angle: a dense grid brackets
each extreme and Newton's method on the angle's first-order condition polishes
it.
"""

from __future__ import annotations

import math

import numpy as np

GRID = 4096


def _phi(b):
    return math.exp(-0.5 * b * b) / math.sqrt(2.0 * math.pi)


def am_cdf(z: float, kappa: float) -> float:
    """P(rho(kappa) <= z)."""
    from scipy import integrate, special
    if z <= 0.0:
        return 0.0
    if kappa <= 0.0:
        return float(2.0 * special.ndtr(z) - 1.0)
    c = 1.0 / kappa

    def f(b):
        r = math.sqrt(max((z - b) * (z + b + 2.0 * c), 0.0))
        return 2.0 * _phi(b) * (2.0 * special.ndtr(r) - 1.0)

    value, _ = integrate.quad(f, 0.0, z, epsabs=1e-13, epsrel=1e-12, limit=200)
    return float(value)


def am_critical_value(kappa: float, alpha: float = 0.05) -> float:
    """z_{alpha, kappa}: the (1 - alpha) quantile of rho(kappa)."""
    from scipy import optimize, special
    z1 = math.sqrt(float(special.chdtri(1, alpha)))
    if kappa <= 0.0:
        return z1
    z2 = math.sqrt(float(special.chdtri(2, alpha)))
    return float(optimize.brentq(lambda z: am_cdf(z, kappa) - (1.0 - alpha), z1 * (1 - 1e-9),
                                 z2 * (1 + 1e-9), xtol=1e-13, rtol=1e-13))


def curvature(lam1: float, sigma) -> float:
    """kappa = 2 |lambda_1| V[b1] / (V[theta1] (1 - r^2))^(1/2)."""
    vb, vt, cv = float(sigma[0][0]), float(sigma[1][1]), float(sigma[0][1])
    return 2.0 * abs(lam1) * vb / math.sqrt(vt * (1.0 - cv * cv / (vb * vt)))


def am_interval(lam1: float, b1: float, theta1: float, sigma, alpha: float = 0.05):
    """(lower, upper, {"kappa", "z", "rho"}) of the q = 1 interval; sigma
    the positive-definite 2x2 covariance of (b1, theta1)."""
    sigma = np.asarray(sigma, dtype=np.float64)
    kappa = curvature(lam1, sigma)
    z = am_critical_value(kappa, alpha)
    l00 = math.sqrt(sigma[0, 0])
    l10 = sigma[1, 0] / l00
    l11 = math.sqrt(max(sigma[1, 1] - l10 * l10, 0.0))
    p, a, bb = z * l00, z * l10, z * l11

    # g(t) = lam1 (b1 + p cos t)^2 + theta1 + a cos t + bb sin t on the boundary
    def g(t):
        x = b1 + p * np.cos(t)
        return lam1 * x * x + theta1 + a * np.cos(t) + bb * np.sin(t)

    def dg(t):
        x = b1 + p * math.cos(t)
        return -2.0 * lam1 * p * math.sin(t) * x - a * math.sin(t) + bb * math.cos(t)

    def d2g(t):
        x = b1 + p * math.cos(t)
        return (-2.0 * lam1 * p * (math.cos(t) * x - p * math.sin(t) ** 2)
                - a * math.cos(t) - bb * math.sin(t))

    ts = np.linspace(0.0, 2.0 * math.pi, GRID, endpoint=False)
    vals = g(ts)
    step = ts[1] - ts[0]

    def polish(t0):
        """g at the stationary point Newton reaches from t0 without leaving
        the grid cells beside it."""
        t = t0
        for _ in range(50):
            h = d2g(t)
            if h == 0.0:
                break
            nt = t - dg(t) / h
            if abs(nt - t0) > step:
                break
            done = abs(nt - t) < 1e-15
            t = nt
            if done:
                break
        return float(g(t))

    lower = min(polish(ts[int(np.argmin(vals))]), float(vals.min()))
    upper = max(polish(ts[int(np.argmax(vals))]), float(vals.max()))
    rho = float(sigma[0, 1] / math.sqrt(sigma[0, 0] * sigma[1, 1]))
    return lower, upper, {"kappa": float(kappa), "z": float(z), "rho": rho}

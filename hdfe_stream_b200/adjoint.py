"""Gradients through the fixed-effects solve: a torch.autograd.Function.

The fit of y = X beta + sum_d D_d gamma_d + D_g alpha + e by weighted least
squares gives theta = (beta, gamma, alpha) = (Z'WZ)^- Z'W y with Z the whole
design (covariates, the non-streamed levels, the streamed groups).  For an
objective f(theta) with gradient c = df/dtheta,

    df/dy_i = w_i (Z u)_i,        df/dw_i = (Z u)_i e_i   (through theta),

where u = (Z'WZ)^- c and e the fit's residuals: dtheta/dy = (Z'WZ)^- Z'W, and
for weighted least squares dtheta/dw_i = (Z'WZ)^- z_i e_i.  So the backward
pass is one more application of the inverse of the same self-adjoint
operator, `InverseOperator.apply_inverse` (S^- with the covariates' Schur
border, the streamed block eliminated), whose row readout (Z u)_i is the
scatter back to the rows; no Krylov state is kept from the forward solve, the
backward one recomputes its own.

The normal equations are singular along the fixed effects' normalisations
(a constant moved between dimensions or into the groups).  The forward pass
reports normalised effects (`fit.normalize`, the reference's rule) and the
backward pass solves with that null space removed, so gradients are exact for
objectives that do not depend on the normalisation: the coefficients beta,
and variances and covariances of the effects within a connected set (the
plug-in AKM components).  `plug_in_components` builds those from the
differentiable outputs.

The y-gradient of a weighted sum of predictions is the reference's own
influence output (normal_equations.py:69-73, `solve_normal_equations` with
`predict`), which is what this generalises.
"""

from __future__ import annotations

import numpy as np

from . import fit as _fit
from .leaveout import InverseOperator


def _torch():
    import torch
    return torch


def _design(gcode, codes, y, X, w, n_levels):
    torch = _torch()
    V = torch.cat([y[None, :], X.T], 0).contiguous() if X is not None and X.shape[1] else \
        y[None, :].contiguous()
    return _fit.DeviceRows(gcode, codes, V, w, list(n_levels))


class FixedEffectsSolve:
    """The differentiable fit: `FixedEffectsSolve.apply(y, w, gcode, codes,
    X, n_levels, tol)` -> (beta (c,), gamma (L,), alpha (G,), e (N,)), every
    row in pass 0's layout on the device; y (N,) and w (N,) may require
    grad (w None: unweighted).  e is returned for inspection and carries no
    gradient."""

    @staticmethod
    def _forward(y, w, gcode, codes, X, n_levels, tol):
        torch = _torch()
        rows = _design(gcode, codes, y.detach().to(torch.float64).contiguous(),
                       None if X is None else X.detach(),
                       None if w is None else w.detach().to(torch.float64).contiguous(),
                       n_levels)
        res = _fit.fit(rows, tol=tol, small_block=False)     # the backward pass needs S whole
        op = InverseOperator(rows, res.cells, res.S, None if X is None else rows.V[1:].T,
                             tol=tol)
        A = op.residual_moments(res.gamma).cpu().numpy()
        beta = np.linalg.solve(A[1:, 1:], A[1:, 0]) if A.shape[0] > 1 else np.zeros(0)
        e, alpha, gam_y, _ = op.row_effects(res.gamma, beta)
        beta_t = torch.as_tensor(beta, dtype=torch.float64, device=y.device)
        return beta_t, gam_y, alpha, e, op

    @classmethod
    def apply(cls, y, w, gcode, codes, X, n_levels, tol=1e-12):
        return _FESolveFunction.apply(y, w, gcode, codes, X, tuple(n_levels), float(tol))


def _make_function():
    torch = _torch()

    class FESolveFunction(torch.autograd.Function):
        @staticmethod
        def forward(ctx, y, w, gcode, codes, X, n_levels, tol):
            beta, gam, alpha, e, op = FixedEffectsSolve._forward(y, w, gcode, codes, X, n_levels,
                                                                 tol)
            ctx.op = op
            ctx.has_w = w is not None
            ctx.save_for_backward(e, w if w is not None else e.new_ones(0))
            ctx.mark_non_differentiable(e)
            return beta, gam, alpha, e

        @staticmethod
        def backward(ctx, g_beta, g_gam, g_alpha, g_e):
            op = ctx.op
            e, w = ctx.saved_tensors
            f64 = dict(dtype=torch.float64, device=e.device)
            c = op.c
            g_beta = torch.zeros(c, **f64) if g_beta is None else g_beta.to(**f64)
            g_gam = torch.zeros(op.L, **f64) if g_gam is None else g_gam.to(**f64)
            g_alpha = torch.zeros(op.G, **f64) if g_alpha is None else g_alpha.to(**f64)
            levels = g_gam[:, None].contiguous()
            cov = g_beta[:, None].contiguous()
            groups = g_alpha[:, None].contiguous()
            _, _, _, rows = op.apply_inverse(levels, cov, groups, rows=True)
            r = rows[:, 0]
            grad_y = r * w if ctx.has_w else r.clone()
            grad_w = r * e if ctx.has_w else None
            return grad_y, grad_w, None, None, None, None, None

    return FESolveFunction


class _Lazy:
    fn = None

    def apply(self, *args):
        if _Lazy.fn is None:
            _Lazy.fn = _make_function()
        return _Lazy.fn.apply(*args)


_FESolveFunction = _Lazy()


def plug_in_components(gamma, alpha, w, gcode, codes, n_levels, psi_column=0):
    """The plug-in AKM components (var(psi), var(alpha), cov(psi, alpha))
    from the fit's effects, weighted by w over rows with the n - 1 divisor
    (leaveout.py:807-833), as differentiable torch expressions: gamma (L,)
    the non-streamed effects, alpha (G,) the streamed ones, rows in pass 0's
    order (gcode (N,), codes (N, D))."""
    torch = _torch()
    N = codes.shape[0]
    offs = np.concatenate(([0], np.cumsum(n_levels)[:-1])).astype(np.int64)
    lev = codes[:, psi_column].to(torch.int64) + int(offs[psi_column])
    psi = gamma[lev]
    _, sizes = torch.unique_consecutive(gcode, return_counts=True)
    a = torch.repeat_interleave(alpha, sizes)
    ww = torch.ones(N, dtype=torch.float64, device=gamma.device) if w is None else w
    T = ww.sum()
    scale = N / (N - 1.0) if N > 1 else 1.0
    ma, mb = (ww * psi).sum() / T, (ww * a).sum() / T
    var_psi = scale * ((ww * psi * psi).sum() / T - ma * ma)
    var_alpha = scale * ((ww * a * a).sum() / T - mb * mb)
    cov = scale * ((ww * psi * a).sum() / T - ma * mb)
    return torch.stack([var_psi, var_alpha, cov])

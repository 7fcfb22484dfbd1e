"""Leaving out a whole worker-firm match (leaveout_match.py:156-214
`leave_out_match`), point estimates, on the device.

From a row-level fit of the user's model: the partialled outcome
y~ = fe_alpha + fe_psi + resid (everything but the worker and firm effects
taken out, leaveout_match.py:76-77), collapsed to one row per match -- a run
of equal (worker, firm) in pass 0's order -- with its weighted mean and total
weight (:63-88); the weighted match-level fit y~ ~ 1 | worker + firm; and the
KSS components of that fit (leaveout.py:634-805) with the match level's
rules: sigma2 centred as the reference does at match level, (sqrt(w) ybar -
its mean over matches) sqrt(w) e / M times the JLA factor (:949-1016); the
stayers' matches, whose leverage is one, given `sigma_for_stayers`
(leaveout_match.py:91-132) from their person-year rows; the moments divided
by person-years - 1 (leaveout_se.py:216-220).  Everything runs on the device
(the collapse and the stayer sums as tensor segment sums; the fits, leverages
and trace through the library's kernels).

With `se`, the standard errors of var(psi) and cov(psi, alpha)
(leaveout.py:760-772, :848-894 `_match_se_sigma2`): each match's variance
is, by `se_variance`, "person_year" -- the within-match variance
(leaveout_match.py:135-153) plus, for movers, the weighted-centred
leave-match-out sigma2 over T -- or "match" -- that sigma2 alone, stayers'
from `sigma_for_stayers`; then `StandardErrors.component_variances` on the
match rows with the stayers' b zeroed, the reference-centred kernel, the
person-year divisor and seed + 5_500_011.
"""

from __future__ import annotations

import numpy as np

from . import fit as _fit
from .leaveout import (COMPONENTS, MAX_BLOCK, SE_SEED_OFFSET, TRACE_SEED_OFFSET,
                       InverseOperator, LeaveOutComponents)
from .leaveout_se import ComponentSE, StandardErrors


def _torch():
    import torch
    return torch


def leave_out_match(rows: _fit.DeviceRows, res: _fit.FitResult, covariates=None,
                    n_draws=250, block=MAX_BLOCK, seed=0, tol=1e-10, se=False,
                    se_variance="person_year", se_draws=None, se_trace=True, smooth_bins=None):
    """The match-level KSS components for a row-level fit `res` of `rows`
    (pass 0's layout; psi = the first non-streamed dimension; covariates
    (N, c) the model's, or None), as the reference's `leave_out_match`
    returns them: a `LeaveOutComponents` (plug_in, bias, leave_out keyed by
    component; n_obs the person-years, n_movers the movers' matches;
    leverages and trace of the match-level fit; se a `ComponentSE` with
    var(alpha) NaN when `se`; fit = `res`, match_fit the match-level
    `FitResult`), its diagnostics holding "sigma2" (per match),
    "n_matches", "stayer_matches", "person_years", "max_leverage" (movers'
    matches) and, with `se`, "sigma2_se"."""
    if se_variance not in ("match", "person_year"):
        raise ValueError("se_variance must be 'match' or 'person_year'")
    if se and se_variance == "person_year" and rows.w is not None:
        # leaveout_match.py:168-171
        raise ValueError("se_variance='person_year' is LeaveOutTwoWay's, which has no user "
                         "weights; use se_variance='match' with a weighted fit")
    torch = _torch()
    dev = rows.gcode.device
    f64 = dict(dtype=torch.float64, device=dev)
    N = rows.n_rows
    op = InverseOperator(rows, res.cells, res.S, covariates, tol=tol)
    A = op.residual_moments(res.gamma).cpu().numpy()
    beta = np.linalg.solve(A[1:, 1:], A[1:, 0]) if A.shape[0] > 1 else np.zeros(0)
    e, alpha_g, gam_y, _ = op.row_effects(res.gamma, beta)
    sizes = op.starts[1:] - op.starts[:-1]
    psi_row = gam_y[rows.codes[:, 0].to(torch.int64)]
    y_t = torch.repeat_interleave(alpha_g, sizes) + psi_row + e
    w = rows.w if rows.w is not None else torch.ones(N, **f64)
    # the matches: runs of equal (worker, firm)
    g = rows.gcode.to(torch.int64)
    f = rows.codes[:, 0].to(torch.int64)
    head = torch.ones(N, dtype=torch.bool, device=dev)
    head[1:] = (g[1:] != g[:-1]) | (f[1:] != f[:-1])
    match = torch.cumsum(head.to(torch.int64), 0) - 1
    n_m = int(match[-1].item()) + 1
    W_m = torch.zeros(n_m, **f64).index_add_(0, match, w)
    Y_m = torch.zeros(n_m, **f64).index_add_(0, match, w * y_t) / W_m
    first = torch.nonzero(head).flatten()
    mrows = _fit.DeviceRows(rows.gcode[first].contiguous(),
                            rows.codes[first][:, :1].contiguous(), Y_m[None, :].contiguous(),
                            W_m.contiguous(), [int(rows.n_levels[0])])
    mres = _fit.fit(mrows, tol=tol)
    mop = InverseOperator(mrows, mres.cells, mres.S, None, tol=tol)
    e_m, _, _, sums = mop.row_effects(mres.gamma, np.zeros(0))
    s = sums.cpu().numpy()
    T, R = s[0], float(N)
    scale = T / (T * (R - 1.0) / R) if R > 1 else 1.0
    ma, mb = s[2] / T, s[3] / T
    plug_in = np.array([scale * (s[4] / T - ma * ma), scale * (s[5] / T - mb * mb),
                        scale * (s[6] / T - ma * mb)])
    jla = mop.jla_leverages(n_draws, block, seed)
    lev, comp, factor = jla.leverage, jla.complement, jla.factor
    root = torch.sqrt(W_m)
    yt = root * Y_m
    sigma2 = (yt - yt.mean()) * root * e_m / comp * factor
    # the stayers' matches: sigma_for_stayers on their person-year rows
    gm = mrows.gcode.to(torch.int64)
    per_worker = torch.bincount(gm)
    stayer = per_worker[gm] == 1
    fitted = Y_m - e_m
    worker_w = torch.zeros(int(g.max().item()) + 1, **f64).index_add_(0, g, w)
    y_mean = (w * y_t).sum() / w.sum()
    r = (y_t - y_mean) * (y_t - fitted[match]) / (1.0 - w / worker_w[g])
    stay = torch.zeros(n_m, **f64).index_add_(0, match, w * w * r) / W_m
    sigma2 = torch.where(stayer, stay, sigma2).contiguous()
    trace = mop.hutchinson_trace(sigma2, n_draws, block, seed + TRACE_SEED_OFFSET,
                                 person_years=R)
    bias = trace.as_array()
    movers = ~stayer
    diag = {"sigma2": sigma2, "n_matches": n_m, "stayer_matches": int(stayer.sum().item()),
            "person_years": N, "leave_out": "match", "stayers": "within_match",
            "centering": "reference", "psi": mop.o_fe[0], "alpha": mop.g_fe,
            "max_leverage": float(lev[movers].max().item()) if bool(movers.any()) else 0.0,
            "sigma2_mean": float((sigma2 / W_m).mean().item())}
    out = LeaveOutComponents(
        plug_in=dict(zip(COMPONENTS, plug_in.tolist())), bias=trace.as_dict(),
        leave_out=dict(zip(COMPONENTS, (plug_in - bias).tolist())), n_obs=N,
        n_movers=int(movers.sum().item()), leverages=jla, trace=trace, diagnostics=diag,
        fit=res, match_fit=mres)
    if not se:
        return out
    # the movers' weighted-centred leave-match-out sigma2 (leaveout.py:949-1016)
    y_bar = (W_m @ Y_m) / W_m.sum()
    block_s2 = W_m * (Y_m - y_bar) * e_m / comp * factor
    if se_variance == "match":
        sigma2_se = torch.where(stayer, stay, block_s2)
    else:
        # leaveout_match.py:135-153: the mean over the match of (y~ - its mean)^2
        dev2 = (y_t - Y_m[match]) ** 2
        within = torch.zeros(n_m, **f64).index_add_(0, match, dev2) / \
            torch.bincount(match, minlength=n_m).to(torch.float64)
        sigma2_se = torch.where(stayer, within, within + block_s2 / W_m)
    sigma2_se = sigma2_se.contiguous()
    ses = StandardErrors(mop, 0, person_years=N)
    draws = n_draws if se_draws is None else int(se_draws)
    raw = ses.component_variances(sigma2_se, lev, comp, factor, None, draws, block,
                                  seed + SE_SEED_OFFSET, se_trace, smooth_bins,
                                  stayer_rows=stayer, centering="reference", reported=(0, 2))
    out.se = ComponentSE.from_dict(raw, trace=se_trace)
    diag["sigma2_se"] = sigma2_se
    return out

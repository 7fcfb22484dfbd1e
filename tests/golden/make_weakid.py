"""Golden vectors for the weak-identification diagnostic, made by the
reference itself.

Run once, in a container where the reference tree is readable:

    python tests/golden/make_weakid.py /path/to/hdfe-stream

On the akm_small golden panel and on a low-mobility panel (few movers, so
that one eigen-direction dominates), each restricted to its leave-one-out
connected set by the reference's core/connected.py:503-557 `_leave_one_out`,
it runs leaveout_weakid.py:565-713 `weak_id_diagnostics` (Lanczos on Q S^-,
the deflated Hutchinson sum of squared eigenvalues, q, the first-stage F)
with the reference's own JLA leverages and a seeded sigma2, without
covariates.  On the low-mobility panel it also runs `component_variances`
with the diagnostic (:737-759, `_weak_moments` :786-888: b1, its raw
variance and the 2x2 covariance of (b1, theta1) for the flagged
components) and am_interval.py `am_interval` (the q = 1 interval of KSS
Section 6) on them, and the interval alone on fixed inputs.  Inputs and
outputs go to tests/golden/weakid.npz.  Nothing at
test time reads the reference.
"""

from __future__ import annotations

import importlib
import sys
import tempfile
from pathlib import Path
from types import SimpleNamespace

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parents[1]))
sys.path.insert(0, str(HERE))

from hdfe_stream_b200.simulate import pass0_layout, simulate_panel  # noqa: E402
from make_golden import GOLDEN, import_reference, make_estimator  # noqa: E402
from make_se import loo_keep  # noqa: E402

PANELS = {
    "akm_small": GOLDEN["akm_small"][0],
    "low_mobility": dict(n_workers=3_000, n_firms=60, n_years=8, spell=(3, 8), p_move=0.02,
                         seed=505),
}


def weak_pieces(est, rows, lev, sigma2, weak_id, keys, out, name):
    """leaveout_se.py:599-784 `component_variances` with the diagnostic, so
    that `_weak_moments` (:786-888) runs for the flagged components, and
    am_interval.py `am_interval` on its output for a fixed leave-out value."""
    am = importlib.import_module("hdfe_stream.am_interval")
    b_ii = est.bii_rows(n_draws=16, block=8, seed=6, covariates=(), in_memory=True)
    res = est.component_variances(SimpleNamespace(depvar="log_earn"), sigma2, lev, b_ii=b_ii,
                                  n_draws=16, block=8, seed=6, covariates=(), in_memory=True,
                                  weak_id=weak_id)
    out[f"{name}_bii"] = np.stack([np.array(b_ii[k]) for k in keys])
    out[f"{name}_complement"] = np.array(lev.complement)
    out[f"{name}_factor"] = np.array(lev.factor)
    for field in ("variance", "first_term", "trace_term", "theta"):
        out[f"{name}_se_{field}"] = np.array([getattr(res, field)[k] for k in keys])
    flagged = [k for k in range(3) if keys[k] in (res.weak or {})]
    out[f"{name}_weak_components"] = np.array(flagged)
    leave_out = np.array([0.03, 0.2, -0.01])
    out[f"{name}_weak_leave_out"] = leave_out
    for k in flagged:
        piece = res.weak[keys[k]]
        for field in ("lambda_1", "b1", "v_raw", "trace", "quadratic"):
            out[f"{name}_weak{k}_{field}"] = np.array([piece[field]])
        out[f"{name}_weak{k}_sigma"] = np.asarray(piece["sigma"])
        out[f"{name}_weak{k}_conservative"] = np.array([piece["conservative"]])
        theta1 = leave_out[k] - piece["lambda_1"] * (piece["b1"] ** 2 - piece["v_raw"])
        lo, hi, info = am.am_interval(piece["lambda_1"], piece["b1"], theta1, piece["sigma"],
                                      0.05)
        out[f"{name}_weak{k}_interval"] = np.array([lo, hi, info["kappa"], info["z"],
                                                     info["rho"]])
        print("  weak", keys[k], piece, (lo, hi, info))
    # the interval alone on fixed inputs, across curvatures
    cases = [(0.5, 0.3, 0.1, [[0.01, 0.002], [0.002, 0.004]], 0.05),
             (2.0, -0.1, 0.05, [[0.02, -0.001], [-0.001, 0.001]], 0.05),
             (0.01, 0.2, 0.3, [[0.001, 0.0], [0.0, 0.003]], 0.1),
             (-1.0, 0.05, 0.2, [[0.05, 0.01], [0.01, 0.02]], 0.05)]
    res_am = []
    for lam, b1, th, sig, alpha in cases:
        lo, hi, info = am.am_interval(lam, b1, th, np.array(sig), alpha)
        res_am.append([lam, b1, th, sig[0][0], sig[0][1], sig[1][1], alpha, lo, hi,
                       info["kappa"], info["z"]])
    out["am_cases"] = np.array(res_am)


def main(root):
    mods = import_reference(root)
    se = importlib.import_module("hdfe_stream.leaveout_se")
    wk = importlib.import_module("hdfe_stream.leaveout_weakid")
    out = {}
    for name, kw in PANELS.items():
        panel = simulate_panel(**kw)
        rows = pass0_layout(panel, loo_keep(mods, panel))
        with tempfile.TemporaryDirectory() as tmp:
            est = make_estimator(mods, rows, Path(tmp))
            est.__class__ = type("EstWeak", (type(est), se._StandardErrorMixin,
                                             wk._WeakIdMixin), {})
            est.vidx = {n: j for j, n in enumerate(rows.names)}
            est._pass1_cells()
            est._components()
            est._solve(in_memory=True)
            lev = est.jla_leverages(n_draws=24, block=8, seed=2, in_memory=True, covariates=())
            sigma2 = np.random.default_rng(51).standard_normal(rows.n_rows) * 0.3 + 0.25
            res = est.weak_id_diagnostics(SimpleNamespace(depvar="log_earn"), sigma2, lev,
                                          n_draws=48, block=12, seed=9, covariates=(),
                                          warn=False)
            keys = list(se.COMPONENTS)
            out[f"{name}_gcode"] = rows.gcode
            out[f"{name}_codes_rows"] = rows.codes
            out[f"{name}_V"] = rows.V
            out[f"{name}_w"] = np.zeros(0)
            out[f"{name}_n_levels"] = np.array(rows.n_levels, np.int64)
            out[f"{name}_n_groups"] = np.array([rows.n_groups])
            out[f"{name}_tol"] = np.array([est.tol])
            out[f"{name}_sigma2"] = sigma2
            out[f"{name}_leverage"] = np.array(lev.leverage)
            for k, key in enumerate(keys):
                out[f"{name}_eig{k}"] = np.array(res.eigenvalues[key])
                out[f"{name}_ratio{k}"] = np.array(res.ratios[key])
            out[f"{name}_sum_sq"] = np.array([res.sum_sq[k] for k in keys])
            out[f"{name}_sum_sq_se"] = np.array([res.sum_sq_se[k] for k in keys])
            out[f"{name}_q"] = np.array([res.q[k] for k in keys])
            out[f"{name}_f_stat"] = np.array([res.f_stat[k] for k in keys])
            out[f"{name}_steps"] = np.array([res.diagnostics["lanczos_steps"]])
            out[f"{name}_lengths"] = np.array(res.diagnostics["lanczos_lengths"])
            out[f"{name}_n_draws"] = np.array([res.diagnostics["n_draws"]])
            out[f"{name}_deflated"] = np.array([res.diagnostics["deflated"]])
            print(name, rows.n_rows, res.summary() if hasattr(res, "summary") else res)
            print("  ", res.diagnostics)
            if name == "low_mobility":
                weak_pieces(est, rows, lev, sigma2, res, keys, out, name)
    np.savez_compressed(HERE / "weakid.npz", **out)


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else "/root/reference")

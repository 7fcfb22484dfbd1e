"""Golden vectors for the KSS standard errors, made by the reference itself.

Run once, in a container where the reference tree is readable:

    python tests/golden/make_se.py /path/to/hdfe-stream

On two of the golden panels restricted to their leave-one-out connected set
(the reference's core/connected.py:503-557 `_leave_one_out`, as
`leave_out_kss` applies it; tests/golden/make_golden.py builds the
estimator) it runs leaveout_se.py's `_StandardErrorMixin`: `bii_rows`
(:228-327, the per-row B_ii of var(psi), var(alpha), cov by random
projection) and `component_variances` (:599-784: b = B_ii / M_ii with the
leverage correction, the sigma2 smoother, C y exactly, the trace term by
Hutchinson draws, V = first - 2 trace), without covariates, weighted
centring, for seeded sigma2 and the reference's own JLA leverages.  Inputs
and outputs go to tests/golden/se.npz.  Nothing at test time reads the
reference.
"""

from __future__ import annotations

import sys
import tempfile
from pathlib import Path
from types import SimpleNamespace

import numpy as np

REPO = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(REPO))
sys.path.insert(0, str(Path(__file__).resolve().parent))

from hdfe_stream_b200.simulate import _rank_codes, pass0_layout, simulate_panel  # noqa: E402
from make_golden import GOLDEN, import_reference, make_estimator  # noqa: E402

PANELS = ("akm_small", "akm_weighted")


def loo_keep(mods, panel):
    """Rows of the panel's leave-one-out connected set, by the reference."""
    cn = mods["core.connected"]
    a, _ = _rank_codes(panel.worker)
    b, flev = _rank_codes(panel.firm)
    n0, n1 = int(a.max()) + 1, len(flev)
    key = a.astype(np.uint64) * np.uint64(n1) + b.astype(np.uint64)
    keys, counts = np.unique(key, return_counts=True)
    alive = np.ones(n0 + n1, bool)
    cn._leave_one_out(keys, counts.astype(np.uint32), np.uint64(n1), n0, n1, alive, None)
    return alive[a] & alive[n0 + b.astype(np.int64)]


def main(root):
    mods = import_reference(root)
    import importlib
    se = importlib.import_module("hdfe_stream.leaveout_se")
    out = {}
    for name in PANELS:
        kw, _ = GOLDEN[name]
        panel = simulate_panel(**kw)
        rows = pass0_layout(panel, loo_keep(mods, panel))
        with tempfile.TemporaryDirectory() as tmp:
            est = make_estimator(mods, rows, Path(tmp))
            est.__class__ = type("EstSE", (type(est), se._StandardErrorMixin), {})
            est.vidx = {n: j for j, n in enumerate(rows.names)}
            est._pass1_cells()
            est._components()
            est._solve(in_memory=True)
            lev = est.jla_leverages(n_draws=24, block=8, seed=2, in_memory=True,
                                    covariates=())
            sigma2 = np.random.default_rng(31).standard_normal(rows.n_rows) * 0.3 + 0.25
            b_ii = est.bii_rows(n_draws=16, block=8, seed=6, covariates=(), in_memory=True)
            res = est.component_variances(SimpleNamespace(depvar="log_earn"), sigma2, lev,
                                          b_ii=b_ii, n_draws=16, block=8, seed=6,
                                          covariates=(), in_memory=True)
            keys = list(se.COMPONENTS)
            out[f"{name}_gcode"] = rows.gcode
            out[f"{name}_codes_rows"] = rows.codes
            out[f"{name}_V"] = rows.V
            out[f"{name}_w"] = rows.w if rows.w is not None else np.zeros(0)
            out[f"{name}_n_levels"] = np.array(rows.n_levels, np.int64)
            out[f"{name}_n_groups"] = np.array([rows.n_groups])
            out[f"{name}_tol"] = np.array([est.tol])
            out[f"{name}_sigma2"] = sigma2
            out[f"{name}_leverage"] = np.array(lev.leverage)
            out[f"{name}_complement"] = np.array(lev.complement)
            out[f"{name}_factor"] = np.array(lev.factor)
            out[f"{name}_bii"] = np.stack([np.array(b_ii[k]) for k in keys])
            for field in ("variance", "first_term", "trace_term", "theta"):
                out[f"{name}_{field}"] = np.array([getattr(res, field)[k] for k in keys])
            print(name, {f: getattr(res, f) for f in ("variance", "first_term", "trace_term",
                                                      "theta")})
    np.savez_compressed(Path(__file__).resolve().parent / "se.npz", **out)


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else "/root/reference")

"""Exact match-level KSS standard errors for the panel of exact.npz, by the
reference's dense prototype (prototypes/kss_exact.py:636-716
`kss_match_se`, centering "reference"), and the reference's own
`component_variances` with the match level's options on a row-level panel.

Run once, in a container where the reference tree is readable, after
make_exact.py:

    python tests/golden/make_match_se.py /path/to/hdfe-stream

Two sets of vectors go to tests/golden/match_se.npz:

* `exact_*`: theta, V, the first term and the trace term of var(psi) and
  cov(psi, alpha) for both per-match variances ("person_year", the
  reference implementation's, and "match"), on the rows stored in
  exact.npz; the dense prototype uses exact leverages and B_ii.
* `ref_*`: leaveout_se.py:599-784 `component_variances` with
  `stayer_rows`, `centering="reference"` (the rank-two term through
  `_m_times`, :387-424) and `reported=(0, 2)` on the akm_small panel's
  leave-one-out set, with the reference's own JLA leverages and B_ii, seeded
  sigma2 and a seeded stayer mask, so the match level's algebra is pinned to
  the streaming code draw for draw.

Nothing at test time reads the reference.
"""

from __future__ import annotations

import importlib.util
import sys
import tempfile
from pathlib import Path
from types import SimpleNamespace

import numpy as np

HERE = Path(__file__).resolve().parent
REPO = HERE.parents[1]
sys.path.insert(0, str(REPO))
sys.path.insert(0, str(HERE))

from hdfe_stream_b200.simulate import pass0_layout, simulate_panel  # noqa: E402
from make_golden import GOLDEN, import_reference, make_estimator  # noqa: E402
from make_se import loo_keep  # noqa: E402


def exact_part(root, out):
    import_reference(root)          # the package's modules, for the shared smoother
    spec = importlib.util.spec_from_file_location("kss_exact",
                                                  Path(root) / "prototypes" / "kss_exact.py")
    ke = importlib.util.module_from_spec(spec)
    sys.modules["kss_exact"] = ke
    spec.loader.exec_module(ke)
    g = np.load(HERE / "exact.npz")
    kp = ke.Panel(worker=g["gcode"].astype(np.int64), firm=g["codes_rows"][:, 0].astype(np.int64),
                  y=g["V"][:, 0].copy())
    names = ("var(psi)", "cov(psi, alpha)")
    for rule in ("person_year", "match"):
        res = ke.kss_match_se(kp, centering="reference", se_variance=rule)
        for field in ("theta", "V", "first", "trace"):
            out[f"exact_{rule}_{field}"] = np.array([res[n][field] for n in names])
        print(rule, {n: {f: res[n][f] for f in ("theta", "V", "first", "trace")}
                     for n in names})


def reference_part(root, out):
    mods = import_reference(root)
    se = importlib.import_module("hdfe_stream.leaveout_se")
    kw, _ = GOLDEN["akm_small"]
    panel = simulate_panel(**kw)
    rows = pass0_layout(panel, loo_keep(mods, panel))
    with tempfile.TemporaryDirectory() as tmp:
        est = make_estimator(mods, rows, Path(tmp))
        est.__class__ = type("EstSE", (type(est), se._StandardErrorMixin), {})
        est.vidx = {n: j for j, n in enumerate(rows.names)}
        est._pass1_cells()
        est._components()
        est._solve(in_memory=True)
        lev = est.jla_leverages(n_draws=24, block=8, seed=2, in_memory=True, covariates=())
        sigma2 = np.random.default_rng(41).standard_normal(rows.n_rows) * 0.3 + 0.25
        stayer = np.random.default_rng(43).random(rows.n_rows) < 0.2
        b_ii = est.bii_rows(n_draws=16, block=8, seed=6, covariates=(), in_memory=True)
        res = est.component_variances(SimpleNamespace(depvar="log_earn"), sigma2, lev,
                                      b_ii=b_ii, n_draws=16, block=8, seed=6, covariates=(),
                                      in_memory=True, stayer_rows=stayer,
                                      centering="reference", reported=(0, 2))
        keys = list(se.COMPONENTS)
        out["ref_gcode"] = rows.gcode
        out["ref_codes_rows"] = rows.codes
        out["ref_V"] = rows.V
        out["ref_n_levels"] = np.array(rows.n_levels, np.int64)
        out["ref_n_groups"] = np.array([rows.n_groups])
        out["ref_tol"] = np.array([est.tol])
        out["ref_sigma2"] = sigma2
        out["ref_stayer"] = stayer
        out["ref_leverage"] = np.array(lev.leverage)
        out["ref_complement"] = np.array(lev.complement)
        out["ref_factor"] = np.array(lev.factor)
        out["ref_bii"] = np.stack([np.array(b_ii[k]) for k in keys])
        for field in ("variance", "first_term", "trace_term", "theta"):
            out[f"ref_{field}"] = np.array([getattr(res, field)[k] for k in keys])
        print("reference", {f: getattr(res, f) for f in ("variance", "first_term",
                                                         "trace_term", "theta")})


def main(root):
    out = {}
    exact_part(root, out)
    reference_part(root, out)
    np.savez_compressed(HERE / "match_se.npz", **out)


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else "/root/reference")

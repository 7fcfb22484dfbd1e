"""The weak-identification diagnostic on the device (leaveout_weakid.py
`weak_id_diagnostics`) against the reference's own outputs
(tests/golden/weakid.npz, made by tests/golden/make_weakid.py) and the
oracle."""

import numpy as np
import pytest

import oracle as orc
from conftest import load_golden

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def device():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch.device("cuda", 0)


def rel(a, b):
    a, b = np.asarray(a, float), np.asarray(b, float)
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def golden_se(g, name):
    from hdfe_stream_b200 import fit, leaveout, leaveout_se
    from hdfe_stream_b200.simulate import Rows
    rows = Rows(gcode=g[f"{name}_gcode"], codes=g[f"{name}_codes_rows"], V=g[f"{name}_V"],
                w=None, n_levels=[int(x) for x in g[f"{name}_n_levels"]],
                n_groups=int(g[f"{name}_n_groups"][0]),
                names=["log_earn", "age_squared", "age_cubed"])
    drows = fit.DeviceRows.from_rows(rows)
    cells = fit.pass1(drows)
    op = leaveout.InverseOperator(drows, cells, fit.build_s(cells), None,
                                  tol=float(g[f"{name}_tol"][0]))
    return rows, leaveout_se.StandardErrors(op)


@pytest.mark.parametrize("name", ["akm_small", "low_mobility"])
def test_weak_id_diagnostics_match_reference(device, name):
    """Eigenvalues, ratios, sum lambda^2, q and the first-stage F against the
    reference on a well-connected (q = 0) and a low-mobility (q = 1) panel.
    The recurrence runs on the device's solves, whose rounding differs from
    the reference's, so the converged eigenvalues are compared to 1e-7 and
    the Monte Carlo parts to 1e-6."""
    from hdfe_stream_b200.weakid import weak_id_diagnostics
    g = load_golden("weakid")
    _, se = golden_se(g, name)
    out = weak_id_diagnostics(se, g[f"{name}_sigma2"], g[f"{name}_leverage"], n_draws=48,
                              block=12, seed=9)
    for k in range(3):
        assert rel(out["eigenvalues"][k], g[f"{name}_eig{k}"]) < 1e-7
        assert rel(out["ratios"][k], g[f"{name}_ratio{k}"]) < 1e-6
    assert rel(out["sum_sq"], g[f"{name}_sum_sq"]) < 1e-6
    assert list(out["q"]) == list(g[f"{name}_q"])
    assert rel(out["f_stat"], g[f"{name}_f_stat"]) < 1e-6
    assert out["n_draws"] == int(g[f"{name}_n_draws"][0])


def test_weak_id_on_a_weighted_panel_matches_oracle(device):
    """A weighted panel (the square-root-weight metric in the draws, the
    readout and the F statistic) against the oracle with the same draws."""
    from hdfe_stream_b200 import fit, leaveout, leaveout_se
    from hdfe_stream_b200.simulate import pass0_layout, simulate_panel, _rank_codes
    from hdfe_stream_b200.weakid import weak_id_diagnostics
    panel = simulate_panel(2_000, 80, 8, spell=(2, 8), p_move=0.05, weights=True, seed=61)
    a, _ = _rank_codes(panel.worker)
    b, flev = _rank_codes(panel.firm)
    n0, n1 = int(a.max()) + 1, len(flev)
    order = np.lexsort((b, a))
    alive, _, _ = orc.leave_one_out(a[order], b[order], n0, n1)
    rows = pass0_layout(panel, alive[a] & alive[n0 + b.astype(np.int64)])
    c = orc.pass1(rows)
    des = orc.Design(rows, c, orc.build_explicit(c), tol=1e-12)
    rng = np.random.default_rng(5)
    sigma2 = rng.standard_normal(rows.n_rows) * 0.2 + 0.3
    lev = rng.uniform(0.05, 0.9, rows.n_rows)
    ref = orc.weak_id_diagnostics(des, sigma2, lev, n_draws=32, block=12, seed=4)
    drows = fit.DeviceRows.from_rows(rows)
    cells = fit.pass1(drows)
    op = leaveout.InverseOperator(drows, cells, fit.build_s(cells), None, tol=1e-12)
    out = weak_id_diagnostics(leaveout_se.StandardErrors(op), sigma2, lev, n_draws=32, block=12,
                              seed=4)
    for k in range(3):
        assert rel(out["eigenvalues"][k], ref["eigenvalues"][k]) < 1e-7
    assert rel(out["sum_sq"], ref["sum_sq"]) < 1e-6
    assert list(out["q"]) == list(ref["q"])
    assert rel(out["f_stat"], ref["f_stat"]) < 1e-6


def test_weak_moments_and_interval_match_reference(device):
    """The q = 1 pieces on the device (`component_variances` with the
    diagnostic: b1, its raw variance, the 2x2 covariance of (b1, theta1)
    from the deflated kernel C2) and the interval formed from them against
    the reference on the low-mobility panel, where all three components are
    flagged."""
    from hdfe_stream_b200.leaveout_se import COMPONENTS, weak_intervals
    from hdfe_stream_b200.weakid import weak_id_diagnostics
    g = load_golden("weakid")
    name = "low_mobility"
    _, se = golden_se(g, name)
    wid = weak_id_diagnostics(se, g[f"{name}_sigma2"], g[f"{name}_leverage"], n_draws=48,
                              block=12, seed=9)
    out = se.component_variances(g[f"{name}_sigma2"], g[f"{name}_leverage"],
                                 g[f"{name}_complement"], g[f"{name}_factor"], None, n_draws=16,
                                 block=8, seed=6, weak_id=wid)
    for f in ("variance", "first_term", "trace_term", "theta"):
        assert rel([out[f][n] for n in COMPONENTS], g[f"{name}_se_{f}"]) < 1e-7, f
    flagged = [int(k) for k in g[f"{name}_weak_components"]]
    assert sorted(COMPONENTS.index(n) for n in out["weak"]) == flagged
    leave_out = g[f"{name}_weak_leave_out"]
    weak = weak_intervals(leave_out, out["weak"], 0.95)
    for k in flagged:
        piece = weak[COMPONENTS[k]]
        for f in ("lambda_1", "b1", "v_raw", "trace", "quadratic"):
            assert rel(piece[f], g[f"{name}_weak{k}_{f}"]) < 1e-6, f
        assert rel(piece["sigma"], g[f"{name}_weak{k}_sigma"]) < 1e-6
        want = g[f"{name}_weak{k}_interval"]
        assert rel([*piece["interval"], piece["kappa"], piece["z"]], want[:4]) < 1e-6


def test_weak_id_against_exact_prototype(device):
    """The device's Lanczos eigenvalues of S^- Q against the reference's dense
    exact prototype (prototypes/kss_exact.py `weak_id`, tests/golden/
    exact_se.npz) to 1e-6, with q equal and sum lambda^2 within 10% at 64
    draws."""
    from hdfe_stream_b200 import fit, leaveout, leaveout_se
    from hdfe_stream_b200.simulate import Rows
    from hdfe_stream_b200.weakid import weak_id_diagnostics
    g, ge = load_golden("exact"), load_golden("exact_se")
    rows = Rows(gcode=g["gcode"], codes=g["codes_rows"], V=g["V"][:, :1], w=None,
                n_levels=[int(x) for x in g["n_levels"]], n_groups=int(g["n_groups"][0]),
                names=["log_earn"])
    drows = fit.DeviceRows.from_rows(rows)
    res = fit.fit(drows, tol=1e-12)
    op = leaveout.InverseOperator(drows, res.cells, res.S, None, tol=1e-12)
    kss = op.leave_out_components(res, 256, block=32, seed=3)
    out = weak_id_diagnostics(leaveout_se.StandardErrors(op), kss.diagnostics["sigma2"],
                              kss.leverages.leverage, n_draws=64, block=32, seed=9)
    for k in range(3):
        assert rel(out["eigenvalues"][k], ge[f"weak_eig{k}"]) < 1e-6
    assert list(out["q"]) == [int(x) for x in ge["weak_q"]]
    assert np.all(np.abs(out["sum_sq"] - ge["weak_sum_sq"]) <= 0.1 * ge["weak_sum_sq"])

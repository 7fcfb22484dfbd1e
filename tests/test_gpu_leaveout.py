"""The inverse operator's row passes and the JLA leverages on the device,
against the reference's own outputs (tests/golden, made by the reference's
project_rows / jla_leverages) and against the oracle with covariates."""

import numpy as np
import pytest

import oracle as orc
from conftest import golden_rows, load_golden, GOLDEN_PANELS

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


COMPONENTS = ("var(psi)", "var(alpha)", "cov(psi, alpha)")


def vals(d):
    """A component dict as an array in the reference's key order."""
    return np.array([d[k] for k in COMPONENTS])


def operator(rows, tol, covariates=False, precision="fp64"):
    from hdfe_stream_b200 import fit, leaveout
    drows = fit.DeviceRows.from_rows(rows)
    cells = fit.pass1(drows)
    S = fit.build_s(cells)
    X = drows.V[1:].T.contiguous() if covariates else None
    return leaveout.InverseOperator(drows, cells, S, X, tol=tol, precision=precision)


@pytest.mark.parametrize("name", GOLDEN_PANELS)
def test_project_rows_matches_reference(device, name):
    g = load_golden(name)
    rows = golden_rows(g)
    op = operator(rows, float(g["tol"]))
    out, info = op.project(6, seed=11, sqrt_weights=rows.w is not None)
    assert info["converged"]
    assert rel(out.cpu().numpy(), g["project_rows_seed11"]) < 1e-8


@pytest.mark.parametrize("name", GOLDEN_PANELS)
def test_jla_leverages_match_reference(device, name):
    g = load_golden(name)
    rows = golden_rows(g)
    op = operator(rows, float(g["tol"]))
    j = op.jla_leverages(24, block=8, seed=2)
    lev, comp, factor = j.leverage, j.complement, j.factor
    assert j.n_draws == 24 and j.diagnostics["blocks"] == 3 and j.n_rows == rows.n_rows
    assert rel(lev.cpu().numpy(), g["jla_leverage"]) < 1e-8
    assert rel(factor.cpu().numpy(), g["jla_factor"]) < 1e-8
    assert np.allclose(lev.cpu().numpy() + comp.cpu().numpy(), 1.0)


def test_jla_blocking_does_not_change_the_answer(device):
    g = load_golden("akm_small")
    op = operator(golden_rows(g), 1e-12)
    a = op.jla_leverages(24, block=8, seed=2).leverage.cpu().numpy().copy()
    b = op.jla_leverages(24, block=24, seed=2).leverage.cpu().numpy().copy()
    c = op.jla_leverages(24, block=5, seed=2).leverage.cpu().numpy().copy()
    assert rel(a, b) < 1e-9 and rel(a, c) < 1e-9


@pytest.mark.parametrize("name", ["akm_small", "akm_weighted"])
def test_projection_with_covariates_matches_oracle(device, name):
    """The design with the model's covariates (age_squared, age_cubed): the
    Schur border of inverse.py:182-218."""
    g = load_golden(name)
    rows = golden_rows(g)
    c = orc.pass1(rows)
    des = orc.Design(rows, c, orc.build_explicit(c), X=rows.V[:, 1:], tol=1e-12)
    ref = des.project_rows(20, 5, 3, sqrt_weights=rows.w is not None)
    op = operator(rows, 1e-12, covariates=True)
    out, _ = op.project(20, seed=5, first_draw=3, sqrt_weights=rows.w is not None)
    assert rel(out.cpu().numpy(), ref) < 1e-8
    lev_ref, _, f_ref = des.jla_leverages(40, 16, 7)
    j = op.jla_leverages(40, block=32, seed=7)
    lev, f = j.leverage, j.factor
    assert rel(lev.cpu().numpy(), lev_ref) < 1e-8
    assert rel(f.cpu().numpy(), f_ref) < 1e-8


def test_projection_is_idempotent(device):
    """A S^- A' is a projection: applying it to its own output returns it
    (tests/test_inverse.py:128 of the reference checks the same)."""
    import torch
    g = load_golden("akm_components")
    rows = golden_rows(g)
    op = operator(rows, 1e-13)
    out, _ = op.project(4, seed=3)
    again, _ = op.center(4, R=out.contiguous()), None
    rhs, _, sq = again
    U, _ = op.solve_reduced(rhs, torch.sqrt(sq))
    out2 = torch.empty_like(out)
    from hdfe_stream_b200 import _lib
    U, out = U.contiguous(), out.contiguous()
    _lib.check(_lib.lib().hdfe_rows_project(
        op.starts.data_ptr(), op.G, op.rows.codes.data_ptr(), len(op.nlev),
        op.nlev.ctypes.data, None, None, 0, None, U.data_ptr(), out.data_ptr(), 4, 0, 0, 0, 0,
        op.N, out2.data_ptr(), None, _lib.stream_handle()))
    assert rel(out2.cpu().numpy(), out.cpu().numpy()) < 1e-8


@pytest.mark.parametrize("weights", [False, True])
def test_long_groups_and_block_widths(device, weights):
    """Workers with 20-36 rows (many groups longer than one 32-row chunk of
    the row passes), two non-streamed dimensions (300 firms: level sums in
    global memory for wide blocks, in shared memory for narrow ones),
    covariates, and blocks of 1, 5, 13 and 32 vectors: projections and JLA
    sums against the oracle."""
    from hdfe_stream_b200.simulate import pass0_layout, simulate_panel
    rows = pass0_layout(simulate_panel(600, 300, 40, spell=(20, 36), p_move=0.05,
                                       weights=weights, seed=5))
    c = orc.pass1(rows)
    des = orc.Design(rows, c, orc.build_explicit(c), X=rows.V[:, 1:], tol=1e-12)
    op = operator(rows, 1e-12, covariates=True)
    sw = rows.w is not None
    for B, first in ((1, 0), (5, 2), (13, 7), (32, 40)):
        ref = des.project_rows(B, 9, first, sqrt_weights=sw)
        out, _ = op.project(B, seed=9, first_draw=first, sqrt_weights=sw)
        assert rel(out.cpu().numpy(), ref) < 1e-8, B
    lev_ref, _, f_ref = des.jla_leverages(45, 16, 4)
    j = op.jla_leverages(45, block=32, seed=4)
    lev, f = j.leverage, j.factor
    assert rel(lev.cpu().numpy(), lev_ref) < 1e-8
    assert rel(f.cpu().numpy(), f_ref) < 1e-8


@pytest.mark.parametrize("weights", [False, True])
def test_mixed_precision_leverages_match_oracle(device, weights):
    """The JLA leverages with the block solves in mixed precision (FP32 inner
    CG on 32 columns, FP64 refinement to the same residual tolerance) and
    the Hutchinson bias terms, against the FP64 oracle with the same draws."""
    from hdfe_stream_b200.simulate import pass0_layout, simulate_panel
    rows = pass0_layout(simulate_panel(3_000, 300, 10, spell=(3, 10), p_move=0.15,
                                       weights=weights, seed=23))
    c = orc.pass1(rows)
    des = orc.Design(rows, c, orc.build_explicit(c), X=rows.V[:, 1:], tol=1e-12)
    lev_ref, _, f_ref = des.jla_leverages(64, 32, 5)
    op = operator(rows, 1e-12, covariates=True, precision="mixed")
    j = op.jla_leverages(64, block=32, seed=5)
    assert rel(j.leverage.cpu().numpy(), lev_ref) < 1e-8
    assert rel(j.factor.cpu().numpy(), f_ref) < 1e-8
    sigma2 = np.abs(rows.V[:, 0] - rows.V[:, 0].mean()) * 0.1 + 0.05
    tr_ref = des.hutchinson_trace(sigma2, 32, 32, 7)
    tr = op.hutchinson_trace(sigma2, 32, block=32, seed=7).as_array()
    # two chained refined solves per draw: within the residual tolerance's reach
    assert rel(tr, tr_ref) < 1e-7


@pytest.mark.parametrize("name", GOLDEN_PANELS)
def test_apply_inverse_matches_reference(device, name):
    """S^- v for a coefficient-space v (inverse.py `apply_inverse`): the
    solution, its streamed block and the rows' (A u)_i against the
    reference's outputs, null-space component dropped as there."""
    import torch
    g = load_golden(name)
    rows = golden_rows(g)
    op = operator(rows, float(g["tol"]))
    dev = torch.device("cuda")
    U, C, Ug, R = op.apply_inverse(torch.as_tensor(g["ainv_levels"], device=dev),
                                   torch.zeros((0, 3), dtype=torch.float64, device=dev),
                                   torch.as_tensor(g["ainv_groups"], device=dev), rows=True)
    assert rel(U.cpu().numpy(), g["ainv_U"]) < 1e-8
    assert rel(Ug.cpu().numpy(), g["ainv_Ug"]) < 1e-8
    assert rel(R.cpu().numpy(), g["ainv_rows"]) < 1e-8


@pytest.mark.parametrize("name", GOLDEN_PANELS)
def test_hutchinson_trace_matches_reference(device, name):
    """leaveout.py `hutchinson_trace`: var(psi), var(alpha), cov for 16
    draws in blocks of 8, against the reference's numbers."""
    g = load_golden(name)
    rows = golden_rows(g)
    op = operator(rows, float(g["tol"]))
    tr = op.hutchinson_trace(g["trace_sigma2"], n_draws=16, block=8, seed=4)
    assert tr.n_draws == 16 and tr.diagnostics["blocks"] == 2
    assert rel(tr.as_array(), g["trace"]) < 1e-8
    assert rel(vals(tr.as_dict()), g["trace"]) < 1e-8


def test_hutchinson_blocking_and_covariates(device):
    """With the model's covariates (Schur border) against the oracle, and
    the same answer whatever the blocking."""
    g = load_golden("akm_weighted")
    rows = golden_rows(g)
    c = orc.pass1(rows)
    des = orc.Design(rows, c, orc.build_explicit(c), X=rows.V[:, 1:], tol=1e-12)
    sigma2 = g["trace_sigma2"]
    ref = des.hutchinson_trace(sigma2, 20, 20, 3)
    op = operator(rows, 1e-12, covariates=True)
    a = op.hutchinson_trace(sigma2, n_draws=20, block=20, seed=3).as_array()
    b = op.hutchinson_trace(sigma2, n_draws=20, block=7, seed=3).as_array()
    assert rel(a, ref) < 1e-8
    assert rel(a, b) < 1e-9


@pytest.mark.parametrize("name", GOLDEN_PANELS)
def test_steps_3_4_match_reference(device, name):
    """V' W V of the residualised variables, beta and the pass-2 residuals
    and effects on the reference's own Gamma, against the reference's
    `_nb_residualize_rows` / `_assemble` / `_nb_pass2` outputs."""
    import torch
    g = load_golden(name)
    a = load_golden("assemble")
    rows = golden_rows(g)
    op = operator(rows, float(g["tol"]))
    gamma = torch.as_tensor(g["gamma"], device=device)
    A = op.residual_moments(gamma).cpu().numpy()
    assert rel(A, a[f"{name}_A"]) < 1e-11
    assert np.array_equal(A, op.residual_moments(gamma).cpu().numpy())
    beta = np.linalg.solve(A[1:, 1:], A[1:, 0])
    assert rel(beta, a[f"{name}_beta"]) < 1e-9
    e, alpha, gam_y, sums = op.row_effects(gamma, beta)
    assert rel(e.cpu().numpy(), a[f"{name}_resid"]) < 1e-9
    assert rel(alpha.cpu().numpy(), a[f"{name}_alpha"]) < 1e-9
    psi = gam_y.cpu().numpy()[rows.codes[:, 0].astype(np.int64)]
    assert rel(psi, a[f"{name}_psi"]) < 1e-9
    w = rows.w if rows.w is not None else np.ones(rows.n_rows)
    s = sums.cpu().numpy()
    assert rel(s[:2], [w.sum(), w @ rows.V[:, 0]]) < 1e-12
    assert rel(s[4], w @ (psi * psi)) < 1e-10


def without_singletons(rows):
    """The rows of groups seen at least twice: a single-row group has
    leverage 1 and no leave-one-out residual (the reference asks for the
    leave-one-out connected set before the KSS components)."""
    from hdfe_stream_b200.simulate import Rows
    sizes = np.bincount(rows.gcode)
    keep = sizes[rows.gcode] >= 2
    number = np.cumsum(sizes >= 2) - 1
    return Rows(gcode=number[rows.gcode[keep]].astype(rows.gcode.dtype), codes=rows.codes[keep],
                V=rows.V[keep], w=None if rows.w is None else rows.w[keep],
                n_levels=rows.n_levels, n_groups=int((sizes >= 2).sum()), names=rows.names)


@pytest.mark.parametrize("name", ["akm_small", "akm_weighted"])
def test_leave_out_components_match_oracle(device, name):
    """leaveout.py `leave_out_components` (plug-in, sigma2, bias, leave-out)
    with the model's covariates, against the oracle on the same Gamma.  (The
    many-component panel has rows of leverage 1 -- its small components --
    whose sigma2 is not defined.)"""
    import torch
    rows = without_singletons(golden_rows(load_golden(name)))
    c = orc.pass1(rows)
    S = orc.build_explicit(c)
    gamma, _ = orc.solve(c, S, tol=1e-12)
    des = orc.Design(rows, c, S, X=rows.V[:, 1:], tol=1e-12)
    ref = des.leave_out_components(gamma, 16, 8, 5)
    assert np.all(np.isfinite(ref["sigma2"]))
    op = operator(rows, 1e-12, covariates=True)
    from hdfe_stream_b200.leaveout import JLALeverages, LeaveOutComponents, TraceEstimate
    got = op.leave_out_components(torch.as_tensor(gamma, device=device), 16, 8, 5)
    assert isinstance(got, LeaveOutComponents)
    assert isinstance(got.leverages, JLALeverages) and isinstance(got.trace, TraceEstimate)
    assert list(got.plug_in) == list(got.bias) == list(got.leave_out) == list(COMPONENTS)
    assert got.n_obs == rows.n_rows and got.leverages.n_draws == 16 and got.trace.n_draws == 16
    d = got.diagnostics
    assert rel(d["beta"], ref["beta"]) < 1e-10
    assert rel(vals(got.plug_in), ref["plug_in"]) < 1e-10
    assert rel(d["sigma2"].cpu().numpy(), ref["sigma2"]) < 1e-8
    assert rel(vals(got.bias), ref["bias"]) < 1e-8
    assert rel(vals(got.leave_out), ref["leave_out"]) < 1e-8
    assert rel(got.leverages.leverage.cpu().numpy(), ref["leverage"]) < 1e-8
    assert rel(got.leverages.factor.cpu().numpy(), ref["factor"]) < 1e-8
    assert abs(d["max_leverage"] - ref["max_leverage"]) < 1e-8
    # movers: rows of workers seen at more than one firm
    firm = rows.codes[:, 0]
    lo = np.full(rows.n_groups, np.iinfo(np.int64).max)
    hi = np.full(rows.n_groups, -1)
    np.minimum.at(lo, rows.gcode, firm)
    np.maximum.at(hi, rows.gcode, firm)
    assert got.n_movers == int((lo != hi)[rows.gcode].sum())
    assert len(got.tidy()) == 3 and "leave-out" in got.summary()


def test_steps_3_4_on_a_device_fit(device):
    """On a 200k-row panel fitted on the device: the residuals have zero
    weighted mean in every group and their weighted sum of squares is
    A_yy - A_yx beta (the normal equations), to the solver's tolerance."""
    import torch
    from hdfe_stream_b200 import fit, simulate
    panel = simulate.simulate_panel(25_000, 1_500, 10, spell=(5, 10), weights=True, seed=7)
    rows = simulate.pass0_layout(panel, simulate.restrict_connected(panel, (1, 1)))
    drows = fit.DeviceRows.from_rows(rows)
    res = fit.fit(drows, tol=1e-12)
    from hdfe_stream_b200 import leaveout
    op = leaveout.InverseOperator(drows, res.cells, res.S, tol=1e-12)
    A = op.residual_moments(res.gamma).cpu().numpy()
    beta = np.linalg.solve(A[1:, 1:], A[1:, 0])
    e, alpha, _, _ = op.row_effects(res.gamma, beta)
    e = e.cpu().numpy()
    w = rows.w
    starts = op.starts.cpu().numpy()
    gsum = np.add.reduceat(w * e, starts[:-1])
    assert np.max(np.abs(gsum)) < 1e-8 * np.sqrt(w @ (e * e))
    assert rel(w @ (e * e), A[0, 0] - A[0, 1:] @ beta) < 1e-7


def test_leave_out_components_against_exact_prototype(device):
    """On the device, the same check as the oracle's against the reference's
    dense exact KSS (prototypes/kss_exact.py on a 1,500-worker leave-one-out
    panel, worker and firm effects only): the plug-in exactly, the leave-out
    components within 5% of the bias term at 1,024 probes and draws."""
    import torch
    from hdfe_stream_b200 import fit, leaveout
    from hdfe_stream_b200.simulate import Rows
    g = load_golden("exact")
    rows = Rows(gcode=g["gcode"], codes=g["codes_rows"], V=g["V"][:, :1], w=None,
                n_levels=[int(x) for x in g["n_levels"]], n_groups=int(g["n_groups"][0]),
                names=["log_earn"])
    drows = fit.DeviceRows.from_rows(rows)
    res = fit.fit(drows, tol=1e-12)
    op = leaveout.InverseOperator(drows, res.cells, res.S, None, tol=1e-12)
    out = op.leave_out_components(res, 1024, 32, 3)
    assert rel(vals(out.plug_in), g["plug_in"]) < 1e-9
    assert np.all(np.abs(vals(out.leave_out) - g["kss"]) <= 0.05 * np.abs(g["bias"]))
    lev = out.leverages.leverage.cpu()
    assert float(torch.mean(torch.abs(lev - torch.as_tensor(g["P_ii"])))) < 0.02


def test_leave_out_match_matches_oracle(device):
    """Leaving out a match on the device against the oracle's restatement with
    the same draws, on a leave-one-out panel with year effects and the
    model's covariates (partialled out before the collapse), and against the
    exact prototype's stayer variances and plug-in on the exact panel."""
    from hdfe_stream_b200 import fit
    from hdfe_stream_b200.leaveout_match import leave_out_match
    from hdfe_stream_b200.simulate import Rows, pass0_layout, simulate_panel, _rank_codes
    panel = simulate_panel(3_000, 300, 8, spell=(2, 8), p_move=0.15, seed=31)
    a, _ = _rank_codes(panel.worker)
    b, flev = _rank_codes(panel.firm)
    n0, n1 = int(a.max()) + 1, len(flev)
    order = np.lexsort((b, a))
    alive, _, _ = orc.leave_one_out(a[order], b[order], n0, n1)
    keep = alive[a] & alive[n0 + b.astype(np.int64)]
    rows = pass0_layout(panel, keep)
    ref = orc.leave_out_match(rows, 64, 32, 5)
    drows = fit.DeviceRows.from_rows(rows)
    res = fit.fit(drows, tol=1e-12)
    got = leave_out_match(drows, res, n_draws=64, block=32, seed=5, tol=1e-12)
    d = got.diagnostics
    assert d["n_matches"] == ref["n_matches"]
    assert d["stayer_matches"] == ref["stayer_matches"]
    assert got.n_obs == rows.n_rows and d["leave_out"] == "match"
    assert rel(vals(got.plug_in), ref["plug_in"]) < 1e-9
    assert rel(d["sigma2"].cpu().numpy(), ref["sigma2"]) < 1e-7
    assert rel(vals(got.bias), ref["bias"]) < 1e-7
    g = load_golden("exact")
    erows = Rows(gcode=g["gcode"], codes=g["codes_rows"], V=g["V"][:, :1], w=None,
                 n_levels=[int(x) for x in g["n_levels"]], n_groups=int(g["n_groups"][0]),
                 names=["log_earn"])
    d2 = fit.DeviceRows.from_rows(erows)
    out = leave_out_match(d2, fit.fit(d2, tol=1e-12), n_draws=256, block=32, seed=3, tol=1e-12)
    st = g["match_stayer"]
    assert rel(vals(out.plug_in), g["match_plug_in"]) < 1e-9
    assert rel(out.diagnostics["sigma2"].cpu().numpy()[st], g["match_sigma2"][st]) < 1e-8


@pytest.mark.parametrize("rule,weights", [("person_year", False), ("match", True)])
def test_leave_out_match_standard_errors_match_oracle(device, rule, weights):
    """Match-level standard errors on the device against the oracle with the
    same draws: the per-match variances and theta, the first and trace
    terms and V of var(psi) and cov(psi, alpha), on a leave-one-out panel
    with year effects (weighted for the "match" rule, which takes weights)."""
    from hdfe_stream_b200 import fit
    from hdfe_stream_b200.leaveout_match import leave_out_match
    from hdfe_stream_b200.simulate import pass0_layout, simulate_panel, _rank_codes
    panel = simulate_panel(2_000, 200, 8, spell=(2, 8), p_move=0.15, weights=weights, seed=37)
    a, _ = _rank_codes(panel.worker)
    b, flev = _rank_codes(panel.firm)
    n0, n1 = int(a.max()) + 1, len(flev)
    order = np.lexsort((b, a))
    alive, _, _ = orc.leave_one_out(a[order], b[order], n0, n1)
    keep = alive[a] & alive[n0 + b.astype(np.int64)]
    rows = pass0_layout(panel, keep)
    ref = orc.leave_out_match(rows, 64, 32, 5, se=True, se_variance=rule, se_draws=24)
    drows = fit.DeviceRows.from_rows(rows)
    res = fit.fit(drows, tol=1e-12)
    got = leave_out_match(drows, res, n_draws=64, block=32, seed=5, tol=1e-12, se=True,
                          se_variance=rule, se_draws=24)
    assert rel(got.diagnostics["sigma2_se"].cpu().numpy(), ref["sigma2_se"]) < 1e-7
    names = ("var(psi)", "cov(psi, alpha)")
    for key in ("theta", "first_term", "trace_term", "variance"):
        part = getattr(got.se, key)
        assert rel([part[n] for n in names], ref["se"][key][[0, 2]]) < 1e-6, key
    assert np.isnan(got.se.variance["var(alpha)"])
    if rule == "person_year":
        with pytest.raises(ValueError):
            wrows = fit.DeviceRows.from_rows(pass0_layout(
                simulate_panel(300, 30, 6, spell=(2, 6), weights=True, seed=3)))
            leave_out_match(wrows, fit.fit(wrows), se=True, se_variance="person_year")

"""The oracle against the reference's own outputs (tests/golden/, made by
tests/golden/make_golden.py from the reference's numba kernels and mixins).

Integer outputs (cell layout, counts, codes, CSR pattern, component labels)
must be identical; floating-point outputs are compared to 1e-12 relative,
and most are bit-identical since the oracle keeps the reference's order of
operations."""

import numpy as np
import pytest

import oracle as orc
from conftest import golden_rows, load_golden


def rel(a, b):
    a, b = np.asarray(a, float), np.asarray(b, float)
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300)) if a.size else 0.0


@pytest.fixture
def cells(golden):
    name, g = golden
    return name, g, orc.pass1(golden_rows(g))


def test_pass1_cells_match_reference(cells):
    name, g, c = cells
    assert np.array_equal(c.starts, g["starts"])
    assert np.array_equal(c.codes, g["codes"])
    assert c.n_cells == int(g["n_cells"])
    assert c.fe0_rank == int(g["fe0_rank"])
    assert np.array_equal(c.cnt, g["cnt"])
    np.testing.assert_array_equal(c.n, g["n"])
    assert rel(c.obs, g["obs"]) < 1e-13
    assert rel(c.sums, g["sums"]) < 1e-12
    assert rel(c.diag, g["diag"]) < 1e-12
    assert rel(c.rhs, g["rhs"]) < 1e-12


def test_pair_components_match_reference(cells):
    name, g, c = cells
    # the reference's keys, sorted: (firm, year), (worker, firm), (worker, year)
    _, nc = orc.component_labels(c)
    year_roots = orc.components(c, 1)
    got = [c.pair_components[(0, 1)], nc,
           int(np.count_nonzero(year_roots == np.arange(len(year_roots))))]
    assert got == [int(x) for x in g["pair_components"]]


def test_component_labels_match_reference(cells):
    name, g, c = cells
    comp, nc = orc.component_labels(c)
    assert nc == int(g["n_components"])
    assert np.array_equal(comp, g["comp"])


def test_explicit_s_matches_reference(cells):
    name, g, c = cells
    indptr, indices, data = orc.build_explicit(c)
    assert np.array_equal(indptr, g["S_indptr"])
    assert np.array_equal(indices, g["S_indices"])
    np.testing.assert_array_equal(data, g["S_data"])


def test_pcg_matches_reference(golden):
    name, g = golden
    S = (g["S_indptr"], g["S_indices"], g["S_data"])
    dinv = orc.jacobi(g["diag"])
    X, it, ok, r = orc.pcg(S, dinv, g["pcg_b"], g["pcg_zero"], None, float(g["tol"]))
    assert it == int(g["pcg_it"]) and ok == bool(g["pcg_ok"])
    np.testing.assert_array_equal(X, g["pcg_X"])
    X2, it2, ok2, r2 = orc.pcg(S, dinv, g["pcg_b"], g["pcg_zero"], g["pcg_x0"], float(g["tol"]))
    assert it2 == int(g["pcg_it2"])
    np.testing.assert_array_equal(X2, g["pcg_X2"])


def test_step2_solve_matches_reference(cells):
    name, g, c = cells
    S = orc.build_explicit(c)
    gamma, info = orc.solve(c, S, tol=float(g["tol"]))
    assert list(np.atleast_1d(info["iterations"])) == list(g["gamma_iterations"])
    assert rel(gamma, g["gamma"]) < 1e-12


def test_rademacher_matches_reference(golden):
    name, g = golden
    np.testing.assert_array_equal(orc.rademacher(1000, 257, 5, 12345, 7), g["rademacher"])


def _project(g, c, seed, n_vec, weighted):
    """project_rows (inverse.py:240-309) restated on the oracle's kernels."""
    rows = golden_rows(g)
    nt = int(g["numba_threads"])
    starts = orc.row_starts(rows.gcode)
    w = rows.w if weighted else np.ones(rows.n_rows)
    R = orc.rademacher(0, rows.n_rows, n_vec, seed, 0)
    if weighted:
        # inverse.py:280-281, 298-303: W^(1/2) A S^- A' W^(1/2) = rows scaled
        # by w^(-1/2) on the way in, by w^(1/2) on the way out
        root = np.sqrt(w)
        R = R * (1.0 / root)[:, None]
    rhs, _ = orc.center_rows(starts, rows.codes, c.offs, w, np.zeros((rows.n_rows, 0)), R,
                             c.L, nt)
    S = orc.build_explicit(c)
    zero = np.linalg.norm(rhs, axis=0) <= orc.RHS_ZERO_TOL * np.sqrt(w @ (R * R))
    U, *_ = orc.pcg(S, orc.jacobi(c.diag), rhs, zero, None, float(g["tol"]))
    R2 = orc.rademacher(0, rows.n_rows, n_vec, seed, 0)
    if weighted:
        R2 = R2 * (1.0 / root)[:, None]
    out = orc.project_rows_kernel(starts, rows.codes, c.offs, w, np.zeros((rows.n_rows, 0)),
                                  np.zeros((0, n_vec)), R2, U)
    return out * root[:, None] if weighted else out


def test_project_rows_matches_reference(cells):
    name, g, c = cells
    out = _project(g, c, 11, 6, len(g["w"]) > 0)
    assert rel(out, g["project_rows_seed11"]) < 1e-10


def test_design_projection_matches_reference(cells):
    """The oracle's project_rows (inverse.py:240-309 restated) on the golden
    projection of seed 11, 6 draws."""
    name, g, c = cells
    rows = golden_rows(g)
    des = orc.Design(rows, c, orc.build_explicit(c), tol=float(g["tol"]), nt=int(g["numba_threads"]))
    out = des.project_rows(6, 11, 0, sqrt_weights=rows.w is not None)
    assert rel(out, g["project_rows_seed11"]) < 1e-10


def test_jla_leverages_match_reference(cells):
    name, g, c = cells
    rows = golden_rows(g)
    des = orc.Design(rows, c, orc.build_explicit(c), tol=float(g["tol"]), nt=int(g["numba_threads"]))
    lev, comp, factor = des.jla_leverages(24, 8, 2)
    assert rel(lev, g["jla_leverage"]) < 1e-9
    assert rel(factor, g["jla_factor"]) < 1e-9


def test_apply_inverse_matches_reference(golden):
    """inverse.py `apply_inverse` on a coefficient-space right-hand side
    (levels and groups, null-space component dropped): U, the streamed block
    and the rows' (A u)_i against the reference's outputs."""
    _, g = golden
    rows = golden_rows(g)
    c = orc.pass1(rows)
    des = orc.Design(rows, c, orc.build_explicit(c), tol=float(g["tol"]))
    U, C, Ug, R = des.apply_inverse(g["ainv_levels"], np.zeros((0, 3)), g["ainv_groups"])
    for got, ref in ((U, g["ainv_U"]), (Ug, g["ainv_Ug"]), (R, g["ainv_rows"])):
        assert np.max(np.abs(got - ref)) < 1e-10 * np.max(np.abs(ref))


def test_hutchinson_trace_matches_reference(golden):
    """leaveout.py `hutchinson_trace`: the three bias terms for 16 draws in
    blocks of 8."""
    _, g = golden
    rows = golden_rows(g)
    c = orc.pass1(rows)
    des = orc.Design(rows, c, orc.build_explicit(c), tol=float(g["tol"]))
    tr = des.hutchinson_trace(g["trace_sigma2"], 16, 8, 4)
    assert np.max(np.abs(tr - g["trace"])) < 1e-10 * np.max(np.abs(g["trace"]))


@pytest.mark.parametrize("panel", ["sparse", "middle", "dense"])
@pytest.mark.parametrize("k", [1, 2])
def test_largest_connected_matches_reference(panel, k):
    """`_find_components` for connected="largest": distinct pairs, the
    min_degree core, component labels ranked by rows, rows per component --
    against the reference's own kernels (tests/golden/connected.npz)."""
    g = load_golden("connected")
    n0, n1 = (int(x) for x in g[f"{panel}_n"])
    largest, labels, rows = orc.largest_connected(g[f"{panel}_a"], g[f"{panel}_b"], n0, n1,
                                                  (k, k))
    assert np.array_equal(labels, g[f"{panel}_k{k}_labels"])
    assert np.array_equal(rows, g[f"{panel}_k{k}_rows"])


def test_steps_3_4_match_reference(golden):
    """V' W V (`_nb_residualize_rows` + `_assemble`), beta, and the row pass
    (`_nb_pass2`): residuals, the streamed effect and the first non-streamed
    effect per row, against the reference's kernels on its own Gamma."""
    name, g = golden
    a = load_golden("assemble")
    rows = golden_rows(g)
    starts = orc.row_starts(rows.gcode)
    offs = np.concatenate(([0], np.cumsum(rows.n_levels)[:-1])).astype(np.int64)
    w = rows.w if rows.w is not None else np.ones(rows.n_rows)
    A = orc.residual_moments(starts, rows.codes, offs, w, rows.V, g["gamma"])
    assert rel(A, a[f"{name}_A"]) < 1e-12
    beta = np.linalg.solve(A[1:, 1:], A[1:, 0])
    assert rel(beta, a[f"{name}_beta"]) < 1e-10
    e, alpha, psi, gam_y = orc.row_effects(starts, rows.codes, offs, w, rows.V, g["gamma"], beta)
    assert rel(e, a[f"{name}_resid"]) < 1e-10
    assert rel(alpha, a[f"{name}_alpha"]) < 1e-10
    assert rel(psi, a[f"{name}_psi"]) < 1e-10


@pytest.mark.parametrize("panel", ["sparse", "middle", "dense", "fringe"])
@pytest.mark.parametrize("k", [1, 2])
def test_leave_one_out_matches_reference(panel, k):
    """`_leave_one_out` (the leave-one-out connected set, after the (k, k)
    core): levels kept, components before, single observations, workers cut
    and rounds, rows kept -- against the reference's own function."""
    g = load_golden("connected")
    n0, n1 = (int(x) for x in g[f"{panel}_n"])
    alive, rows, info = orc.leave_one_out(g[f"{panel}_a"], g[f"{panel}_b"], n0, n1, (k, k))
    assert np.array_equal(alive, g[f"{panel}_k{k}_loo_alive"])
    got = [info["components_before"], info["single_observation"], info["cut"], info["rounds"],
           rows]
    assert got == [int(x) for x in g[f"{panel}_k{k}_loo_counts"]]


def se_rows(g, name):
    """The standard-error golden panel's rows (its leave-one-out set)."""
    from hdfe_stream_b200.simulate import Rows
    w = g[f"{name}_w"] if len(g[f"{name}_w"]) else None
    return Rows(gcode=g[f"{name}_gcode"], codes=g[f"{name}_codes_rows"], V=g[f"{name}_V"], w=w,
                n_levels=[int(x) for x in g[f"{name}_n_levels"]],
                n_groups=int(g[f"{name}_n_groups"][0]),
                names=["log_earn", "age_squared", "age_cubed"])


@pytest.mark.parametrize("name", ["akm_small", "akm_weighted"])
def test_standard_errors_match_reference(name):
    """leaveout_se.py `bii_rows` and `component_variances` (B_ii per row,
    the first and trace terms, theta, the variance) against the reference's
    own outputs for the same draws."""
    g = load_golden("se")
    rows = se_rows(g, name)
    c = orc.pass1(rows)
    des = orc.Design(rows, c, orc.build_explicit(c), tol=float(g[f"{name}_tol"][0]))
    b_ii = des.bii_rows(16, 8, 6)
    assert rel(b_ii, g[f"{name}_bii"]) < 1e-9
    out = des.component_variances(g[f"{name}_sigma2"], g[f"{name}_leverage"],
                                  g[f"{name}_complement"], g[f"{name}_factor"], b_ii, 16, 8, 6)
    for key in ("first_term", "trace_term", "theta", "variance"):
        assert rel(out[key], g[f"{name}_{key}"]) < 1e-8, key


def exact_rows(g):
    from hdfe_stream_b200.simulate import Rows
    return Rows(gcode=g["gcode"], codes=g["codes_rows"], V=g["V"][:, :1], w=None,
                n_levels=[int(x) for x in g["n_levels"]], n_groups=int(g["n_groups"][0]),
                names=["log_earn"])


def test_jla_components_against_exact_prototype():
    """The leave-out components by JLA (1,024 probes and draws) against the
    reference's dense exact prototype (prototypes/kss_exact.py `kss`,
    tests/golden/exact.npz): the plug-in exactly, the leave-out estimates
    within 5% of the bias term, the leverages within 0.02 on average."""
    g = load_golden("exact")
    rows = exact_rows(g)
    c = orc.pass1(rows)
    S = orc.build_explicit(c)
    gamma, _ = orc.solve(c, S, tol=1e-12)
    des = orc.Design(rows, c, S, tol=1e-12)
    out = des.leave_out_components(gamma, 1024, 32, 3)
    assert rel(out["plug_in"], g["plug_in"]) < 1e-9
    assert np.all(np.abs(out["leave_out"] - g["kss"]) <= 0.05 * np.abs(g["bias"]))
    lev, _, _ = des.jla_leverages(1024, 32, 3)
    assert np.mean(np.abs(lev - g["P_ii"])) < 0.02


def test_variances_match_reference(golden):
    """The pass-2 sums (bread, heteroskedastic meat, the streamed groups'
    clustered meat, rss) against the reference's `_nb_pass2` and
    core/inference.py's sums, and the iid / HC1 / CRV1 variances."""
    name, g = golden
    a = load_golden("assemble")
    rows = golden_rows(g)
    starts = orc.row_starts(rows.gcode)
    offs = np.concatenate(([0], np.cumsum(rows.n_levels)[:-1])).astype(np.int64)
    w = rows.w if rows.w is not None else np.ones(rows.n_rows)
    B, mhc, mg, rss = orc.variance_sums(starts, rows.codes, offs, w, rows.V, g["gamma"],
                                        a[f"{name}_beta"])
    for got, key in ((B, "B"), (mhc, "meat_hc"), (mg, "meat_g"), (rss, "rss")):
        assert rel(got, a[f"{name}_{key}"]) < 1e-10, key
    v = orc.variances(B, mhc, mg, rss, rows.n_rows, rows.n_groups, rows.n_levels,
                      [int(x) for x in g["pair_components"]])
    assert v["k_fe"] == int(a[f"{name}_k_fe"][0])
    for key, ref in (("iid", "V_iid"), ("hetero", "V_hc1"), ("CRV1", "V_crv1")):
        assert rel(v[key], a[f"{name}_{ref}"]) < 1e-9, key


def test_leave_out_match_against_exact_prototype():
    """Leaving out a match (leaveout_match.py `leave_out_match`) against the
    reference's dense exact `kss_match` on the same leave-one-out panel: the
    plug-in exactly, the stayers' matches' sigma2 (`sigma_for_stayers`, no
    leverage involved) to 1e-8, and the leave-out components within 15% of
    the bias term at 1,024 draws (the movers' leverages come from JLA, which
    at match level -- leverages up to 0.9 -- converges slowly)."""
    g = load_golden("exact")
    rows = exact_rows(g)
    out = orc.leave_out_match(rows, 1024, 32, 3)
    assert rel(out["plug_in"], g["match_plug_in"]) < 1e-9
    st = g["match_stayer"]
    assert out["n_matches"] == len(st) and out["stayer_matches"] == int(st.sum())
    assert rel(out["sigma2"][st], g["match_sigma2"][st]) < 1e-8
    assert np.all(np.abs(out["leave_out"] - g["match_kss"]) <= 0.15 * np.abs(g["match_bias"]))


def test_match_level_kernel_matches_reference():
    """The match level's options of leaveout_se.py `component_variances`
    (stayers' b zeroed, the reference-centred kernel with its rank-two term
    through `_m_times`, var(alpha) unreported) against the reference's own
    outputs for the same sigma2, leverages and draws (tests/golden/
    match_se.npz, made by tests/golden/make_match_se.py)."""
    g = load_golden("match_se")
    ref = {f"r_{k[4:]}": v for k, v in g.items() if k.startswith("ref_")}
    ref["r_w"] = np.zeros(0)
    rows = se_rows(ref, "r")
    c = orc.pass1(rows)
    des = orc.Design(rows, c, orc.build_explicit(c), tol=float(ref["r_tol"][0]))
    b_ii = des.bii_rows(16, 8, 6)
    assert rel(b_ii, ref["r_bii"]) < 1e-9
    with np.errstate(divide="ignore", invalid="ignore"):
        out = des.component_variances(ref["r_sigma2"], ref["r_leverage"], ref["r_complement"],
                                      ref["r_factor"], b_ii, 16, 8, 6,
                                      stayer_rows=ref["r_stayer"], centering="reference",
                                      reported=(0, 2))
    for key in ("first_term", "trace_term", "theta", "variance"):
        assert np.isnan(out[key][1]) and np.isnan(ref[f"r_{key}"][1])
        assert rel(out[key][[0, 2]], ref[f"r_{key}"][[0, 2]]) < 1e-8, key


@pytest.mark.parametrize("rule", ["person_year", "match"])
def test_match_standard_errors_against_exact_prototype(rule):
    """Match-level standard errors of var(psi) and cov(psi, alpha) with 512
    JLA and trace draws against the reference's dense exact `kss_match_se`
    (prototypes/kss_exact.py:636-716, exact leverages and B_ii) on the
    exact panel: theta within 1%, the variance and its first term within
    10%, the trace term within 25% (the JLA leverages and B_ii move the
    smoother's cells)."""
    g = load_golden("match_se")
    rows = exact_rows(load_golden("exact"))
    with np.errstate(divide="ignore", invalid="ignore"):
        se = orc.leave_out_match(rows, 512, 32, 3, se=True, se_variance=rule)["se"]
    for key, ek, tol in (("theta", "theta", 0.01), ("variance", "V", 0.1),
                         ("first_term", "first", 0.1), ("trace_term", "trace", 0.25)):
        want = g[f"exact_{rule}_{ek}"]
        assert np.all(np.abs(se[key][[0, 2]] - want) <= tol * np.abs(want)), key
    assert np.isnan(se["variance"][1])


@pytest.mark.parametrize("name", ["akm_small", "low_mobility"])
def test_weak_id_diagnostics_match_reference(name):
    """leaveout_weakid.py `weak_id_diagnostics` (Lanczos on Q S^-, the
    deflated Hutchinson sum of squared eigenvalues, q, the first-stage F)
    against the reference's own outputs on a well-connected panel (q = 0)
    and a low-mobility one (q = 1) (tests/golden/weakid.npz, made by
    tests/golden/make_weakid.py)."""
    g = load_golden("weakid")
    rows = se_rows(g, name)
    c = orc.pass1(rows)
    des = orc.Design(rows, c, orc.build_explicit(c), tol=float(g[f"{name}_tol"][0]))
    out = orc.weak_id_diagnostics(des, g[f"{name}_sigma2"], g[f"{name}_leverage"], n_draws=48,
                                  block=12, seed=9)
    assert out["steps"] == int(g[f"{name}_steps"][0])
    assert list(out["lengths"]) == list(g[f"{name}_lengths"])
    assert out["n_draws"] == int(g[f"{name}_n_draws"][0])
    assert out["deflated"] == int(g[f"{name}_deflated"][0])
    for k in range(3):
        assert rel(out["eigenvalues"][k], g[f"{name}_eig{k}"]) < 1e-10
        assert rel(out["ratios"][k], g[f"{name}_ratio{k}"]) < 1e-10
    assert rel(out["sum_sq"], g[f"{name}_sum_sq"]) < 1e-10
    assert rel(out["sum_sq_se"], g[f"{name}_sum_sq_se"]) < 1e-8
    assert list(out["q"]) == list(g[f"{name}_q"])
    assert rel(out["f_stat"], g[f"{name}_f_stat"]) < 1e-10


def test_weak_moments_match_reference():
    """leaveout_se.py `_weak_moments` (b1, its raw variance, the 2x2
    covariance of (b1, theta1) from the deflated kernel C2) for the
    components the diagnostic flags on the low-mobility panel, and the
    standard errors beside them, against the reference's own outputs."""
    g = load_golden("weakid")
    name = "low_mobility"
    rows = se_rows(g, name)
    c = orc.pass1(rows)
    des = orc.Design(rows, c, orc.build_explicit(c), tol=float(g[f"{name}_tol"][0]))
    wid = orc.weak_id_diagnostics(des, g[f"{name}_sigma2"], g[f"{name}_leverage"], n_draws=48,
                                  block=12, seed=9)
    b_ii = des.bii_rows(16, 8, 6)
    out = des.component_variances(g[f"{name}_sigma2"], g[f"{name}_leverage"],
                                  g[f"{name}_complement"], g[f"{name}_factor"], b_ii, 16, 8, 6,
                                  weak_id=wid)
    for f in ("variance", "first_term", "trace_term", "theta"):
        assert rel(out[f], g[f"{name}_se_{f}"]) < 1e-10, f
    flagged = list(g[f"{name}_weak_components"])
    assert sorted(out["weak"]) == flagged and flagged
    for k in flagged:
        piece = out["weak"][k]
        for f in ("lambda_1", "b1", "v_raw", "trace", "quadratic"):
            assert rel(piece[f], g[f"{name}_weak{k}_{f}"]) < 1e-10, f
        assert rel(piece["sigma"], g[f"{name}_weak{k}_sigma"]) < 1e-10
        assert piece["conservative"] == bool(g[f"{name}_weak{k}_conservative"][0])


def test_am_interval_matches_reference():
    """The q = 1 interval (am_interval.py `am_interval`: the Andrews-
    Mikusheva critical value for KSS's curvature and the range of
    lambda_1 b^2 + t over the ellipse) against the reference on fixed inputs
    across curvatures and on the low-mobility panel's moments."""
    from hdfe_stream_b200.am_interval import am_interval
    g = load_golden("weakid")
    for lam, b1, th, s00, s01, s11, alpha, lo, hi, kap, z in g["am_cases"]:
        l2, h2, info = am_interval(lam, b1, th, [[s00, s01], [s01, s11]], alpha)
        assert rel([l2, h2, info["kappa"], info["z"]], [lo, hi, kap, z]) < 1e-12
    name = "low_mobility"
    for k in g[f"{name}_weak_components"]:
        lam, b1 = g[f"{name}_weak{k}_lambda_1"][0], g[f"{name}_weak{k}_b1"][0]
        theta1 = g[f"{name}_weak_leave_out"][k] - lam * (b1 ** 2 - g[f"{name}_weak{k}_v_raw"][0])
        lo, hi, info = am_interval(lam, b1, theta1, g[f"{name}_weak{k}_sigma"], 0.05)
        want = g[f"{name}_weak{k}_interval"]
        assert rel([lo, hi, info["kappa"], info["z"], info["rho"]], want) < 1e-12


def test_am_critical_value_at_small_curvature():
    """Where kappa is tiny the drop of the integrand over b is ~1/(2 kappa^-1)
    wide; the critical value must still exceed the chi-squared(1) bound
    (P(rho <= z1) < 1 - alpha for every kappa > 0).  Checked against the
    distribution function integrated over b on a split interval."""
    import math
    from scipy import integrate, special
    from hdfe_stream_b200.am_interval import am_cdf, am_critical_value
    for kappa in (1e-6, 1.5e-4, 1e-2, 1.0, 50.0):
        c = 1.0 / kappa
        z1 = math.sqrt(special.chdtri(1, 0.05))
        z = am_critical_value(kappa, 0.05)
        assert z > z1

        def f(b, zz=z):
            r = math.sqrt(max((zz - b) * (zz + b + 2.0 * c), 0.0))
            return 2.0 * math.exp(-0.5 * b * b) / math.sqrt(2.0 * math.pi) * (
                2.0 * special.ndtr(r) - 1.0)
        cuts = sorted({0.0, max(z - 50.0 / c, 0.0), max(z - 5.0 / c, 0.0), z})
        F = sum(integrate.quad(f, a, b, epsabs=1e-15, epsrel=1e-13, limit=500)[0]
                for a, b in zip(cuts[:-1], cuts[1:]))
        assert abs(F - 0.95) < 1e-11, (kappa, F)
        assert abs(am_cdf(z, kappa) - 0.95) < 1e-13


def test_ritz_selection_matches_oracle():
    """weakid.ritz_top (ghost runs, the Cullum-Willoughby test, ranking)
    against the oracle's restatement of the reference's `_ritz_top` on
    random tridiagonals and on ones with exact and near copies of an
    eigenvalue (two identical blocks joined by a zero or tiny coupling)."""
    from hdfe_stream_b200.weakid import ritz_top
    rng = np.random.default_rng(8)
    cases = []
    for m in (1, 2, 3, 7, 20):
        cases.append((rng.normal(size=m), np.abs(rng.normal(size=m))))
    for couple in (0.0, 1e-14, 1e-3):
        a = rng.normal(size=6)
        b = np.abs(rng.normal(size=6))
        cases.append((np.concatenate([a, a]), np.concatenate([b[:5], [couple], b[:5], [b[5]]])))
    for alpha, beta in cases:
        for top in (1, 3):
            got = ritz_top(alpha, beta, top)
            ref = orc.ritz_top(alpha, beta, top)
            for x, y in zip(got, ref):
                assert np.array_equal(np.asarray(x), np.asarray(y))


@pytest.mark.parametrize("name", ["akm_small", "akm_weighted", "akm_components"])
def test_cluster_variances_match_reference(name):
    """Pass 2's per-row scores and the CRV1 variances for cluster requests
    beyond the streamed dimension -- another dimension, two-way
    (inclusion-exclusion), a refinement of the streamed groups, two-way over
    the non-streamed dimensions -- against the reference's own kernel outputs
    and formulas (tests/golden/assemble.npz)."""
    ga = load_golden("assemble")
    g = load_golden(name)
    rows = golden_rows(g)
    starts = orc.row_starts(rows.gcode)
    codes = np.asarray(rows.codes, np.int64)
    nlev = np.asarray(rows.n_levels, np.int64)
    offs = np.concatenate(([0], np.cumsum(nlev)[:-1]))
    w = rows.w if rows.w is not None else np.ones(rows.n_rows)
    he = orc.row_scores(starts, codes, offs, w, rows.V, g["gamma"], ga[f"{name}_beta"])
    assert rel(he, ga[f"{name}_scores"]) < 1e-10
    pcs = [int(x) for x in g["pair_components"]]
    pc = {("firm", "year"): pcs[0], ("worker", "firm"): pcs[1], ("worker", "year"): pcs[2]}
    Binv = np.linalg.inv(ga[f"{name}_B"])
    reqs = ("firm", "worker+firm", "worker^firm", "firm+year")
    out = orc.cluster_variances(he, rows.gcode, codes, nlev, Binv, reqs,
                                ("worker", "firm", "year"), pc)
    for req in reqs:
        V, Gs, adj, _ = out[req]
        assert list(Gs) == [int(x) for x in ga[f"{name}_crv1_{req}_G"]], req
        assert abs(adj - ga[f"{name}_crv1_{req}_adj"][0]) < 1e-12, req
        assert rel(V, ga[f"{name}_crv1_{req}_V"]) < 1e-9, req
    # the one-way request on the streamed dimension is the kernel's own CRV1
    V, Gs, adj, nest = orc.cluster_variances(he, rows.gcode, codes, nlev, Binv, ("worker",),
                                             ("worker", "firm", "year"), pc)["worker"]
    assert nest == ["worker"] and rel(V, ga[f"{name}_V_crv1"]) < 1e-9


def test_standard_errors_and_weak_id_against_exact_prototype():
    """The observation-level standard errors (512 JLA probes, B_ii and trace
    draws) and the weak-identification diagnostic against the reference's
    dense exact prototype on the exact panel (prototypes/kss_exact.py
    `kss_se` with the smoothed sigma2 and `weak_id`; tests/golden/
    exact_se.npz): theta within 0.5%, V and its first term within 3%, the
    trace term within 10%; the Lanczos eigenvalues to 1e-6 (no Monte Carlo
    in them), sum lambda^2 within 10% at 64 draws, q equal, F within 10%."""
    g, ge = load_golden("exact"), load_golden("exact_se")
    rows = exact_rows(g)
    c = orc.pass1(rows)
    S = orc.build_explicit(c)
    gamma, _ = orc.solve(c, S, tol=1e-12)
    des = orc.Design(rows, c, S, tol=1e-12)
    out = des.leave_out_components(gamma, 512, 32, 3)
    lev, comp, factor = des.jla_leverages(512, 32, 3)
    se = des.component_variances(out["sigma2"], lev, comp, factor, des.bii_rows(512, 32, 8), 512,
                                 32, 8)
    for key, ek, tol in (("theta", "se_theta", 0.005), ("variance", "se_V", 0.03),
                         ("first_term", "se_V_first_term", 0.03),
                         ("trace_term", "se_V_trace_term", 0.1)):
        assert np.all(np.abs(se[key] - ge[ek]) <= tol * np.abs(ge[ek])), key
    wid = orc.weak_id_diagnostics(des, out["sigma2"], lev, n_draws=64, block=32, seed=9)
    for k in range(3):
        assert rel(wid["eigenvalues"][k], ge[f"weak_eig{k}"]) < 1e-6
    assert np.all(np.abs(wid["sum_sq"] - ge["weak_sum_sq"]) <= 0.1 * ge["weak_sum_sq"])
    assert list(wid["q"]) == [int(x) for x in ge["weak_q"]]
    assert np.all(np.abs(wid["f_stat"] - ge["weak_f_stat"]) <= 0.1 * ge["weak_f_stat"])


@pytest.mark.parametrize("name", ["akm_small", "akm_weighted", "akm_components"])
def test_crv3_jackknife_matches_reference(name):
    """The CRV3 jackknife sums (core/kernels_base.py `_nb_crv3_groups`,
    `_nb_crv3_scatter`, `_nb_crv3_finish`: sum over clusters of d_g d_g',
    d_g = pinv(B - A_g) s_g) by worker and by firm against the reference's
    kernels on its own pass-2 outputs (tests/golden/assemble.npz)."""
    ga = load_golden("assemble")
    g = load_golden(name)
    rows = golden_rows(g)
    starts = orc.row_starts(rows.gcode)
    codes = np.asarray(rows.codes, np.int64)
    nlev = np.asarray(rows.n_levels, np.int64)
    offs = np.concatenate(([0], np.cumsum(nlev)[:-1]))
    w = rows.w if rows.w is not None else np.ones(rows.n_rows)
    he, H = orc.row_scores(starts, codes, offs, w, rows.V, g["gamma"], ga[f"{name}_beta"],
                           with_h=True)
    B = ga[f"{name}_B"]
    for key, code in (("worker", rows.gcode), ("firm", codes[:, 0])):
        assert rel(orc.crv3_jack(code, w, H, he, B), ga[f"{name}_crv3_{key}_jack"]) < 1e-9, key


CASES_WB = [("rademacher", True, 999, 11), ("rademacher", False, 999, 12),
            ("mammen", True, 499, 13), ("webb", True, 499, 14), ("norm", False, 499, 15),
            ("rademacher", True, 999, 16)]


@pytest.mark.parametrize("c", range(6))
def test_wild_bootstrap_matches_reference(c):
    """The wild cluster bootstrap (the oracle and the library's host draws
    with its arithmetic in torch on the CPU) against the reference's
    core/wildboot.py `_draws` / `_Test` for every weight distribution,
    restricted and not, and the Rademacher enumeration (tests/golden/
    wildboot.npz): t and every t* to 1e-10."""
    import torch
    from hdfe_stream_b200.wildboot import bootstrap_t
    g = load_golden("wildboot")
    kind, null, reps, seed = CASES_WB[c]
    args = (g[f"c{c}_AG"], g[f"c{c}_sG"], g[f"c{c}_beta"], 1, float(g[f"c{c}_adj"][0]))
    t, tstar, _ = orc.wild_bootstrap(*args, reps, kind, null, seed)
    assert abs(t - g[f"c{c}_t"][0]) <= 1e-10 * abs(g[f"c{c}_t"][0])
    assert rel(tstar, g[f"c{c}_tstar"]) < 1e-10
    t2, tstar2, _ = bootstrap_t(*args, reps, kind, null, seed, device=torch.device("cpu"))
    assert abs(t2 - g[f"c{c}_t"][0]) <= 1e-10 * abs(g[f"c{c}_t"][0])
    assert rel(tstar2, g[f"c{c}_tstar"]) < 1e-10

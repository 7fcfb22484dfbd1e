"""beta and its variances on the device (hdfe_stream_b200.inference): the
iid, HC1 and CRV1 (streamed dimension) variances, the fixed-effect parameter
count and the pairs' components against the reference's `_nb_pass2` sums and
`_estimate` formulas (tests/golden/assemble.npz) and against the oracle on a
device fit."""

import numpy as np
import pytest

import oracle as orc
from conftest import GOLDEN_PANELS, golden_rows, load_golden

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


@pytest.mark.parametrize("name", GOLDEN_PANELS)
def test_variances_match_reference(device, name):
    import torch
    from hdfe_stream_b200 import fit, inference
    g = load_golden(name)
    a = load_golden("assemble")
    drows = fit.DeviceRows.from_rows(golden_rows(g))
    cells = fit.pass1(drows)
    out = inference.estimate(drows, cells, torch.as_tensor(g["gamma"]))
    assert rel(out["beta"], a[f"{name}_beta"]) < 1e-10
    assert sorted(out["pair_components"]) == sorted(int(x) for x in g["pair_components"])
    assert out["k_fe"] == int(a[f"{name}_k_fe"][0])
    for key, ref in (("iid", "V_iid"), ("hetero", "V_hc1"), ("CRV1", "V_crv1")):
        assert rel(out["vcov"][key], a[f"{name}_{ref}"]) < 1e-9, key


def test_variances_on_a_device_fit(device):
    """A 60k-worker weighted panel fitted on the device: the variances from
    its own Gamma against the oracle's on the same Gamma."""
    from hdfe_stream_b200 import fit, inference
    from hdfe_stream_b200.simulate import pass0_layout, restrict_connected, simulate_panel
    panel = simulate_panel(60_000, 6_000, 10, spell=(3, 10), p_move=0.1, weights=True, seed=4)
    rows = pass0_layout(panel, restrict_connected(panel, (1, 1)))
    drows = fit.DeviceRows.from_rows(rows)
    res = fit.fit(drows, tol=1e-12)
    out = inference.estimate(drows, res.cells, res.gamma)
    gamma = res.gamma.cpu().numpy()
    starts = orc.row_starts(rows.gcode)
    offs = np.concatenate(([0], np.cumsum(rows.n_levels)[:-1])).astype(np.int64)
    A = orc.residual_moments(starts, rows.codes, offs, rows.w, rows.V, gamma)
    beta = np.linalg.solve(A[1:, 1:], A[1:, 0])
    assert rel(out["beta"], beta) < 1e-10
    c = orc.pass1(rows)
    pcs = [c.pair_components[(0, 1)], orc.component_labels(c)[1],
           int(np.count_nonzero(orc.components(c, 1) == np.arange(rows.n_levels[1])))]
    assert sorted(out["pair_components"]) == sorted(pcs)
    v = orc.variances(*orc.variance_sums(starts, rows.codes, offs, rows.w, rows.V, gamma, beta),
                      rows.n_rows, rows.n_groups, rows.n_levels, pcs)
    assert out["k_fe"] == v["k_fe"]
    for key in ("iid", "hetero", "CRV1"):
        assert rel(out["vcov"][key], v[key]) < 1e-9, key


REQUESTS = ("firm", "worker+firm", "worker^firm", "firm+year")


@pytest.mark.parametrize("name", GOLDEN_PANELS)
def test_cluster_requests_match_reference(device, name):
    """CRV1 for cluster requests beyond the streamed dimension (another
    dimension, two-way, a refinement of the streamed groups, two-way over the
    non-streamed dimensions): the device's per-row scores against pass 2's
    and the variances against the reference's formulas on its own Gamma."""
    import torch
    from hdfe_stream_b200 import fit, inference
    g = load_golden(name)
    a = load_golden("assemble")
    drows = fit.DeviceRows.from_rows(golden_rows(g))
    cells = fit.pass1(drows)
    gamma = torch.as_tensor(g["gamma"])
    scores = inference.row_scores(drows, cells, gamma, a[f"{name}_beta"]).cpu().numpy()
    assert rel(scores, a[f"{name}_scores"]) < 1e-10
    out = inference.estimate(drows, cells, gamma, clusters=REQUESTS,
                             fe_names=("worker", "firm", "year"))
    for req in REQUESTS:
        assert out["clusters"][req]["G"] == [int(x) for x in a[f"{name}_crv1_{req}_G"]], req
        assert abs(out["clusters"][req]["adj"] - a[f"{name}_crv1_{req}_adj"][0]) < 1e-12, req
        assert rel(out["vcov"][f"CRV1:{req}"], a[f"{name}_crv1_{req}_V"]) < 1e-9, req


def test_cluster_requests_with_an_extra_column_match_oracle(device):
    """A request on a column that is not a fixed effect (a region of the
    firms, given per row) and its two-way with the workers, on a weighted
    device fit, against the oracle on the same Gamma."""
    from hdfe_stream_b200 import fit, inference
    from hdfe_stream_b200.simulate import pass0_layout, restrict_connected, simulate_panel
    panel = simulate_panel(30_000, 3_000, 8, spell=(3, 8), p_move=0.1, weights=True, seed=9)
    rows = pass0_layout(panel, restrict_connected(panel, (1, 1)))
    region = (rows.codes[:, 0].astype(np.int64) * 7919) % 37
    drows = fit.DeviceRows.from_rows(rows)
    res = fit.fit(drows, tol=1e-12)
    reqs = ("region", "worker+region", "firm^region")
    out = inference.estimate(drows, res.cells, res.gamma, clusters=reqs,
                             fe_names=("worker", "firm", "year"), extra={"region": region})
    gamma = res.gamma.cpu().numpy()
    starts = orc.row_starts(rows.gcode)
    codes = np.asarray(rows.codes, np.int64)
    nlev = np.asarray(rows.n_levels, np.int64)
    offs = np.concatenate(([0], np.cumsum(nlev)[:-1]))
    he = orc.row_scores(starts, codes, offs, rows.w, rows.V, gamma, out["beta"])
    pcs = out["pair_components"]
    pc = {("worker", "firm"): pcs[0], ("worker", "year"): pcs[1], ("firm", "year"): pcs[2]}
    B = orc.variance_sums(starts, codes, offs, rows.w, rows.V, gamma, out["beta"])[0]
    ref = orc.cluster_variances(he, rows.gcode, codes, nlev, np.linalg.inv(B), reqs,
                                ("worker", "firm", "year"), pc, extra={"region": region})
    for req in reqs:
        V, Gs, adj, nest = ref[req]
        assert out["clusters"][req]["G"] == list(Gs), req
        assert out["clusters"][req]["nested"] == nest, req
        assert abs(out["clusters"][req]["adj"] - adj) < 1e-12, req
        assert rel(out["vcov"][f"CRV1:{req}"], V) < 1e-8, req
    assert out["clusters"]["region"]["nested"] == ["firm"]


@pytest.mark.parametrize("name", GOLDEN_PANELS)
def test_crv3_jackknife_matches_reference(device, name):
    """The device's CRV3 jackknife sums by worker and by firm against the
    reference's `_nb_crv3_*` kernels on its own Gamma."""
    import torch
    from hdfe_stream_b200 import fit, inference
    g = load_golden(name)
    a = load_golden("assemble")
    rows = golden_rows(g)
    drows = fit.DeviceRows.from_rows(rows)
    cells = fit.pass1(drows)
    he, h = inference.row_scores(drows, cells, torch.as_tensor(g["gamma"]), a[f"{name}_beta"],
                                 with_h=True)
    for key, code in (("worker", drows.gcode.to(torch.int64)),
                      ("firm", drows.codes[:, 0].to(torch.int64))):
        G = int(code.max().item()) + 1
        S = torch.zeros((G, he.shape[1]), dtype=torch.float64, device=he.device)
        S.index_add_(0, code, he)
        jack = inference.crv3_jack(code, G, drows.w, h, S, a[f"{name}_B"])
        assert rel(jack, a[f"{name}_crv3_{key}_jack"]) < 1e-9, key


def regions_panel(n_regions=30, seed=0):
    """Regions with their own workers and firms (no one moves between
    regions), so that both fixed effects are nested in the region clusters."""
    from hdfe_stream_b200.simulate import Panel, pass0_layout, simulate_panel
    parts = [simulate_panel(300, 30, 6, spell=(3, 6), p_move=0.2, weights=True, seed=seed + r)
             for r in range(n_regions)]
    cat = lambda f: np.concatenate([getattr(p, f) for p in parts])
    panel = Panel(worker=np.concatenate([p.worker + 300 * r for r, p in enumerate(parts)]),
                  firm=np.concatenate([p.firm + 30 * r for r, p in enumerate(parts)]),
                  year=cat("year"), log_earn=cat("log_earn"), age_squared=cat("age_squared"),
                  age_cubed=cat("age_cubed"), weight=cat("weight"))
    rows = pass0_layout(panel, year_fe=False)      # year effects would span the regions
    firms = np.unique(panel.firm)
    return rows, firms[rows.codes[:, 0]] // 30


def test_crv3_on_nested_regions_matches_oracle(device):
    """CRV3 by region (worker and firm effects, both nested in the regions)
    and CRV1 by region on a device fit of 30 separate regions, against the
    oracle on the same Gamma; CRV3 on a request whose fixed effects are not
    nested is refused (firm clusters: the workers move between firms)."""
    from hdfe_stream_b200 import fit, inference
    rows, region = regions_panel()
    drows = fit.DeviceRows.from_rows(rows)
    res = fit.fit(drows, tol=1e-12)
    names = ("worker", "firm")
    out = inference.estimate(drows, res.cells, res.gamma, clusters=("region",), fe_names=names,
                             extra={"region": region}, crv3=("region",))
    assert sorted(out["clusters"]["region"]["nested"]) == ["firm", "worker"]
    gamma = res.gamma.cpu().numpy()
    starts = orc.row_starts(rows.gcode)
    codes = np.asarray(rows.codes, np.int64)
    nlev = np.asarray(rows.n_levels, np.int64)
    offs = np.concatenate(([0], np.cumsum(nlev)[:-1]))
    he, H = orc.row_scores(starts, codes, offs, rows.w, rows.V, gamma, out["beta"], with_h=True)
    B = orc.variance_sums(starts, codes, offs, rows.w, rows.V, gamma, out["beta"])[0]
    pc = {("worker", "firm"): out["pair_components"][0]}
    assert pc[("worker", "firm")] == 30
    V1, Gs, adj, nest = orc.cluster_variances(he, rows.gcode, codes, nlev, np.linalg.inv(B),
                                              ("region",), names, pc,
                                              extra={"region": region})["region"]
    assert Gs == [30] and sorted(nest) == ["firm", "worker"]
    assert rel(out["vcov"]["CRV1:region"], V1) < 1e-8
    V3 = adj * orc.crv3_jack(region, rows.w, H, he, B)
    assert rel(out["vcov"]["CRV3:region"], V3) < 1e-8
    with pytest.raises(ValueError):
        inference.estimate(drows, res.cells, res.gamma, fe_names=names, crv3=("firm",))


def test_wild_bootstrap_on_nested_regions_matches_oracle(device):
    """The wild cluster bootstrap by region on a device fit of 30 separate
    regions (worker and firm effects nested in them): the clusters' sums from
    the device against the oracle's, and the t statistic, every t* and the
    p-value against the oracle's bootstrap on the same draws; a bootstrap
    clustering that does not nest the effects is refused."""
    from hdfe_stream_b200 import fit, inference, wildboot
    rows, region = regions_panel()
    drows = fit.DeviceRows.from_rows(rows)
    res = fit.fit(drows, tol=1e-12)
    names = ("worker", "firm")
    est = inference.estimate(drows, res.cells, res.gamma, clusters=("region",),
                             fe_names=names, extra={"region": region}, bootcluster="region")
    boot = est["boot"]
    assert abs(boot["adj"] - est["clusters"]["region"]["adj"]) < 1e-15
    gamma = res.gamma.cpu().numpy()
    starts = orc.row_starts(rows.gcode)
    codes = np.asarray(rows.codes, np.int64)
    offs = np.concatenate(([0], np.cumsum(rows.n_levels)[:-1]))
    he, H = orc.row_scores(starts, codes, offs, rows.w, rows.V, gamma, est["beta"], with_h=True)
    AG = np.zeros((30, 2, 2))
    np.add.at(AG, region, rows.w[:, None, None] * H[:, :, None] * H[:, None, :])
    sG = np.zeros((30, 2))
    np.add.at(sG, region, he)
    assert rel(boot["AG"].cpu().numpy(), AG) < 1e-10
    assert rel(boot["sG"].cpu().numpy(), sG) < 1e-10
    for kind, null in (("rademacher", True), ("webb", False)):
        got = wildboot.wildboottest(est, 0, reps=999, weights_type=kind, impose_null=null,
                                    seed=5)
        t, tstar, p = orc.wild_bootstrap(AG, sG, est["beta"], 0, boot["adj"], 999, kind, null, 5)
        assert abs(got["t value"] - t) <= 1e-8 * abs(t)
        assert got["Pr(>|t|)"] == p and got["reps"] == 999
    with pytest.raises(ValueError):
        inference.estimate(drows, res.cells, res.gamma, fe_names=names, bootcluster="firm")


def test_saturated_model_and_single_cluster_give_nan(device):
    """core/inference.py:83-87 `_ratio`: a model with no residual degrees of
    freedom (N = K) has undefined iid and HC1 variances, and a cluster
    request with a single cluster an undefined CRV1 -- NaN, not an error."""
    from hdfe_stream_b200 import fit, inference
    from hdfe_stream_b200.simulate import Rows
    rng = np.random.default_rng(3)
    # two workers, two firms: w0 at f0, f0, f1; w1 at f0, f1.  N = 5 rows,
    # K = 2 covariates + (2 workers + 2 firms - 1) effects = 5
    gcode = np.array([0, 0, 0, 1, 1], np.uint32)
    firm = np.array([[0], [0], [1], [0], [1]], np.uint32)
    V = rng.standard_normal((5, 3))
    rows = Rows(gcode=gcode, codes=firm, V=V, w=None, n_levels=[2], n_groups=2,
                names=["y", "x1", "x2"])
    drows = fit.DeviceRows.from_rows(rows)
    res = fit.fit(drows, tol=1e-13)
    out = inference.estimate(drows, res.cells, res.gamma, clusters=("one",),
                             extra={"one": np.zeros(5, np.int64)})
    assert out["df_resid"] == 0
    assert np.isnan(out["vcov"]["iid"]).all()
    assert np.isnan(out["vcov"]["hetero"]).all()
    assert np.isfinite(out["vcov"]["CRV1"]).all()
    assert np.isnan(out["vcov"]["CRV1:one"]).all()

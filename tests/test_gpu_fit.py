"""The device fit's step 2 (components, PCG, normalisation) against the
oracle's `_solve` (pinned to the reference's): fixed effects within 1e-8
relative, component roots identical."""

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


def _panels():
    from hdfe_stream_b200.simulate import pass0_layout, simulate_panel
    out = [(n, golden_rows(load_golden(n))) for n in GOLDEN_PANELS]
    out.append(("akm_20k", pass0_layout(simulate_panel(20_000, 2_000, 10, spell=(8, 8),
                                                        p_move=0.1, seed=21))))
    out.append(("weighted", pass0_layout(simulate_panel(20_000, 1_000, 10, spell=(1, 10),
                                                         p_move=0.1, weights=True, seed=22))))
    return out


PANELS = _panels()


@pytest.mark.parametrize("name,rows", PANELS, ids=[p[0] for p in PANELS])
def test_components_match_oracle(device, name, rows):
    from hdfe_stream_b200 import fit
    ref = orc.pass1(rows)
    root_ref = orc.components(ref, 0)
    cells = fit.pass1(fit.DeviceRows.from_rows(rows))
    root, n = fit.components(cells, 0)
    assert np.array_equal(root.cpu().numpy(), root_ref)
    comp, nc = fit.rank_components(root.cpu().numpy(), ref.cnt[:ref.n_levels[0]])
    comp_ref, nc_ref = orc.component_labels(ref)
    assert nc == nc_ref == int(n.cpu().numpy()[0])
    assert np.array_equal(comp, comp_ref)


@pytest.mark.parametrize("name,rows", PANELS, ids=[p[0] for p in PANELS])
def test_fixed_effects_match_oracle(device, name, rows):
    from hdfe_stream_b200 import fit
    ref = orc.pass1(rows)
    S = orc.build_explicit(ref)
    gamma_ref, info_ref = orc.solve(ref, S, tol=1e-12)
    res = fit.fit(fit.DeviceRows.from_rows(rows), tol=1e-12)
    gamma = res.gamma.cpu().numpy()
    assert res.info["converged"]
    err = np.max(np.abs(gamma - gamma_ref)) / np.max(np.abs(gamma_ref))
    assert err < 1e-8, err
    its = np.atleast_1d(res.info["iterations"])
    assert np.all(np.abs(its - np.atleast_1d(info_ref["iterations"])) <= 1)


def test_golden_gamma(device):
    """Against the reference's own _solve output, stored in the golden file."""
    from hdfe_stream_b200 import fit
    for name in GOLDEN_PANELS:
        g = load_golden(name)
        res = fit.fit(fit.DeviceRows.from_rows(golden_rows(g)), tol=float(g["tol"]))
        gamma = res.gamma.cpu().numpy()
        err = np.max(np.abs(gamma - g["gamma"])) / np.max(np.abs(g["gamma"]))
        assert err < 1e-8, (name, err)


@pytest.mark.parametrize("name,rows", PANELS[:4], ids=[p[0] for p in PANELS[:4]])
def test_mixed_precision_fit(device, name, rows):
    """The fit with the mixed-precision solve: fixed effects within 1e-8 of
    the FP64 oracle at the same residual tolerance."""
    from hdfe_stream_b200 import fit
    ref = orc.pass1(rows)
    gamma_ref, _ = orc.solve(ref, orc.build_explicit(ref), tol=1e-13)
    res = fit.fit(fit.DeviceRows.from_rows(rows), tol=1e-11, precision="mixed")
    gamma = res.gamma.cpu().numpy()
    assert res.info["converged"]
    assert np.max(np.abs(gamma - gamma_ref)) / np.max(np.abs(gamma_ref)) < 1e-8


@pytest.mark.parametrize("panel", ["sparse", "middle", "dense", "fringe"])
@pytest.mark.parametrize("k", [1, 2])
def test_pair_components_match_reference(device, panel, k):
    """The connected set on the device (`_find_components`, min_degree core,
    labels ranked by rows) against the reference's kernels' golden output."""
    import torch
    from conftest import load_golden
    from hdfe_stream_b200.connected import pair_components
    g = load_golden("connected")
    n0, n1 = (int(x) for x in g[f"{panel}_n"])
    a = torch.as_tensor(g[f"{panel}_a"].astype(np.int32), device=device)
    b = torch.as_tensor(g[f"{panel}_b"].astype(np.int32), device=device)
    for _ in range(3):      # the same answer every time (the union-find races are benign)
        labels, rows, info = pair_components(a, b, n0, n1, (k, k))
        assert np.array_equal(labels.cpu().numpy(), g[f"{panel}_k{k}_labels"])
        assert np.array_equal(rows, g[f"{panel}_k{k}_rows"])
        assert info["pruning_rounds"] == int(g[f"{panel}_k{k}_rounds"][0])


def test_pair_components_5m_panel_matches_oracle(device):
    """The 5M-worker panel's restriction (min_degree 2, largest set) on the
    device agrees with the oracle's on a 200k-worker panel of the same shape."""
    import torch
    from hdfe_stream_b200.connected import pair_components
    from hdfe_stream_b200.simulate import pass0_layout, simulate_panel
    rows = pass0_layout(simulate_panel(200_000, 20_000, 15, spell=(5, 12), p_move=0.08, seed=3))
    a, b = rows.gcode.astype(np.uint32), rows.codes[:, 0].astype(np.uint32)
    n0, n1 = int(rows.n_groups), int(rows.n_levels[0])
    _, ref_labels, ref_rows = orc.largest_connected(a, b, n0, n1, (2, 2))
    labels, got_rows, _ = pair_components(torch.as_tensor(a.astype(np.int32), device=device),
                                          torch.as_tensor(b.astype(np.int32), device=device),
                                          n0, n1, (2, 2))
    assert np.array_equal(labels.cpu().numpy(), ref_labels)
    assert np.array_equal(got_rows, ref_rows)


@pytest.mark.parametrize("panel", ["sparse", "middle", "dense", "fringe"])
@pytest.mark.parametrize("k", [1, 2])
def test_leave_one_out_matches_reference(device, panel, k):
    """The leave-one-out connected set on the device (`_leave_one_out` after
    the (k, k) core) against the reference's own function: the levels kept
    and every count of its diagnostics."""
    import torch
    from conftest import load_golden
    from hdfe_stream_b200.connected import leave_one_out
    g = load_golden("connected")
    n0, n1 = (int(x) for x in g[f"{panel}_n"])
    a = torch.as_tensor(g[f"{panel}_a"].astype(np.int32), device=device)
    b = torch.as_tensor(g[f"{panel}_b"].astype(np.int32), device=device)
    for _ in range(3):
        alive, info = leave_one_out(a, b, n0, n1, (k, k))
        assert np.array_equal(alive.cpu().numpy(), g[f"{panel}_k{k}_loo_alive"])
        got = [info[x] for x in ("components_before", "single_observation", "cut", "rounds",
                                 "rows")]
        assert got == [int(x) for x in g[f"{panel}_k{k}_loo_counts"]]


def test_leave_one_out_random_graphs_match_oracle(device):
    """Small random bipartite networks (pendants, bridges, cut workers and
    firms, several components) against the oracle's depth-first version."""
    import torch
    from hdfe_stream_b200.connected import leave_one_out
    rng = np.random.default_rng(5)
    for trial in range(60):
        n0, n1 = int(rng.integers(2, 60)), int(rng.integers(2, 30))
        E = int(rng.integers(1, 4 * (n0 + n1)))
        a = rng.integers(0, n0, E)
        b = rng.integers(0, n1, E)
        order = np.lexsort((b, a))
        a, b = a[order].astype(np.uint32), b[order].astype(np.uint32)
        ref_alive, ref_rows, ref = orc.leave_one_out(a, b, n0, n1)
        alive, info = leave_one_out(torch.as_tensor(a.astype(np.int32), device=device),
                                    torch.as_tensor(b.astype(np.int32), device=device), n0, n1)
        assert np.array_equal(alive.cpu().numpy(), ref_alive), trial
        assert (info["cut"], info["rounds"], info["rows"]) == (ref["cut"], ref["rounds"],
                                                               ref_rows), trial


def test_leave_one_out_panel_matches_oracle(device):
    """A 200k-worker panel with short spells and few moves (many single
    observations and articulation-point movers) against the oracle."""
    import torch
    from hdfe_stream_b200.connected import leave_one_out
    from hdfe_stream_b200.simulate import pass0_layout, simulate_panel
    rows = pass0_layout(simulate_panel(200_000, 40_000, 10, spell=(1, 10), p_move=0.05, seed=8))
    a, b = rows.gcode.astype(np.uint32), rows.codes[:, 0].astype(np.uint32)
    n0, n1 = int(rows.n_groups), int(rows.n_levels[0])
    ref_alive, ref_rows, ref = orc.leave_one_out(a, b, n0, n1)
    alive, info = leave_one_out(torch.as_tensor(a.astype(np.int32), device=device),
                                torch.as_tensor(b.astype(np.int32), device=device), n0, n1)
    assert np.array_equal(alive.cpu().numpy(), ref_alive)
    assert info["rows"] == ref_rows
    assert {k: info[k] for k in ref} == ref
    assert ref["cut"] > 0 and ref["single_observation"] > 0


def test_restrict_leave_one_out_rows(device):
    """The panel restriction built on the device set keeps exactly the rows
    whose worker and firm the oracle keeps."""
    from hdfe_stream_b200.simulate import _rank_codes, restrict_leave_one_out, simulate_panel
    panel = simulate_panel(20_000, 4_000, 8, spell=(1, 8), p_move=0.05, seed=12)
    keep = restrict_leave_one_out(panel)
    a, _ = _rank_codes(panel.worker)
    b, flev = _rank_codes(panel.firm)
    n0, n1 = int(a.max()) + 1, len(flev)
    order = np.lexsort((b, a))
    alive, _, _ = orc.leave_one_out(a[order], b[order], n0, n1)
    assert np.array_equal(keep, alive[a] & alive[n0 + b.astype(np.int64)])
    assert 0 < keep.sum() < panel.n_rows


def test_pair_components_rejects_unsorted_rows(device):
    import torch
    from hdfe_stream_b200 import _lib
    from hdfe_stream_b200.connected import pair_components
    a = torch.tensor([0, 1, 0], dtype=torch.int32, device=device)
    b = torch.tensor([0, 0, 1], dtype=torch.int32, device=device)
    with pytest.raises(_lib.HDFEError):
        pair_components(a, b, 2, 2)


@pytest.mark.parametrize("name,rows", PANELS, ids=[p[0] for p in PANELS])
def test_fit_from_host_equals_device_fit(device, name, rows):
    """`fit.fit_host` (the upload overlapped with the structure-only pass 1
    and the S build) gives the same S, bit for bit, as `fit.fit` on rows
    already on the device, and the same right-hand sides and fixed effects up
    to the rounding of pass 1's atomic level sums."""
    import torch
    from hdfe_stream_b200 import fit
    pin = {"gcode": torch.from_numpy(rows.gcode.astype(np.uint32).view(np.int32)).pin_memory(),
           "codes": torch.from_numpy(np.ascontiguousarray(rows.codes.astype(np.uint32))
                                     .view(np.int32)).pin_memory(),
           "V": torch.from_numpy(np.ascontiguousarray(rows.V.T)).pin_memory()}
    w = None if rows.w is None else torch.from_numpy(rows.w.astype(np.float64)).pin_memory()
    got = fit.fit_host(pin["gcode"], pin["codes"], pin["V"], rows.n_levels, w=w, tol=1e-12)
    want = fit.fit(fit.DeviceRows.from_rows(rows), tol=1e-12)
    assert torch.equal(got.S.indptr, want.S.indptr)
    assert torch.equal(got.S.indices, want.S.indices)
    assert torch.equal(got.S.data, want.S.data)
    def rel(a, b):
        return float((a - b).abs().max() / b.abs().max())
    assert rel(got.cells.rhs, want.cells.rhs) < 1e-13
    assert torch.equal(got.cells.diag, want.cells.diag) or rel(got.cells.diag,
                                                               want.cells.diag) < 1e-13
    assert rel(got.gamma, want.gamma) < 1e-9
    its = np.atleast_1d(got.info["iterations"]) - np.atleast_1d(want.info["iterations"])
    assert np.all(np.abs(its) <= 1)


@pytest.mark.parametrize("name", ["akm_20k", "weighted"])
@pytest.mark.parametrize("batch_rows", [20_000, 57_311])
def test_fit_stream_matches_one_pass(device, name, batch_rows):
    """`fit.fit_stream` over row batches cut at group boundaries against the
    one-pass `fit.fit` of the same rows: the identifying cells and S's
    pattern identical, the level sums and S's values to rounding, the fixed
    effects within 1e-10 of the one-pass fit and 1e-8 of the oracle."""
    from hdfe_stream_b200 import fit
    rows = dict(PANELS)[name]
    batches = fit.group_batches(rows, batch_rows)
    assert sum(int(b[0].shape[0]) for b in batches) == rows.n_rows
    assert len(batches) >= rows.n_rows // batch_rows
    for a, b in zip(batches[:-1], batches[1:]):       # no group is cut
        assert int(a[0][-1]) != int(b[0][0])
    res = fit.fit_stream(batches, rows.n_levels, tol=1e-12, names=rows.names)
    one = fit.fit(fit.DeviceRows.from_rows(rows), tol=1e-12)
    assert res.info["batches"] == len(batches)
    for k in ("starts", "codes", "lcount", "work"):
        assert np.array_equal(getattr(res.cells, k).cpu().numpy(),
                              getattr(one.cells, k).cpu().numpy()), k
    assert res.cells.counts == one.cells.counts
    # weighted level sums are atomic adds: equal to rounding, not bit for bit
    for k in ("n", "group_n", "obs", "cnt", "diag", "rhs", "raw_ss"):
        a, b = getattr(res.cells, k).cpu().numpy(), getattr(one.cells, k).cpu().numpy()
        assert np.max(np.abs(a - b)) <= 1e-12 * np.max(np.abs(b)), k
    assert np.array_equal(res.S.indptr.cpu().numpy(), one.S.indptr.cpu().numpy())
    assert np.array_equal(res.S.indices.cpu().numpy(), one.S.indices.cpu().numpy())
    d, d1 = res.S.data.cpu().numpy(), one.S.data.cpu().numpy()
    assert np.max(np.abs(d - d1)) <= 1e-12 * np.max(np.abs(d1))
    g, g1 = res.gamma.cpu().numpy(), one.gamma.cpu().numpy()
    assert np.max(np.abs(g - g1)) / np.max(np.abs(g1)) < 1e-10
    ref = orc.pass1(rows)
    g_ref, _ = orc.solve(ref, orc.build_explicit(ref), tol=1e-12)
    assert np.max(np.abs(g - g_ref)) / np.max(np.abs(g_ref)) < 1e-8


@pytest.mark.parametrize("name,rows", PANELS, ids=[p[0] for p in PANELS])
def test_split_build_equals_split_of_whole_s(device, name, rows):
    """The S build in the split form (`fit.build_s_split`: the years' levels
    forced wide, their columns of the firm rows summed in direct slots) gives
    bit for bit what the whole build followed by `hdfe_small_split` gives,
    and the fit on it matches the fit on the whole S."""
    import torch
    from hdfe_stream_b200 import fit, gpu
    cells = fit.pass1(fit.DeviceRows.from_rows(rows))
    small = gpu.small_levels(cells.n_levels)
    assert small is not None
    direct = fit.build_s_split(cells, *small)
    assert direct is not None
    whole = gpu.SmallSplit(fit.build_s(cells), *small)
    for a, b in ((direct.S_big.indptr, whole.S_big.indptr),
                 (direct.S_big.indices, whole.S_big.indices),
                 (direct.S_big.data, whole.S_big.data), (direct.cross, whole.cross)):
        assert torch.equal(a, b)
    # the years' own block: when the whole build takes the years as narrow
    # rows (small panels), their entries are summed in another order
    d = float((direct.small - whole.small).abs().max() / whole.small.abs().max())
    assert d < 1e-13, d
    res = fit.fit(fit.DeviceRows.from_rows(rows), tol=1e-12)
    assert res.split is not None and res.info["small_block"]["count"] == small[1]
    plain = fit.fit(fit.DeviceRows.from_rows(rows), tol=1e-12, small_block=False)
    assert plain.split is None
    assert float((res.gamma - plain.gamma).abs().max() / plain.gamma.abs().max()) < 1e-9
    assert torch.equal(res.S.indices, plain.S.indices)       # the lazily built whole S


def test_pipelined_host_fits(device):
    """Back-to-back fits with the next rows' upload issued before this fit
    (`fit.upload_host` then `fit.fit_uploaded`), two sets of device buffers
    in turn: every fit equals its own `fit.fit_host`, whatever was in flight
    beside it."""
    import torch
    from hdfe_stream_b200 import fit

    def pin(rows):
        return (torch.from_numpy(rows.gcode.astype(np.uint32).view(np.int32)).pin_memory(),
                torch.from_numpy(np.ascontiguousarray(rows.codes.astype(np.uint32))
                                 .view(np.int32)).pin_memory(),
                torch.from_numpy(np.ascontiguousarray(rows.V.T)).pin_memory(),
                None if rows.w is None else torch.from_numpy(rows.w.astype(np.float64))
                .pin_memory())
    panels = [dict(PANELS)[n] for n in ("akm_20k", "weighted", "akm_20k", "weighted")]
    host = [pin(r) for r in panels]
    want = [fit.fit_host(g, c, V, r.n_levels, w=w, tol=1e-12).gamma.cpu()
            for (g, c, V, w), r in zip(host, panels)]
    up, prev = fit.upload_host(*host[0][:3], w=host[0][3]), None
    for i, r in enumerate(panels):
        # step i + 1 reuses step i - 1's buffers (the same panel shape)
        nxt = fit.upload_host(*host[i + 1][:3], w=host[i + 1][3], reuse=prev) \
            if i + 1 < len(panels) else None
        if i >= 1 and nxt is not None:
            assert nxt.gcode is prev.gcode
        got = fit.fit_uploaded(up, r.n_levels, tol=1e-12).gamma.cpu()
        assert float((got - want[i]).abs().max() / want[i].abs().max()) < 1e-10, i
        prev, up = up, nxt

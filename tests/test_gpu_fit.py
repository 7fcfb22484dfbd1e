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


@pytest.mark.parametrize("panel", ["sparse", "middle", "dense"])
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


def test_pair_components_rejects_unsorted_rows(device):
    import torch
    from hdfe_stream_b200 import _lib
    from hdfe_stream_b200.connected import pair_components
    a = torch.tensor([0, 1, 0], dtype=torch.int32, device=device)
    b = torch.tensor([0, 0, 1], dtype=torch.int32, device=device)
    with pytest.raises(_lib.HDFEError):
        pair_components(a, b, 2, 2)

"""Pass 0 on the device (hdfe_stream_b200.pass0): codes, row order, values and
weights identical to the host layout (`simulate.pass0_layout`) on shuffled
raw rows, with rows sharing (worker, firm, year), and a fit from them."""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def device():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch.device("cuda", 0)


@pytest.mark.parametrize("year_fe", [True, False])
def test_pass0_matches_host_layout(device, year_fe):
    import torch
    from hdfe_stream_b200 import fit, pass0
    from hdfe_stream_b200.simulate import pass0_layout, simulate_panel
    panel = simulate_panel(5_000, 500, 10, spell=(2, 10), p_move=0.1, weights=True, seed=13)
    rng = np.random.default_rng(2)
    # sparse ids, a few duplicated (worker, firm, year) rows, shuffled
    panel.worker = panel.worker * 7 + 3
    panel.firm = panel.firm * 13 + 100
    dup = rng.choice(panel.n_rows, 200, replace=False)
    for name in ("worker", "firm", "year", "log_earn", "age_squared", "age_cubed", "weight"):
        a = getattr(panel, name)
        setattr(panel, name, np.concatenate([a, a[dup]]))
    panel.log_earn[-200:] += rng.standard_normal(200)
    perm = rng.permutation(panel.n_rows)
    for name in ("worker", "firm", "year", "log_earn", "age_squared", "age_cubed", "weight"):
        setattr(panel, name, getattr(panel, name)[perm])
    ref = pass0_layout(panel, year_fe=year_fe)
    t = lambda a: torch.as_tensor(np.ascontiguousarray(a), device=device)
    V = t(np.column_stack([panel.log_earn, panel.age_squared, panel.age_cubed]))
    fes = [t(panel.firm), t(panel.year)] if year_fe else [t(panel.firm)]
    rows, levels = pass0.pass0(t(panel.worker), fes, V, t(panel.weight),
                               sort_only=() if year_fe else [t(panel.year)])
    assert np.array_equal(rows.gcode.cpu().numpy(), ref.gcode.astype(np.int32))
    assert np.array_equal(rows.codes.cpu().numpy(), ref.codes.astype(np.int32))
    assert np.array_equal(rows.V.T.cpu().numpy(), ref.V)
    assert np.array_equal(rows.w.cpu().numpy(), ref.w)
    assert rows.n_levels == list(ref.n_levels)
    assert np.array_equal(levels[1].cpu().numpy(), ref.ids["firm"])
    res = fit.fit(rows, tol=1e-12)
    ref_res = fit.fit(fit.DeviceRows.from_rows(ref), tol=1e-12)
    # the same fit (its weighted level sums are atomic, so equal to rounding)
    assert float((res.gamma - ref_res.gamma).abs().max() / ref_res.gamma.abs().max()) < 1e-10

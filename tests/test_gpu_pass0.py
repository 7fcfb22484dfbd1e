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


@pytest.mark.parametrize("n", [1, 5, 4096, 4097, 1_000_003])
def test_radix_sort_and_factorize_match_numpy(device, n):
    """hdfe_sort_pairs / hdfe_factorize (csrc/sort.cu) against numpy: the
    stable order of 64-bit keys at every bit width the tiles meet (one
    partial tile, exactly one, one plus one item, many), the rank codes and
    levels of int32, int64 and float ids with many repeats."""
    import torch
    from hdfe_stream_b200 import pass0
    rng = np.random.default_rng(n)
    for bits in (8, 13, 40, 64):
        hi = 2 ** bits
        k = rng.integers(0, min(hi, 2 ** 63), n, dtype=np.int64)
        if bits == 64:
            k = k ^ rng.integers(0, 2, n, dtype=np.int64) << 63   # the top bit too
        k[: n // 3] = k[0]                                         # long runs of one key
        ks, pos = pass0.sort_pairs(torch.as_tensor(k, device=device), None, bits)
        ref = np.argsort(k.view(np.uint64), kind="stable")
        assert np.array_equal(pos.cpu().numpy(), ref)
        assert np.array_equal(ks.cpu().numpy(), k[ref])
    vals = rng.integers(-2 ** 31, 2 ** 31 - 1, n, dtype=np.int64).astype(np.int32)
    k = rng.integers(0, 1000, n, dtype=np.int64)
    _, v = pass0.sort_pairs(torch.as_tensor(k, device=device),
                            torch.as_tensor(vals, device=device), 10)
    assert np.array_equal(v.cpu().numpy(), vals[np.argsort(k, kind="stable")])
    for ids in (rng.integers(-50, 50, n).astype(np.int32),
                rng.integers(-2 ** 62, 2 ** 62, max(n // 7, 1))[rng.integers(0, max(n // 7, 1), n)],
                np.round(rng.standard_normal(n), 2)):
        codes, levels = pass0.factorize(torch.as_tensor(ids, device=device))
        lev, inv = np.unique(ids, return_inverse=True)
        assert np.array_equal(levels.cpu().numpy(), lev)
        assert levels.dtype == torch.as_tensor(ids).dtype
        assert np.array_equal(codes.cpu().numpy(), inv)

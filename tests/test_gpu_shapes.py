"""Designs off the measured shapes, fitted on the device against the oracle:
three non-streamed dimensions, many variables (two right-hand-side blocks),
the outcome alone, and a tiny panel."""

import numpy as np
import pytest

import oracle as orc

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def device():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch.device("cuda", 0)


def rows_of(n_workers, n_firms, extra_vars=0, third_dim=False, seed=0, y_only=False,
            n_years=6, fourth_dim=False, unused=0, constant_dim=False):
    from hdfe_stream_b200.simulate import Rows, pass0_layout, simulate_panel
    panel = simulate_panel(n_workers, n_firms, n_years, spell=(min(3, n_years), n_years),
                           p_move=0.3, seed=seed)
    r = pass0_layout(panel)
    rng = np.random.default_rng(seed)
    V = r.V[:, :1] if y_only else np.column_stack(
        [r.V] + [rng.standard_normal(r.n_rows) for _ in range(extra_vars)])
    codes, n_levels = r.codes, list(r.n_levels)
    if third_dim:
        region = (r.codes[:, 0].astype(np.int64) % 5).astype(np.uint32)
        codes = np.column_stack([r.codes, region])
        n_levels = n_levels + [5]
        key = ((r.gcode.astype(np.int64) * n_levels[0] + codes[:, 0]) * n_levels[1]
               + codes[:, 1]) * 5 + codes[:, 2]
        assert np.all(np.diff(key) >= 0)          # still pass 0's order
    if fourth_dim:                              # a 3-level dimension after the regions
        band = (codes[:, 0].astype(np.int64) % 3).astype(np.uint32)
        codes = np.column_stack([codes, band])
        n_levels = n_levels + [3]
    if constant_dim:                            # a dimension of one level (every row)
        codes = np.column_stack([codes, np.zeros(len(codes), np.uint32)])
        n_levels = n_levels + [1]
    if unused:                                  # levels no row uses, after the used ones
        n_levels = [n + unused for n in n_levels]
    return Rows(gcode=r.gcode, codes=np.ascontiguousarray(codes), V=np.ascontiguousarray(V),
                w=None, n_levels=n_levels, n_groups=r.n_groups,
                names=[f"v{j}" for j in range(V.shape[1])])


CASES = ["three_dims", "many_vars", "y_only", "tiny", "one_year", "constant_dim", "four_dims",
         "unused_levels"]


@pytest.mark.parametrize("case", CASES)
def test_fit_shapes_match_oracle(device, case):
    """Every case also runs the split form of S where it applies (the
    trailing dimensions' levels, at most 16: the years; years and regions;
    years, regions and bands; years and a one-level dimension; a single
    year, where no group has two cells and S is empty; with unused
    levels)."""
    from hdfe_stream_b200 import fit
    rows = {"three_dims": lambda: rows_of(3_000, 300, third_dim=True, seed=1),
            "many_vars": lambda: rows_of(3_000, 300, extra_vars=7, seed=2),
            "y_only": lambda: rows_of(3_000, 300, y_only=True, seed=3),
            "tiny": lambda: rows_of(6, 3, seed=4),
            "one_year": lambda: rows_of(3_000, 300, n_years=1, seed=5),     # no identifying cell
            "constant_dim": lambda: rows_of(3_000, 300, constant_dim=True, seed=8),
            "four_dims": lambda: rows_of(3_000, 300, third_dim=True, fourth_dim=True, seed=6),
            "unused_levels": lambda: rows_of(3_000, 300, unused=2, seed=7)}[case]()
    res = fit.fit(fit.DeviceRows.from_rows(rows), tol=1e-12)
    c = orc.pass1(rows)
    S = orc.build_explicit(c)
    gamma, info = orc.solve(c, S, tol=1e-12)
    assert res.S.nnz == len(S[2])
    got = res.gamma.cpu().numpy()
    assert got.shape == gamma.shape
    scale = max(np.max(np.abs(gamma)), 1e-300)
    assert np.max(np.abs(got - gamma)) <= 1e-8 * scale, case

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


def rows_of(n_workers, n_firms, extra_vars=0, third_dim=False, seed=0, y_only=False):
    from hdfe_stream_b200.simulate import Rows, pass0_layout, simulate_panel
    panel = simulate_panel(n_workers, n_firms, 6, spell=(3, 6), p_move=0.3, seed=seed)
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
    return Rows(gcode=r.gcode, codes=np.ascontiguousarray(codes), V=np.ascontiguousarray(V),
                w=None, n_levels=n_levels, n_groups=r.n_groups,
                names=[f"v{j}" for j in range(V.shape[1])])


@pytest.mark.parametrize("case", ["three_dims", "many_vars", "y_only", "tiny"])
def test_fit_shapes_match_oracle(device, case):
    from hdfe_stream_b200 import fit
    rows = {"three_dims": lambda: rows_of(3_000, 300, third_dim=True, seed=1),
            "many_vars": lambda: rows_of(3_000, 300, extra_vars=7, seed=2),
            "y_only": lambda: rows_of(3_000, 300, y_only=True, seed=3),
            "tiny": lambda: rows_of(6, 3, seed=4)}[case]()
    res = fit.fit(fit.DeviceRows.from_rows(rows), tol=1e-12)
    c = orc.pass1(rows)
    S = orc.build_explicit(c)
    gamma, info = orc.solve(c, S, tol=1e-12)
    assert res.S.nnz == len(S[2])
    got = res.gamma.cpu().numpy()
    assert got.shape == gamma.shape
    scale = max(np.max(np.abs(gamma)), 1e-300)
    assert np.max(np.abs(got - gamma)) <= 1e-8 * scale, case

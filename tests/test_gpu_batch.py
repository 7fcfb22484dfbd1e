"""Many regressions in one launch (hdfe_stream_b200.batch): every system's
fixed effects and iteration count against its own single fit, for each
lanes-per-row choice, weighted and unweighted, with a zero right-hand side."""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def device():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch.device("cuda", 0)


def systems(sizes, weights=False, seed=0):
    from hdfe_stream_b200.simulate import pass0_layout, restrict_connected, simulate_panel
    out = []
    for i, n in enumerate(sizes):
        p = simulate_panel(n, max(n // 10, 5), 10, spell=(4, 10), p_move=0.1, weights=weights,
                           seed=seed + i)
        out.append(pass0_layout(p, restrict_connected(p, (1, 1))))
    return out


def rel(a, b):
    a, b = np.asarray(a, float), np.asarray(b, float)
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


@pytest.mark.parametrize("weights", [False, True])
def test_batch_matches_single_fits(device, weights):
    from hdfe_stream_b200 import batch, fit
    sys_rows = systems([2_000, 500, 8_000, 1_200, 300, 20_000], weights, seed=11)
    solver = batch.BatchSolver(batch.concat(sys_rows), tol=1e-12)
    ref = []
    for r in sys_rows:
        res = fit.fit(fit.DeviceRows.from_rows(r), tol=1e-12)
        ref.append((res.gamma.cpu().numpy(), int(np.max(np.atleast_1d(res.info["iterations"])))))
    for lanes in batch.LANE_CHOICES:
        X, info = solver.solve(lanes)
        gammas = solver.gammas(solver.normalize(X))
        assert info["converged"].all()
        for i, (g, it) in enumerate(ref):
            assert rel(gammas[i].cpu().numpy(), g) < 1e-9, (lanes, i)
            assert abs(int(info["iterations"][i]) - it) <= 1, (lanes, i)


def test_batch_tune_and_zero_column(device):
    """The tuner picks one of the choices; the systems match their own fits,
    one of them with an outcome of zeros: pass 1 over the batch centres by
    the batch's means, so that system's right-hand side is rounding noise
    rather than exactly zero and its effects come out at rounding size."""
    from hdfe_stream_b200 import batch, fit
    sys_rows = systems([3_000, 900, 5_000], seed=21)
    sys_rows[1].V[:, 0] = 0.0                 # y zero: a zero right-hand side
    solver = batch.BatchSolver(batch.concat(sys_rows), tol=1e-12)
    lanes = solver.tune()
    # lanes, then chunk length, then row cost, each shape timed once
    assert len(solver.tuning) == 8
    assert lanes in batch.LANE_CHOICES
    assert solver.shape["long_row"] in batch.LONG_ROW_CHOICES
    assert solver.shape["row_cost"] in batch.ROW_COST_CHOICES
    X, info = solver.solve()
    assert (info["lanes"], info["long_row"], info["row_cost"]) == \
        (lanes, solver.shape["long_row"], solver.shape["row_cost"])
    gammas = solver.gammas(solver.normalize(X))
    for i, r in enumerate(sys_rows):
        res = fit.fit(fit.DeviceRows.from_rows(r), tol=1e-12)
        g = res.gamma.cpu().numpy()
        cols = slice(1, None) if i == 1 else slice(None)
        assert rel(gammas[i].cpu().numpy()[:, cols], g[:, cols]) < 1e-9
    # rounding size against effects of order one (seen up to 1.01e-6)
    assert np.max(np.abs(gammas[1].cpu().numpy()[:, 0])) < 1e-5


def test_batch_matches_oracle(device):
    """Each system of a weighted batch against the oracle's own FP64 solve of
    that system alone (oracle/hdfe_oracle.c: pass 1, explicit S, Jacobi PCG,
    normalisation), with long rows cut into short chunks and a small row
    cost, so the chunked path carries most of the work."""
    import oracle as orc
    from hdfe_stream_b200 import batch
    sys_rows = systems([1_500, 4_000, 700, 9_000], weights=True, seed=31)
    solver = batch.BatchSolver(batch.concat(sys_rows), tol=1e-12)
    X, info = solver.solve(16, long_row=512, row_cost=16)
    assert info["converged"].all() and info["long_row"] == 512
    gammas = solver.gammas(solver.normalize(X))
    for i, r in enumerate(sys_rows):
        c = orc.pass1(r)
        g_ref, info_ref = orc.solve(c, orc.build_explicit(c), tol=1e-12)
        assert rel(gammas[i].cpu().numpy(), g_ref) < 1e-8, i
        assert abs(int(info["iterations"][i]) - int(info_ref["iterations"])) <= 1, i

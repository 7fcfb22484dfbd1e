"""Parity against the oracle at the benchmark's own sizes.

* The 5M-worker panel (5,000,000 workers, 500,000 firms, 15 years; 20.5M
  rows after the largest connected set with min_degree = 2): the host
  restriction that defines the benchmark's rows against the device's
  `pair_components` (core/connected.py:378-493 `_find_components`); pass 1's
  groups, cell codes and counts and S's CSR pattern bit for bit, S's values
  to 1e-10, and the fixed effects of the fit at the benchmark's own
  tolerance (1e-10) within 1e-8 of the oracle's FP64 solve at the same
  tolerance (core/solve.py:294-368 `_solve`).
* The 1M-worker panel's leave-one-out set (8.5M rows, model with the two
  covariates): one block of 32 JLA probes and one of 32 Hutchinson draws
  with the same seeds on both sides (leaveout.py:130-198, :321-448,
  :634-805): leverages, sigma2 and the three components (plug-in, bias,
  leave-out) within 1e-6 relative.

The oracle runs on all host threads: about 15 s for the fit, 30 s for the
KSS block.
"""

import os

import numpy as np
import pytest

import oracle as orc

pytestmark = [pytest.mark.gpu,
              pytest.mark.filterwarnings("ignore:Sparse:UserWarning")]


@pytest.fixture(scope="module")
def device():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    orc.set_threads(os.cpu_count() or 1)
    return torch.device("cuda", 0)


def rel(a, b):
    a, b = np.asarray(a, float), np.asarray(b, float)
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300)) if a.size else 0.0


@pytest.fixture(scope="module")
def akm_5m(device):
    from hdfe_stream_b200.simulate import PANELS, pass0_layout, restrict_connected, simulate_panel
    panel = simulate_panel(seed=0, **PANELS["akm_5m"])
    keep = restrict_connected(panel, (2, 2))
    return panel, keep, pass0_layout(panel, keep)


def test_akm_5m_restriction_matches_device_components(akm_5m):
    """The benchmark's rows: the host restriction equals the largest
    component of the device's min_degree = 2 core, row for row."""
    import torch
    from hdfe_stream_b200.connected import pair_components
    panel, keep, _ = akm_5m
    _, a = np.unique(panel.worker, return_inverse=True)
    flev, b = np.unique(panel.firm, return_inverse=True)
    n0, n1 = int(a.max()) + 1, len(flev)
    order = np.lexsort((b, a))
    dev = torch.device("cuda", 0)
    labels, rows_per, info = pair_components(
        torch.as_tensor(a[order].astype(np.int32), device=dev),
        torch.as_tensor(b[order].astype(np.int32), device=dev), n0, n1, (2, 2))
    lab = labels.cpu().numpy()
    on_device = (lab[a] == 0) & (lab[n0 + b] == 0)
    assert np.array_equal(on_device, keep)
    assert int(rows_per[0]) == int(keep.sum())


def test_akm_5m_fit_matches_oracle(akm_5m):
    from hdfe_stream_b200 import fit
    _, _, rows = akm_5m
    ref = orc.pass1(rows)
    ip, ix, dt = orc.build_explicit(ref)
    gamma_ref, info_ref = orc.solve(ref, (ip, ix, dt), tol=1e-10)

    drows = fit.DeviceRows.from_rows(rows)
    res = fit.fit(drows, tol=1e-10)
    cells = res.cells
    assert cells.counts["n_cells"] == ref.n_cells
    assert np.array_equal(cells.starts.cpu().numpy(), ref.starts)
    assert np.array_equal(cells.codes.cpu().numpy().view(np.uint32), ref.codes)
    assert np.array_equal(cells.cnt.cpu().numpy(), ref.cnt)
    assert np.array_equal(cells.n.cpu().numpy(), ref.n)
    # the level sums run over up to 1.4M cells per level, on the device in
    # another order than the oracle's sequential loop, with cancellation in
    # diag = sum n - sum u^2 / N_g: 1e-10 at this size (1e-12 on small panels)
    assert rel(cells.diag.cpu().numpy(), ref.diag) < 1e-10
    assert rel(cells.rhs.cpu().numpy(), ref.rhs) < 1e-10
    S = res.S
    assert S.nnz == len(dt)
    assert np.array_equal(S.indptr.cpu().numpy(), ip)
    assert np.array_equal(S.indices.cpu().numpy(), ix)
    # the years' rows sum over up to 1.4M cells each: 1e-10 at this size (the
    # small panels' S matches the oracle to 1e-12)
    assert rel(S.data.cpu().numpy(), dt) < 1e-10

    assert res.info["converged"] and info_ref["converged"]
    assert abs(int(res.info["iterations"]) - int(info_ref["iterations"])) <= 1
    err = rel(res.gamma.cpu().numpy(), gamma_ref)
    assert err < 1e-8, err


def test_kss_1m_block_matches_oracle(device):
    from hdfe_stream_b200 import fit, leaveout
    from hdfe_stream_b200.simulate import prepare
    rows = prepare("kss_1m", seed=100)
    drows = fit.DeviceRows.from_rows(rows)
    res = fit.fit(drows, tol=1e-10)
    op = leaveout.InverseOperator(drows, res.cells, res.S, drows.V[1:].T.contiguous(),
                                  tol=1e-10)
    got = op.leave_out_components(res, 32, block=32, seed=1)

    c = orc.pass1(rows)
    S = orc.build_explicit(c)
    gamma_ref, _ = orc.solve(c, S, tol=1e-10)
    des = orc.Design(rows, c, S, X=rows.V[:, 1:], tol=1e-10, nt=os.cpu_count() or 1)
    ref = des.leave_out_components(gamma_ref, 32, 32, 1)

    names = ("var(psi)", "var(alpha)", "cov(psi, alpha)")
    assert rel(got.leverages.leverage.cpu().numpy(), ref["leverage"]) < 1e-6
    assert rel(got.leverages.factor.cpu().numpy(), ref["factor"]) < 1e-6
    assert rel(got.diagnostics["sigma2"].cpu().numpy(), ref["sigma2"]) < 1e-6
    assert rel(got.diagnostics["beta"], ref["beta"]) < 1e-6
    for key in ("plug_in", "bias", "leave_out"):
        a = np.array([getattr(got, key)[n] for n in names])
        b = np.asarray(ref[key])
        assert np.all(np.abs(a - b) <= 1e-6 * np.abs(b)), (key, a, b)

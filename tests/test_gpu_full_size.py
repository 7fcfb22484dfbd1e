"""The path at the benchmark's full sizes, through properties that do not
depend on size, beside the oracle comparisons at the same sizes
(tests/test_gpu_full_size_parity.py):

* the 5M-worker panel (20.5M rows after pruning, L = 499,862): the solve's
  residual recomputed independently, the normalisation's zero means, the
  fit repeated (S bit for bit) and the overlapped host-input fit;
* the 1M-worker panel's leave-one-out set (8.5M rows): the KSS leave-out
  components recover the variances and covariance of the generator's true
  effects over the same rows, which they estimate without bias;
* the weighted 400k-worker panel: residual and weighted normalisation, and
  the gradients through the fit against central finite differences on 1,000
  random coordinates (weights: step 1e-6, within 1e-5).
"""

import numpy as np
import pytest

pytestmark = [pytest.mark.gpu,
              pytest.mark.filterwarnings("ignore:Sparse:UserWarning")]


@pytest.fixture(scope="module")
def device():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch.device("cuda", 0)


def residual(res):
    """max over columns of ||rhs - S gamma|| / ||rhs||, in float64 with a
    sparse product outside the library."""
    import torch
    S = res.S
    A = torch.sparse_csr_tensor(S.indptr, S.indices.to(torch.int64), S.data,
                                size=(S.L, S.L))
    r = res.cells.rhs - A @ res.gamma
    num = torch.linalg.vector_norm(r, dim=0)
    den = torch.linalg.vector_norm(res.cells.rhs, dim=0).clamp(min=1e-300)
    return float((num / den).max())


def normalisation(res):
    """The largest obs-weighted mean of the first dimension's effects within a
    component and of a further dimension's effects, relative to the effects'
    scale (core/solve.py:383-399 `_normalize` makes them zero)."""
    import torch
    from hdfe_stream_b200 import fit
    cells, gamma = res.cells, res.gamma
    offs = np.concatenate(([0], np.cumsum(cells.n_levels)[:-1]))
    root, _ = fit.components(cells, 0)
    nl0 = int(cells.n_levels[0])
    w = cells.obs[:nl0]
    comp = root.to(torch.int64)
    tot = torch.zeros((nl0, gamma.shape[1]), dtype=torch.float64, device=gamma.device)
    tot.index_add_(0, comp, w[:, None] * gamma[:nl0])
    cw = torch.zeros(nl0, dtype=torch.float64, device=gamma.device).index_add_(0, comp, w)
    worst = float((tot[cw > 0] / cw[cw > 0][:, None]).abs().max())
    for d in range(1, len(cells.n_levels)):
        o, n = int(offs[d]), int(cells.n_levels[d])
        wd = cells.obs[o:o + n]
        worst = max(worst, float(((wd @ gamma[o:o + n]) / wd.sum()).abs().max()))
    return worst / float(gamma.abs().max())


def test_akm_5m_fit_properties(device):
    import torch
    from hdfe_stream_b200 import fit
    from hdfe_stream_b200.simulate import prepare
    rows = prepare("akm_5m", seed=0)
    drows = fit.DeviceRows.from_rows(rows)
    res = fit.fit(drows, tol=1e-10)
    assert res.info["converged"] and res.info["max_rel_residual"] <= 1e-10
    assert residual(res) < 1e-8
    assert normalisation(res) < 1e-10
    again = fit.fit(drows, tol=1e-10)
    assert torch.equal(again.S.indptr, res.S.indptr)
    assert torch.equal(again.S.indices, res.S.indices)
    assert torch.equal(again.S.data, res.S.data)
    assert float((again.gamma - res.gamma).abs().max() / res.gamma.abs().max()) < 1e-9
    pin = {"g": torch.from_numpy(rows.gcode.view(np.int32)).pin_memory(),
           "c": torch.from_numpy(np.ascontiguousarray(rows.codes).view(np.int32)).pin_memory(),
           "V": torch.from_numpy(np.ascontiguousarray(rows.V.T)).pin_memory()}
    host = fit.fit_host(pin["g"], pin["c"], pin["V"], rows.n_levels, tol=1e-10)
    assert torch.equal(host.S.data, res.S.data)
    assert float((host.gamma - res.gamma).abs().max() / res.gamma.abs().max()) < 1e-9


def test_kss_1m_recovers_the_true_components(device):
    """KSS leave-out components (256 JLA probes and Hutchinson draws) against
    the variances and covariance of the generator's own worker and firm
    effects over the rows of the leave-one-out set, with the n - 1 divisor
    the estimator uses; the plug-in components, biased upward for the
    variances, are further away."""
    from hdfe_stream_b200 import fit, leaveout
    from hdfe_stream_b200.simulate import (PANELS, pass0_layout, restrict_leave_one_out,
                                           simulate_panel)
    panel = simulate_panel(seed=100, **PANELS["kss_1m"])
    keep = restrict_leave_one_out(panel)
    rows = pass0_layout(panel, keep, year_fe=False)
    psi = panel.truth["psi"][panel.firm[keep]]
    alpha = panel.truth["alpha"][panel.worker[keep]]
    n = len(psi)
    truth = np.array([np.var(psi) * n / (n - 1), np.var(alpha) * n / (n - 1),
                      np.cov(psi, alpha)[0, 1]])
    drows = fit.DeviceRows.from_rows(rows)
    res = fit.fit(drows, tol=1e-10)
    op = leaveout.InverseOperator(drows, res.cells, res.S, drows.V[1:].T.contiguous(),
                                  tol=1e-10)
    kss = op.leave_out_components(res, 256, block=32, seed=1)
    est = np.array(list(kss.leave_out.values()))
    assert np.all(np.abs(est - truth) <= 0.03 * np.abs(truth)), (est, truth)
    plug = np.array(list(kss.plug_in.values()))
    assert np.all(np.abs(est - truth)[:2] < np.abs(plug - truth)[:2])


def test_akm_400k_weighted_fit_properties(device):
    from hdfe_stream_b200 import fit
    from hdfe_stream_b200.simulate import prepare
    rows = prepare("akm_400k_w", seed=300)
    res = fit.fit(fit.DeviceRows.from_rows(rows), tol=1e-10)
    assert res.info["converged"]
    assert residual(res) < 1e-8
    assert normalisation(res) < 1e-10


def test_adjoint_400k_matches_finite_differences(device):
    """Gradients through the fit on the weighted 400k-worker panel (3.4M
    rows) -- the age_squared coefficient and the plug-in var(psi) with
    respect to y and the weights -- against central finite differences on
    1,000 random coordinates, within 1e-5: in y along random signs with a
    unit step (the objectives are linear and quadratic in y, so the
    difference is exact up to the solves' tolerance); in the weights with a
    step of 1e-6 along each objective's own gradient signs on those
    coordinates (a direction whose derivative is the sum of |g_i|, so the
    difference of the two fits stands well above their FP64 rounding: along
    random signs the derivative is ~sqrt(1000) times smaller and the
    difference at this step reaches the last digits of the fits)."""
    import torch
    from hdfe_stream_b200.adjoint import FixedEffectsSolve, plug_in_components
    from hdfe_stream_b200.simulate import prepare
    rows = prepare("akm_400k_w", seed=300)
    dev = device
    t = lambda a, dt: torch.as_tensor(np.ascontiguousarray(a), device=dev).to(dt)
    gcode, codes = t(rows.gcode.view(np.int32), torch.int32), t(rows.codes.view(np.int32),
                                                                  torch.int32)
    X = t(rows.V[:, 1:], torch.float64)
    nl = rows.n_levels

    def objectives(y, w):
        beta, gam, alpha, _ = FixedEffectsSolve.apply(y, w, gcode, codes, X, nl, 1e-13)
        return beta[0], plug_in_components(gam, alpha, w, gcode, codes, nl)[0]

    y = t(rows.V[:, 0], torch.float64).requires_grad_(True)
    w = t(rows.w, torch.float64).requires_grad_(True)
    b0, vpsi = objectives(y, w)
    grads = [torch.autograd.grad(f, (y, w), retain_graph=True) for f in (b0, vpsi)]
    rng = np.random.default_rng(17)
    idx = torch.as_tensor(rng.choice(rows.n_rows, 1_000, replace=False), device=dev)
    v = torch.zeros(rows.n_rows, dtype=torch.float64, device=dev)
    v[idx] = torch.as_tensor(rng.choice([-1.0, 1.0], 1_000), device=dev)
    y0, w0 = y.detach(), w.detach()

    def values(yy, ww):
        with torch.no_grad():
            bb, vv = objectives(yy, ww)
        return np.array([bb.item(), vv.item()])
    fd_y = (values(y0 + v, w0) - values(y0 - v, w0)) / 2.0
    h = 1e-6
    for j, (gy, gw) in enumerate(grads):
        an_y = float((gy * v).sum())
        assert abs(fd_y[j] - an_y) <= 1e-6 * abs(an_y) + 1e-14, (j, fd_y[j], an_y)
        u = torch.zeros_like(v)
        u[idx] = torch.sign(gw[idx])
        an_w = float((gw * u).sum())
        fd_w = (values(y0, w0 + h * u)[j] - values(y0, w0 - h * u)[j]) / (2 * h)
        assert abs(fd_w - an_w) <= 1e-5 * abs(an_w), (j, fd_w, an_w)

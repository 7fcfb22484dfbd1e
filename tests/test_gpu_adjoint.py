"""Gradients through the fixed-effects solve (hdfe_stream_b200.adjoint):
the age_squared coefficient and the plug-in AKM components with respect to
y and the observation weights, against (a) a dense float64 torch model of
the same regression differentiated by autograd, and (b) central finite
differences through the device fit."""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def device():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch.device("cuda", 0)


def panel_rows(n_workers, n_firms, seed):
    from hdfe_stream_b200.simulate import pass0_layout, restrict_connected, simulate_panel
    panel = simulate_panel(n_workers, n_firms, 8, spell=(3, 8), p_move=0.2, weights=True,
                           seed=seed)
    return pass0_layout(panel, restrict_connected(panel, (1, 1)))


def device_inputs(rows, device):
    import torch
    t = lambda a, dt: torch.as_tensor(np.ascontiguousarray(a), device=device).to(dt)
    gcode = t(rows.gcode.astype(np.int32), torch.int32)
    codes = t(rows.codes.astype(np.int32), torch.int32)
    y = t(rows.V[:, 0], torch.float64)
    X = t(rows.V[:, 1:], torch.float64)
    w = t(rows.w, torch.float64)
    return gcode, codes, y, X, w


def objectives(y, w, gcode, codes, X, n_levels, tol=1e-13):
    from hdfe_stream_b200.adjoint import FixedEffectsSolve, plug_in_components
    beta, gam, alpha, e = FixedEffectsSolve.apply(y, w, gcode, codes, X, n_levels, tol)
    comp = plug_in_components(gam, alpha, w, gcode, codes, n_levels)
    return beta[0], comp


def dense_objectives(rows, y, w):
    """The same weighted regression with explicit dummies (one firm and one
    year dropped for full rank), solved densely in float64 torch."""
    import torch
    N = rows.n_rows
    G, (nf, ny) = rows.n_groups, rows.n_levels
    Z = torch.zeros((N, 2 + G + (nf - 1) + (ny - 1)), dtype=torch.float64)
    Z[:, :2] = torch.as_tensor(rows.V[:, 1:])
    r = torch.arange(N)
    Z[r, 2 + torch.as_tensor(rows.gcode.astype(np.int64))] = 1.0
    f = torch.as_tensor(rows.codes[:, 0].astype(np.int64))
    yr = torch.as_tensor(rows.codes[:, 1].astype(np.int64))
    mf, my = f > 0, yr > 0
    Z[r[mf], 2 + G + f[mf] - 1] = 1.0
    Z[r[my], 2 + G + nf - 1 + yr[my] - 1] = 1.0
    ZW = Z * w[:, None]
    theta = torch.linalg.solve(ZW.T @ Z, ZW.T @ y)
    psi = torch.cat([torch.zeros(1, dtype=torch.float64), theta[2 + G:2 + G + nf - 1]])[f]
    a = theta[2:2 + G][torch.as_tensor(rows.gcode.astype(np.int64))]
    T = w.sum()
    scale = N / (N - 1.0)
    ma, mb = (w * psi).sum() / T, (w * a).sum() / T
    comp = torch.stack([scale * ((w * psi * psi).sum() / T - ma * ma),
                        scale * ((w * a * a).sum() / T - mb * mb),
                        scale * ((w * psi * a).sum() / T - ma * mb)])
    return theta[0], comp


def test_gradients_match_dense_autograd(device):
    import torch
    rows = panel_rows(300, 40, 5)
    gcode, codes, y, X, w = device_inputs(rows, device)
    y.requires_grad_(True)
    w.requires_grad_(True)
    b0, comp = objectives(y, w, gcode, codes, X, rows.n_levels)
    yc = torch.as_tensor(rows.V[:, 0]).clone().requires_grad_(True)
    wc = torch.as_tensor(rows.w).clone().requires_grad_(True)
    rb0, rcomp = dense_objectives(rows, yc, wc)
    assert abs(b0.item() - rb0.item()) < 1e-9 * abs(rb0.item())
    assert np.allclose(comp.detach().cpu().numpy(), rcomp.detach().numpy(), rtol=1e-9)
    for k, (f, rf) in enumerate([(b0, rb0)] + [(comp[j], rcomp[j]) for j in range(3)]):
        gy, gw = torch.autograd.grad(f, (y, w), retain_graph=True)
        ry, rw = torch.autograd.grad(rf, (yc, wc), retain_graph=True)
        for got, ref in ((gy, ry), (gw, rw)):
            got, ref = got.cpu().numpy(), ref.numpy()
            assert np.max(np.abs(got - ref)) <= 1e-7 * np.max(np.abs(ref)), k


def test_gradients_match_finite_differences(device):
    """Per-coordinate central differences in y (exact: the objectives are
    linear and quadratic in y) and directional ones in w, on a 2,000-worker
    panel."""
    import torch
    rows = panel_rows(2_000, 200, 7)
    gcode, codes, y, X, w = device_inputs(rows, device)
    nl = rows.n_levels
    y.requires_grad_(True)
    w.requires_grad_(True)
    b0, comp = objectives(y, w, gcode, codes, X, nl)
    rng = np.random.default_rng(3)
    idx = rng.choice(rows.n_rows, 10, replace=False)
    dirs = [torch.as_tensor(rng.choice([-1.0, 1.0], rows.n_rows), device=device)
            for _ in range(3)]
    for f_index in range(4):
        f = b0 if f_index == 0 else comp[f_index - 1]
        gy, gw = torch.autograd.grad(f, (y, w), retain_graph=True)

        def value(yy, ww):
            with torch.no_grad():
                bb, cc = objectives(yy, ww, gcode, codes, X, nl)
            return (bb if f_index == 0 else cc[f_index - 1]).item()
        y0, w0 = y.detach(), w.detach()
        fd_y, an_y = [], []
        for i in idx:
            d = torch.zeros_like(y0)
            d[int(i)] = 1.0
            fd_y.append((value(y0 + d, w0) - value(y0 - d, w0)) / 2.0)
            an_y.append(gy[int(i)].item())
        assert np.max(np.abs(np.subtract(fd_y, an_y))) <= 1e-5 * np.max(np.abs(an_y)), f_index
        h = 1e-4
        for v in dirs:
            fd = (value(y0, w0 + h * v) - value(y0, w0 - h * v)) / (2 * h)
            an = float((gw * v).sum().item())
            assert abs(fd - an) <= 1e-5 * abs(an) + 1e-12, f_index


def test_y_gradient_is_the_references_influence_output(device):
    """The reference's influence output (normal_equations.py:69-73 `predict`
    with :115-231 `solve_normal_equations`): for a right-hand side v over
    the rows, u = (Z'WZ)^- Z'v and w_i z_i'u is the derivative of the sum of
    predictions sum_i v_i yhat_i with respect to y_i.  The autograd
    y-gradient of that sum through `FixedEffectsSolve` against the oracle's
    `Design.apply_inverse` (inverse.py:311-374) of the same Z'v -- its level
    sums D_d'v, covariate sums X'v and group sums -- read out on the rows."""
    import torch
    import oracle as orc
    from hdfe_stream_b200.adjoint import FixedEffectsSolve
    rows = panel_rows(1_500, 150, 41)
    gcode, codes, y, X, w = device_inputs(rows, device)
    y.requires_grad_(True)
    nl = rows.n_levels
    beta, gam, alpha, _ = FixedEffectsSolve.apply(y, w, gcode, codes, X, nl, 1e-13)
    offs = np.concatenate(([0], np.cumsum(nl)[:-1])).astype(np.int64)
    c64 = codes.to(torch.int64)
    yhat = X @ beta + alpha[gcode.to(torch.int64)]
    for d in range(len(nl)):
        yhat = yhat + gam[int(offs[d]) + c64[:, d]]
    rng = np.random.default_rng(8)
    v = rng.standard_normal(rows.n_rows)
    (grad_y,) = torch.autograd.grad((torch.as_tensor(v, device=device) * yhat).sum(), y)

    c = orc.pass1(rows)
    des = orc.Design(rows, c, orc.build_explicit(c), X=rows.V[:, 1:], tol=1e-13)
    levels = np.concatenate([np.bincount(rows.codes[:, d].astype(np.int64), weights=v,
                                         minlength=nl[d]) for d in range(len(nl))])
    cov = rows.V[:, 1:].T @ v
    streamed = np.bincount(rows.gcode.astype(np.int64), weights=v, minlength=rows.n_groups)
    *_, zu = des.apply_inverse(levels[:, None], cov[:, None], streamed[:, None])
    influence = rows.w * zu[:, 0]
    got = grad_y.cpu().numpy()
    assert np.max(np.abs(got - influence)) <= 1e-8 * np.max(np.abs(influence))

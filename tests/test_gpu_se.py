"""KSS standard errors on the device (leaveout_se.py's `bii_rows` and
`component_variances`) against the reference's own outputs
(tests/golden/se.npz, made by tests/golden/make_se.py) and the oracle."""

import numpy as np
import pytest

import oracle as orc
from conftest import load_golden

pytestmark = pytest.mark.gpu

PANELS = ["akm_small", "akm_weighted"]


@pytest.fixture(scope="module")
def device():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch.device("cuda", 0)


def rel(a, b):
    a, b = np.asarray(a, float), np.asarray(b, float)
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def se_rows(g, name):
    from hdfe_stream_b200.simulate import Rows
    w = g[f"{name}_w"] if len(g[f"{name}_w"]) else None
    return Rows(gcode=g[f"{name}_gcode"], codes=g[f"{name}_codes_rows"], V=g[f"{name}_V"], w=w,
                n_levels=[int(x) for x in g[f"{name}_n_levels"]],
                n_groups=int(g[f"{name}_n_groups"][0]),
                names=["log_earn", "age_squared", "age_cubed"])


def standard_errors(rows, tol):
    from hdfe_stream_b200 import fit, leaveout, leaveout_se
    drows = fit.DeviceRows.from_rows(rows)
    cells = fit.pass1(drows)
    S = fit.build_s(cells)
    op = leaveout.InverseOperator(drows, cells, S, None, tol=tol)
    return leaveout_se.StandardErrors(op)


@pytest.mark.parametrize("name", PANELS)
def test_bii_rows_match_reference(device, name):
    g = load_golden("se")
    se = standard_errors(se_rows(g, name), float(g[f"{name}_tol"][0]))
    b_ii = se.bii_rows(16, block=8, seed=6).cpu().numpy()
    assert rel(b_ii, g[f"{name}_bii"]) < 1e-8


@pytest.mark.parametrize("name", PANELS)
def test_component_variances_match_reference(device, name):
    """First term, trace term, theta and V against the reference's
    `component_variances` for the same sigma2, leverages and draws."""
    g = load_golden("se")
    se = standard_errors(se_rows(g, name), float(g[f"{name}_tol"][0]))
    out = se.component_variances(g[f"{name}_sigma2"], g[f"{name}_leverage"],
                                 g[f"{name}_complement"], g[f"{name}_factor"], None, n_draws=16,
                                 block=8, seed=6)
    names = ("var(psi)", "var(alpha)", "cov(psi, alpha)")
    for key in ("first_term", "trace_term", "theta", "variance"):
        got = [out[key][n] for n in names]
        assert rel(got, g[f"{name}_{key}"]) < 1e-7, key
    assert all(np.isfinite(out["se"][n]) for n in names)


def test_smoother_matches_oracle(device):
    """The sigma2 smoother (cells in the quantile grid, bilinear evaluation)
    against the oracle's restatement on the golden rows."""
    import torch
    g = load_golden("se")
    name = "akm_weighted"
    se = standard_errors(se_rows(g, name), float(g[f"{name}_tol"][0]))
    s2, lev, b = g[f"{name}_sigma2"], g[f"{name}_leverage"], g[f"{name}_bii"][1]
    for bins in (None, 3, 7):
        got = se.smooth(torch.as_tensor(s2, device=device), torch.as_tensor(lev, device=device),
                        torch.as_tensor(b, device=device), bins).cpu().numpy()
        ref = orc.smooth_eval(orc.fit_smoother(s2, lev, b, bins), lev, b)
        assert rel(got, ref) < 1e-12


def test_match_level_kernel_matches_reference(device):
    """The match level's options (stayers' b zeroed, the reference-centred
    kernel with the rank-two term, var(alpha) unreported) against the
    reference's `component_variances` for the same sigma2, leverages and
    draws (tests/golden/match_se.npz)."""
    g = load_golden("match_se")
    ref = {f"r_{k[4:]}": v for k, v in g.items() if k.startswith("ref_")}
    ref["r_w"] = np.zeros(0)
    se = standard_errors(se_rows(ref, "r"), float(ref["r_tol"][0]))
    out = se.component_variances(ref["r_sigma2"], ref["r_leverage"], ref["r_complement"],
                                 ref["r_factor"], None, n_draws=16, block=8, seed=6,
                                 stayer_rows=ref["r_stayer"], centering="reference",
                                 reported=(0, 2))
    for key in ("first_term", "trace_term", "theta", "variance"):
        got = [out[key][n] for n in ("var(psi)", "cov(psi, alpha)")]
        assert rel(got, ref[f"r_{key}"][[0, 2]]) < 1e-7, key
        assert np.isnan(out[key]["var(alpha)"])

"""Steps 3-4 of a fit on the device: beta and its variances.

core/inference.py:833-912 `_estimate` for OLS: V' W V of the residualised
variables (`hdfe_resid_moments`, the row assembly of `_assemble`), beta =
A[x, x] \\ A[x, y], then one row pass (`hdfe_variance_sums`, `_nb_pass2` with
the sums of :566-578) for the bread, the heteroskedastic meat, the meat of the
scores clustered on the streamed dimension and the residual sum of squares,
and the iid, HC1 and CRV1 variances with pyfixest's small-sample factors
(:886-912).  The fixed-effect parameter count is core/estimator.py:446-464
`_k_fe` with fe_dof "exact": the levels of every dimension less the
components of the pair of dimensions with the most, less one per further
non-streamed dimension; for CRV1 on the streamed dimension its levels, which
are nested in their own clusters, count as one.  The pairs' components come
from the device: the streamed dimension against each other one from the
identifying cells' union-find (`fit.components`), two non-streamed dimensions
from their distinct code pairs (`connected.pair_components`).
"""

from __future__ import annotations

import numpy as np

from . import _lib
from .connected import pair_components
from .fit import DeviceCells, DeviceRows, components


def _torch():
    import torch
    return torch


def row_groups(rows: DeviceRows):
    """(starts (G+1) int64 device tensor, G): the runs of equal gcode."""
    torch = _torch()
    lib = _lib.lib()
    dev = rows.gcode.device
    N = rows.n_rows
    starts = torch.empty(N + 1, dtype=torch.int64, device=dev)
    ng = torch.zeros(1, dtype=torch.int64, device=dev)
    ws = torch.empty(int(lib.hdfe_row_groups_workspace_bytes(N)), dtype=torch.uint8, device=dev)
    _lib.check(lib.hdfe_row_groups(rows.gcode.data_ptr(), N, starts.data_ptr(), ng.data_ptr(),
                                   ws.data_ptr(), ws.numel(), _lib.stream_handle()))
    G = int(ng.item())
    return starts[:G + 1], G


def fe_pair_components(rows: DeviceRows, cells: DeviceCells):
    """Components of every pair of fixed-effect dimensions (the streamed one
    with each other, then the other pairs), as core/passes.py's pass 1
    collects them for the degrees of freedom."""
    torch = _torch()
    D = rows.D
    counts = []
    for d in range(D):
        _, out = components(cells, d)
        counts.append(int(out[0].item()))
    nl = [int(x) for x in rows.n_levels]
    for d1 in range(D):
        for d2 in range(d1 + 1, D):
            c1 = rows.codes[:, d1].to(torch.int64)
            c2 = rows.codes[:, d2].to(torch.int64)
            keys = torch.unique(c1 * nl[d2] + c2)
            a = (keys // nl[d2]).to(torch.int32).contiguous()
            b = (keys % nl[d2]).to(torch.int32).contiguous()
            _, _, info = pair_components(a, b, nl[d1], nl[d2])
            counts.append(int(info["components"]))
    return counts


def estimate(rows: DeviceRows, cells: DeviceCells, gamma):
    """beta (k,) and its variances for y = V[0] on X = V[1:] with the fit's
    normalised effects gamma (L, m): {"beta", "vcov": {"iid", "hetero",
    "CRV1"}, "se": {...}, "k_fe", "df_resid", "df_cluster", "rss",
    "pair_components", "n_obs", "n_groups"}; CRV1 clusters on the streamed
    dimension."""
    torch = _torch()
    lib = _lib.lib()
    m = rows.m
    if m < 2:
        raise ValueError("estimate needs at least one covariate")
    dev = rows.gcode.device
    starts, G = row_groups(rows)
    nlev = np.asarray(rows.n_levels, dtype=np.int64)
    gamma = gamma.to(dev, torch.float64).contiguous()
    status = torch.zeros(1, dtype=torch.int32, device=dev)
    w = rows.w
    base = (starts.data_ptr(), G, rows.codes.data_ptr(), len(nlev), nlev.ctypes.data,
            None if w is None else w.data_ptr(), rows.V.data_ptr(), m, rows.n_rows)
    A = torch.empty((m, m), dtype=torch.float64, device=dev)
    ws = torch.empty(int(lib.hdfe_assemble_workspace_bytes(m)), dtype=torch.uint8, device=dev)
    _lib.check(lib.hdfe_resid_moments(*base, gamma.data_ptr(), A.data_ptr(), ws.data_ptr(),
                                      ws.numel(), status.data_ptr(), _lib.stream_handle()))
    A = A.cpu().numpy()
    beta = np.linalg.solve(A[1:, 1:], A[1:, 0])
    k = m - 1
    T = k * (k + 1) // 2
    beta_d = torch.as_tensor(beta, dtype=torch.float64, device=dev)
    sums = torch.empty(3 * T + 1, dtype=torch.float64, device=dev)
    ws2 = torch.empty(int(lib.hdfe_variance_sums_workspace_bytes(m)), dtype=torch.uint8,
                      device=dev)
    _lib.check(lib.hdfe_variance_sums(*base, gamma.data_ptr(), beta_d.data_ptr(),
                                      sums.data_ptr(), ws2.data_ptr(), ws2.numel(),
                                      status.data_ptr(), _lib.stream_handle()))
    s = sums.cpu().numpy()
    if int(status.item()) != _lib.HDFE_OK:
        raise _lib.HDFEError(int(status.item()), "estimate: a level code is out of range")
    iu = np.triu_indices(k)

    def sym(v):
        out = np.zeros((k, k))
        out[iu] = v
        return out + np.triu(out, 1).T
    B, meat_hc, meat_g, rss = sym(s[:T]), sym(s[T:2 * T]), sym(s[2 * T:3 * T]), float(s[3 * T])
    pcs = fe_pair_components(rows, cells)
    N = float(rows.n_rows)
    k_fe = G + int(nlev.sum()) - (max(pcs) + len(nlev) - 1)
    K = k + k_fe
    Binv = np.linalg.inv(B)
    Kc = k + k_fe - G + 1
    adj = G / (G - 1) * (N - 1) / (N - Kc)
    vcov = {"iid": rss / (N - K) * Binv, "hetero": N / (N - K) * Binv @ meat_hc @ Binv,
            "CRV1": adj * Binv @ meat_g @ Binv}
    return {"beta": beta, "vcov": vcov,
            "se": {key: np.sqrt(np.diag(v)) for key, v in vcov.items()},
            "k_fe": k_fe, "df_resid": N - K, "df_cluster": G - 1, "rss": rss,
            "pair_components": pcs, "n_obs": int(N), "n_groups": G}

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


def ratio(num, den):
    """num / den, or nan when den is zero (core/inference.py:83-87 `_ratio`):
    a saturated model or a request with a single cluster has no degrees of
    freedom left, so its variances are undefined rather than an error."""
    return num / den if den else np.nan


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


def row_scores(rows: DeviceRows, cells: DeviceCells, gamma, beta, with_h=False):
    """The per-row scores w e h (N, m - 1) of pass 2 (`hdfe_row_scores`);
    with_h: also the residualised covariates h, as (scores, h)."""
    torch = _torch()
    lib = _lib.lib()
    dev = rows.gcode.device
    starts, G = row_groups(rows)
    nlev = np.asarray(rows.n_levels, dtype=np.int64)
    gamma = gamma.to(dev, torch.float64).contiguous()
    beta_d = torch.as_tensor(np.asarray(beta, np.float64), device=dev)
    out = torch.empty((rows.n_rows, rows.m - 1), dtype=torch.float64, device=dev)
    h = torch.empty_like(out) if with_h else None
    status = torch.zeros(1, dtype=torch.int32, device=dev)
    w = rows.w
    _lib.check(lib.hdfe_row_scores(starts.data_ptr(), G, rows.codes.data_ptr(), len(nlev),
                                   nlev.ctypes.data, None if w is None else w.data_ptr(),
                                   rows.V.data_ptr(), rows.m, rows.n_rows, gamma.data_ptr(),
                                   beta_d.data_ptr(), out.data_ptr(),
                                   None if h is None else h.data_ptr(), status.data_ptr(),
                                   _lib.stream_handle()))
    if int(status.item()) != _lib.HDFE_OK:
        raise _lib.HDFEError(int(status.item()), "row_scores: a level code is out of range")
    return (out, h) if with_h else out


def cluster_vcov(rows: DeviceRows, scores, Binv, k, requests, fe_names, pair_components,
                 group_meat=None, extra=None, crv3=(), h=None, B=None, boot=None):
    """CRV1 variances for cluster requests (core/inference.py:176-240
    `_resolve_clusters`, :242-269 `_nested_dims`, :886-906): a request "a",
    "a^b" (one cluster per distinct combination) or "a+b" (two-way,
    inclusion-exclusion over a, b and a^b); the names are `fe_names` (the
    streamed dimension first, then the others in column order) or keys of
    `extra` (per-row integer codes).  Each term's meat sums the scores per
    cluster (a device index_add over the cluster codes found by a sort of the
    combined keys) and takes S'S; a fixed-effect dimension is nested in a
    term when its columns are among the term's or (except for a refinement of
    the streamed groups) every level lies within one cluster; K drops the
    nested dimensions' levels (core/estimator.py:446-464 `_k_fe` with the
    pairs whose both dimensions are nested left out); G is the smallest
    one-way count.  Returns {request: (V, {"G", "adj", "nested"})}.

    `crv3` lists one-way requests that also get the cluster jackknife
    (core/inference.py:270-298, core/kernels_base.py:620-680): leaving
    cluster g out moves beta by -(B - A_g)^+ s_g, with A_g the cluster's sum
    of w h h' and s_g its sum of w e h, so CRV3 = adj sum_g d_g d_g' (the
    CRV1 factor), from h (N, k) and the bread B; every fixed-effect dimension
    must be nested in the clusters (else ValueError).  Its entries come back
    under "CRV3:<request>".  `boot`, a one-way request with the same nesting
    and not a refinement of the streamed groups (core/inference.py:312-330),
    keeps its clusters' sums for the wild bootstrap under "BOOT:<request>":
    ({"AG", "sG", "adj", "cluster"}, info)."""
    torch = _torch()
    from itertools import combinations
    dev = rows.gcode.device
    N = rows.n_rows
    D = rows.D
    g0 = fe_names[0]
    col = {g0: rows.gcode.to(torch.int64)}
    for d in range(D):
        col[fe_names[d + 1]] = rows.codes[:, d].to(torch.int64)
    for name, c in (extra or {}).items():
        col[name] = torch.as_tensor(c, device=dev).to(torch.int64)
    card = {name: int(c.max().item()) + 1 if N else 0 for name, c in col.items()}
    G_groups = int(rows.gcode[-1].item()) + 1 if N else 0
    fe_params = {g0: G_groups}
    for d in range(D):
        fe_params[fe_names[d + 1]] = int(rows.n_levels[d])
    fe_dims = list(fe_params)
    cache = {}

    def term(cols):
        key_name = "^".join(cols)
        if key_name in cache:
            return cache[key_name]
        cs = set(cols)
        if cs == {g0}:
            kind, code, G = "seg", col[g0], G_groups
        elif len(cols) == 1 and cols[0] in fe_params:
            kind, code, G = "fe", col[cols[0]], card[cols[0]]
        else:
            # compose the clusters column by column, re-coding densely after
            # each step, so the packed key never exceeds (distinct so far) x
            # card[c] < 2^63 whatever the columns' cardinalities
            code, G = None, 1
            for c in cols:
                if G * max(card[c], 1) >= 2 ** 63:
                    raise ValueError(f"cluster request {'^'.join(cols)!r}: too many clusters")
                key = col[c] if code is None else code * card[c] + col[c]
                _, code = torch.unique(key, sorted=True, return_inverse=True)
                G = int(code.max().item()) + 1 if N else 0
            kind = "segsub" if g0 in cs else ("fe" if len(cols) == 1 else "extra")
        S = None
        if kind == "seg" and group_meat is not None and key_name not in crv3_terms:
            meat = group_meat
        else:
            S = torch.zeros((G, k), dtype=torch.float64, device=dev).index_add_(0, code, scores)
            meat = (S.T @ S).cpu().numpy()
        nested = []
        for d in fe_dims:
            if cs <= {d}:
                nested.append(d)
                continue
            if kind == "segsub":
                continue
            nl = fe_params[d]
            lo = torch.full((nl,), N, dtype=torch.int64, device=dev).scatter_reduce_(
                0, col[d], code, "amin")
            hi = torch.full((nl,), -1, dtype=torch.int64, device=dev).scatter_reduce_(
                0, col[d], code, "amax")
            if bool((lo == hi).all().item()):
                nested.append(d)
        cache[key_name] = (G, meat, nested, code, S)
        return cache[key_name]

    def k_fe(nest):
        total = sum(fe_params.values())
        if len(fe_params) < 2:
            return total
        comps = max((c for (a, b), c in pair_components.items()
                     if a not in nest or b not in nest), default=1)
        return total - (comps + len(fe_params) - 2)

    crv3_terms = set()
    for req in list(crv3) + ([boot] if boot else []):
        if "+" in req:
            raise ValueError(f"CRV3 takes a one-way cluster request, not {req!r}")
        crv3_terms.add("^".join(dict.fromkeys(c.strip() for c in req.split("^"))))
    out = {}
    for req in list(dict.fromkeys(list(requests) + list(crv3) + ([boot] if boot else []))):
        parts = [[c.strip() for c in p.split("^")] for p in req.split("+")]
        terms = []
        for r in range(1, len(parts) + 1):
            for combo in combinations(range(len(parts)), r):
                cols = list(dict.fromkeys(c for i in combo for c in parts[i]))
                terms.append((term(cols), (-1) ** (r + 1), r == 1))
        Gs = [t[0] for t, _, single in terms if single]
        Gm = min(Gs)
        nest = list(dict.fromkeys(d for t, _, _ in terms for d in t[2]))
        Kc = k + k_fe(nest) - sum(fe_params[d] for d in nest) + len(nest)
        adj = ratio(Gm, Gm - 1) * ratio(N - 1, N - Kc)
        V = sum(sign * adj * (Binv @ t[1] @ Binv) for t, sign, _ in terms)
        out[req] = (V, {"G": Gs, "adj": adj, "nested": nest, "df": Gm - 1})
        if req == boot:
            (t, _, _), = terms
            loose = [d for d in fe_dims if d not in t[2]]
            if loose or g0 in [c for part in parts for c in part] and len(parts[0]) > 1:
                raise ValueError(
                    f"the wild cluster bootstrap by {req!r} needs every fixed effect nested "
                    "within clusters that are not a refinement of the streamed groups")
            if h is None:
                raise ValueError("the bootstrap sums need the residualised covariates h")
            G, _, _, code, S = t
            out["BOOT:" + req] = ({"AG": cluster_sums(code, G, rows.w, h), "sG": S, "adj": adj,
                                   "cluster": req}, {"G": Gs, "adj": adj, "nested": nest,
                                                     "df": Gm - 1})
        if req in crv3:
            (t, _, _), = terms
            loose = [d for d in fe_dims if d not in t[2]]
            if loose:
                raise ValueError(
                    f"CRV3 standard errors need every fixed effect to be nested within the "
                    f"clusters, and {', '.join(map(repr, loose))} "
                    f"{'is' if len(loose) == 1 else 'are'} not nested within {req!r}; "
                    "only CRV1 is supported there")
            if h is None or B is None:
                raise ValueError("CRV3 needs the residualised covariates h and the bread B")
            G, _, _, code, S = t
            jack = crv3_jack(code, G, rows.w, h, S, B)
            out["CRV3:" + req] = (adj * jack, {"G": Gs, "adj": adj, "nested": nest,
                                               "df": Gm - 1})
    return out


def cluster_sums(code, G, w, h):
    """A_g = sum over the cluster's rows of w h h' (G, k, k), by a device
    index-add (core/kernels_base.py:658-670 `_nb_crv3_scatter`)."""
    torch = _torch()
    N, k = h.shape
    dev = h.device
    w = w if w is not None else torch.ones(N, dtype=torch.float64, device=dev)
    outer = (w[:, None, None] * h[:, :, None] * h[:, None, :]).reshape(N, k * k)
    return torch.zeros((G, k * k), dtype=torch.float64, device=dev).index_add_(
        0, code, outer).reshape(G, k, k)


def crv3_jack(code, G, w, h, S, B):
    """sum over clusters of d_g d_g', d_g = (B - A_g)^+ s_g (core/kernels_base.py:
    658-680 `_nb_crv3_scatter` / `_nb_crv3_finish`): code (N,) cluster ids, w
    (N,) or None, h (N, k) the residualised covariates, S (G, k) the clusters'
    sums of w e h, B the bread; A_g by a device index-add of w h h', the
    pseudo-inverses batched on the device."""
    torch = _torch()
    AG = cluster_sums(code, G, w, h)
    Bd = torch.as_tensor(np.asarray(B, np.float64), device=h.device)
    d = (torch.linalg.pinv(Bd[None] - AG) @ S[:, :, None])[:, :, 0]
    return (d.T @ d).cpu().numpy()


def estimate(rows: DeviceRows, cells: DeviceCells, gamma, clusters=(), fe_names=None,
             extra=None, crv3=(), bootcluster=None):
    """beta (k,) and its variances for y = V[0] on X = V[1:] with the fit's
    normalised effects gamma (L, m): {"beta", "vcov": {"iid", "hetero",
    "CRV1", "CRV1:<request>" ...}, "se": {...}, "k_fe", "df_resid",
    "df_cluster", "rss", "pair_components", "n_obs", "n_groups"}; "CRV1"
    clusters on the streamed dimension; `clusters` adds the requests of
    `cluster_vcov` (names from `fe_names`, default "fe0" for the streamed
    dimension and "fe1", "fe2", ... for the others, or from `extra`); `crv3`
    one-way requests that also get the cluster jackknife ("CRV3:<request>");
    `bootcluster` a one-way request whose clusters' sums are kept as
    "boot" for `wildboot.wildboottest`."""
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
    adj = ratio(G, G - 1) * ratio(N - 1, N - Kc)
    vcov = {"iid": ratio(rss, N - K) * Binv, "hetero": ratio(N, N - K) * Binv @ meat_hc @ Binv,
            "CRV1": adj * Binv @ meat_g @ Binv}
    cluster_info = {}
    boot = None
    if clusters or crv3 or bootcluster:
        names = list(fe_names) if fe_names else [f"fe{d}" for d in range(len(nlev) + 1)]
        D = len(nlev)
        pair = {}
        for d in range(D):
            pair[(names[0], names[d + 1])] = pcs[d]
        j = D
        for d1 in range(D):
            for d2 in range(d1 + 1, D):
                pair[(names[d1 + 1], names[d2 + 1])] = pcs[j]
                j += 1
        if crv3 or bootcluster:
            scores, h = row_scores(rows, cells, gamma, beta, with_h=True)
        else:
            scores, h = row_scores(rows, cells, gamma, beta), None
        for req, (V, info) in cluster_vcov(rows, scores, Binv, k, clusters, names, pair,
                                           group_meat=meat_g, extra=extra, crv3=crv3, h=h,
                                           B=B, boot=bootcluster).items():
            if req.startswith("BOOT:"):
                boot = V
                continue
            key = req if req.startswith("CRV3:") else f"CRV1:{req}"
            vcov[key] = V
            cluster_info[req] = info
    return {"beta": beta, "vcov": vcov,
            "se": {key: np.sqrt(np.diag(v)) for key, v in vcov.items()},
            "k_fe": k_fe, "df_resid": N - K, "df_cluster": G - 1, "rss": rss,
            "pair_components": pcs, "n_obs": int(N), "n_groups": G, "clusters": cluster_info,
            "boot": boot}

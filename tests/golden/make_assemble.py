"""Golden vectors for steps 3-4 of a fit (what the KSS components read from
the residual file), made by the reference's own kernels.

Run once, in a container where the reference tree is readable:

    python tests/golden/make_assemble.py /path/to/hdfe-stream

For each golden panel (tests/golden/<panel>.npz: its rows and the
reference's normalised Gamma), it runs core/kernels_base.py
`_nb_residualize_rows` and forms V' W V as core/inference.py:109-135
`_assemble` does, solves for beta as :874 does (A[xk, xk] \\ A[xk, y]), and
runs `_nb_pass2` (:544) with gam_y = Gamma_y - Gamma_x beta (:454-456) for the
residuals and the streamed effect; the non-streamed effect per row is
gam_y[level] (:615).  With the kernel's group scores (sum over a group of
w e z~) it forms the pass's sums as core/inference.py:566-578 does -- the
bread sum w h h', the heteroskedastic meat sum (w e)^2 h h', the meat of
scores clustered on the streamed dimension, the residual sum of squares --
and the iid, HC1 and CRV1(streamed dimension) variances with the small-sample
factors of :886-912 and the fixed-effect parameter count of
core/estimator.py:446-464 (fe_dof "exact"; the streamed dimension's levels
nested in its own clusters).  It also keeps the per-row scores w e z~ and,
for the CRV1 requests in REQUESTS (another dimension, two-way, a refinement
of the streamed groups, two-way over the non-streamed dimensions), the
variances of :886-906 with each term's meat from the reference's own scatter
(core/utils.py `_scatter`) and its nested dimensions (:242-269).  Outputs go
to tests/golden/assemble.npz.
Nothing at test time reads the reference.
"""

from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE))

from make_golden import import_reference  # noqa: E402

PANELS = ("akm_small", "akm_weighted", "akm_components")
# CRV1 requests beyond the streamed dimension: one-way on another dimension,
# two-way with inclusion-exclusion, a refinement of the streamed groups
# ("segsub") and two-way over the non-streamed dimensions (their intersection
# an "extra" cluster)
REQUESTS = ("firm", "worker+firm", "worker^firm", "firm+year")
DIMS = ("worker", "firm", "year")


def cluster_variances(utils, gcode, codes, nlev, G, he, meat_g, Binv, k, N, pc):
    """core/inference.py:176-240 `_resolve_clusters`, :242-269
    `_nested_dims`, :597-606 and :656-658 (the meats), :886-906 (the CRV1
    variances) and core/estimator.py:446-464 `_k_fe` (fe_dof "exact") for
    REQUESTS, on the reference's own pass-2 scores `he` and group scores."""
    from itertools import combinations
    col = {"worker": gcode.astype(np.int64), "firm": codes[:, 0], "year": codes[:, 1]}
    card = {"worker": G, "firm": int(nlev[0]), "year": int(nlev[1])}
    fe_params = {"worker": G, "firm": int(nlev[0]), "year": int(nlev[1])}

    def term(cols):
        cs = set(cols)
        if cs == {"worker"}:
            return {"kind": "seg", "code": col["worker"], "G": G, "meat": meat_g}
        key = np.zeros(N, np.int64)
        for c in cols:
            key = key * card[c] + col[c]
        if len(cols) == 1:
            code, Gt = col[cols[0]], card[cols[0]]
            kind = "fe"
        else:
            _, code = np.unique(key, return_inverse=True)
            Gt = int(code.max()) + 1
            kind = "segsub" if "worker" in cs else "extra"
        S = utils._scatter(code.astype(np.int64), he, Gt)
        return {"kind": kind, "code": code, "G": Gt, "meat": S.T @ S}

    def nested(t, cols):
        out = []
        for d in DIMS:
            if set(cols) <= {d}:
                out.append(d)
                continue
            if t["kind"] == "segsub":
                continue
            lo = np.full(card[d], np.iinfo(np.int64).max)
            hi = np.full(card[d], -1)
            np.minimum.at(lo, col[d], t["code"])
            np.maximum.at(hi, col[d], t["code"])
            if np.all(lo == hi):
                out.append(d)
        return out

    def k_fe(nest):
        comps = max((c for (a, b), c in pc.items() if a not in nest or b not in nest),
                    default=1)
        return sum(fe_params.values()) - (comps + len(DIMS) - 2)

    out = {}
    for req in REQUESTS:
        parts = [[c.strip() for c in p_.split("^")] for p_ in req.split("+")]
        terms = []
        for r in range(1, len(parts) + 1):
            for combo in combinations(range(len(parts)), r):
                cols = list(dict.fromkeys(c for i in combo for c in parts[i]))
                t = term(cols)
                terms.append((t, (-1) ** (r + 1), r == 1, nested(t, cols)))
        Gm = min(t["G"] for t, _, single, _ in terms if single)
        nest = list(dict.fromkeys(d for *_, nd in terms for d in nd))
        Kc = k + k_fe(nest) - sum(fe_params[d] for d in nest) + len(nest)
        adj = Gm / (Gm - 1) * (N - 1) / (N - Kc)
        out[req] = {"V": sum(sign * adj * (Binv @ t["meat"] @ Binv) for t, sign, _, _ in terms),
                    "G": [t["G"] for t, _, single, _ in terms if single], "adj": adj,
                    "nested": nest}
    return out


def main(root):
    kb = import_reference(root)["core.kernels_base"]
    import importlib
    utils = importlib.import_module("hdfe_stream.core.utils")
    out = {}
    for name in PANELS:
        g = np.load(HERE / f"{name}.npz")
        gcode = g["gcode"]
        codes = np.ascontiguousarray(g["codes_rows"], dtype=np.int64)
        V = np.ascontiguousarray(g["V"], dtype=np.float64)
        N, m = V.shape
        w = g["w"] if len(g["w"]) else np.ones(N)
        w = np.ascontiguousarray(w, dtype=np.float64)
        nlev = np.asarray(g["n_levels"], dtype=np.int64)
        offs = np.concatenate(([0], np.cumsum(nlev)[:-1])).astype(np.int64)
        starts = np.concatenate(([0], np.flatnonzero(gcode[1:] != gcode[:-1]) + 1, [N]))
        starts = starts.astype(np.int64)
        Gamma = np.ascontiguousarray(g["gamma"], dtype=np.float64)
        Vr = V.copy()
        kb._nb_residualize_rows(starts, codes, offs, w, Vr, Gamma, True, 4)
        Vs = Vr * np.sqrt(w)[:, None]
        A = Vs.T @ Vs
        yj, xk = 0, list(range(1, m))
        beta = np.linalg.solve(A[np.ix_(xk, xk)], A[xk, yj])
        gam_x = Gamma[:, xk]
        gam_y0 = np.ascontiguousarray(Gamma[:, yj])
        gam_y = np.ascontiguousarray(gam_y0 - gam_x @ beta)
        y = np.ascontiguousarray(V[:, yj])
        X = np.ascontiguousarray(V[:, xk])
        G = len(starts) - 1
        e = np.empty(N)
        zt = np.empty((N, len(xk)))
        g_eff = np.empty(G)
        acc_s = np.zeros((4, 4))
        k = len(xk)
        sg = np.empty((G, k))
        kb._nb_pass2(starts, codes, offs, w, y, X, beta, gam_y, gam_y0, X,
                     np.ascontiguousarray(gam_x), float(g["means"][yj]), True, g_eff, e, zt,
                     sg, acc_s)
        # inference.py:566-578 (analytic weights, OLS: h = z~)
        sw = np.sqrt(w)
        B = (zt * sw[:, None]).T @ (zt * sw[:, None])
        he = zt * (w * e)[:, None]
        meat_hc = he.T @ he
        meat_g = sg.T @ sg
        rss = float(acc_s[:, 0].sum())
        # estimator.py:446-464: fixed-effect parameters net of the redundant
        n_o = len(nlev)
        fe_params = [G] + [int(x) for x in nlev]
        comps = max(int(x) for x in g["pair_components"])
        k_fe = sum(fe_params) - (comps + n_o - 1)
        K = k + k_fe
        Binv = np.linalg.inv(B)
        V_iid = rss / (N - K) * Binv
        V_hc1 = N / (N - K) * Binv @ meat_hc @ Binv
        Kc = k + k_fe - G + 1
        adj = G / (G - 1) * (N - 1) / (N - Kc)
        V_crv1 = adj * Binv @ meat_g @ Binv
        out[f"{name}_B"] = B
        out[f"{name}_meat_hc"] = meat_hc
        out[f"{name}_meat_g"] = meat_g
        out[f"{name}_rss"] = np.array([rss])
        out[f"{name}_k_fe"] = np.array([k_fe])
        out[f"{name}_V_iid"] = V_iid
        out[f"{name}_V_hc1"] = V_hc1
        out[f"{name}_V_crv1"] = V_crv1
        out[f"{name}_A"] = A
        out[f"{name}_beta"] = beta
        out[f"{name}_gam_y"] = gam_y
        out[f"{name}_resid"] = e
        out[f"{name}_alpha"] = g_eff
        out[f"{name}_psi"] = gam_y[offs[0] + codes[:, 0]]
        out[f"{name}_scores"] = he
        # the CRV3 jackknife sums of core/kernels_base.py:620-680 (the kernels
        # alone: whether the request is valid is the caller's check)
        nt = 4
        acc = np.zeros((nt, k, k))
        kb._nb_crv3_groups(starts, w, e, np.ascontiguousarray(zt), B, acc)
        out[f"{name}_crv3_worker_jack"] = acc.sum(axis=0)
        nf = int(nlev[0])
        AG, sG = np.zeros((nf, k, k)), np.zeros((nf, k))
        kb._nb_crv3_scatter(codes[:, 0].astype(np.int64), w, e, np.ascontiguousarray(zt), AG, sG)
        acc = np.zeros((nt, k, k))
        kb._nb_crv3_finish(B, AG, sG, acc)
        out[f"{name}_crv3_firm_jack"] = acc.sum(axis=0)
        pcs = [int(x) for x in g["pair_components"]]      # sorted keys of the pairs
        pc = {("firm", "year"): pcs[0], ("worker", "firm"): pcs[1], ("worker", "year"): pcs[2]}
        for req, res in cluster_variances(utils, gcode, codes, nlev, G, he, meat_g, Binv, k, N,
                                          pc).items():
            out[f"{name}_crv1_{req}_V"] = res["V"]
            out[f"{name}_crv1_{req}_G"] = np.array(res["G"])
            out[f"{name}_crv1_{req}_adj"] = np.array([res["adj"]])
            print(name, req, "G", res["G"], "nested", res["nested"], "adj", res["adj"])
        print(name, "beta", beta, "rss", float(w @ (e * e)))
    np.savez_compressed(HERE / "assemble.npz", **out)


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else "/root/reference")

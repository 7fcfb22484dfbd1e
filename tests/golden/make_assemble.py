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
nested in its own clusters).  Outputs go to tests/golden/assemble.npz.
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


def main(root):
    kb = import_reference(root)["core.kernels_base"]
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
        print(name, "beta", beta, "rss", float(w @ (e * e)))
    np.savez_compressed(HERE / "assemble.npz", **out)


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else "/root/reference")

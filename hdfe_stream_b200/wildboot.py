"""The wild cluster bootstrap from per-cluster sums (core/wildboot.py,
core/results.py:245-307 `wildboottest`), the draws' arithmetic on the device.

With every fixed effect nested in the clusters, a test of beta_j = 0 needs
only each cluster's H_g = sum w h h' and s_g = sum w e h (Roodman, MacKinnon,
Nielsen and Webb 2019).  With A = (sum_g H_g)^-1: the restricted fit moves
beta by delta = A_j beta_j / A_jj, its scores are s_g + H_g delta (s_g itself
unrestricted), a draw v (a weight per cluster) gives the numerator
sum_g v_g a_g (a_g = A_j' s_g) and the cluster scores v_g a_g - c_g' w
(c_g = A H_g A_j, w = sum_g v_g s_g), whose CRV1 variance (with the fit's
small-sample factor) is the denominator.  A block of B draws is a few
(G x B)(B x k) products, on the device.

The weights are drawn on the host exactly as the `wildboottest` package draws
them (one G x B matrix from numpy's default_rng(seed), clusters in sorted
order; every sign pattern once when Rademacher and 2^G < B), so a seed gives
the reference's draws and p-values.
"""

from __future__ import annotations

from itertools import product

import numpy as np

BLOCK = 1 << 25                     # weights held at once (core/wildboot.py:38)


def _torch():
    import torch
    return torch


def _weights(kind, n, rng):
    if kind == "rademacher":
        return rng.choice([-1, 1], size=n, replace=True)
    if kind == "mammen":
        r5 = np.sqrt(5)
        return rng.choice(np.array([-1, 1]) * (r5 + np.array([-1, 1])) / 2, size=n,
                          replace=True, p=(r5 + np.array([1, -1])) / (2 * r5))
    if kind == "webb":
        return rng.choice(np.concatenate([-np.sqrt(np.array([3, 2, 1]) / 2),
                                          np.sqrt(np.array([1, 2, 3]) / 2)]),
                          replace=True, size=n)
    if kind == "norm":
        return rng.normal(size=n)
    raise ValueError("weights_type must be one of ['mammen', 'norm', 'rademacher', 'webb'], "
                     f"got {kind!r}")


def draws(weights_type, G, reps, seed):
    """Blocks of weights (G x b) and whether they enumerate every sign
    pattern (core/wildboot.py:65-82 `_draws`)."""
    _weights(weights_type, 0, np.random.default_rng(0))     # validates the name
    if weights_type == "rademacher" and 2 ** G < reps:
        return [np.array(list(product([-1, 1], repeat=G)), dtype=float).T], True
    rng = np.random.default_rng(seed)
    per = reps if G * reps <= BLOCK else max(1, BLOCK // G)
    out, left = [], reps
    while left:
        b = min(per, left)
        out.append(np.asarray(_weights(weights_type, G * b, rng), dtype=float).reshape(G, b))
        left -= b
    return out, False


def bootstrap_t(AG, sG, beta, j, adj, reps=9999, weights_type="rademacher", impose_null=True,
                seed=None, device=None):
    """(t, t* (B,), enumerated) for the test of beta_j = 0 from the clusters'
    sums AG (G, k, k) and sG (G, k) (core/wildboot.py:85-102 `_Test`)."""
    torch = _torch()
    dev = device if device is not None else torch.device("cuda", torch.cuda.current_device())
    f64 = dict(dtype=torch.float64, device=dev)
    AG = torch.as_tensor(np.asarray(AG) if not torch.is_tensor(AG) else AG).to(**f64)
    sG = torch.as_tensor(np.asarray(sG) if not torch.is_tensor(sG) else sG).to(**f64)
    beta = np.asarray(beta, np.float64)
    A = torch.linalg.inv(AG.sum(dim=0))
    Aj = A[:, j]
    S = sG + torch.einsum("gab,b->ga", AG, Aj * (beta[j] / A[j, j])) if impose_null else sG
    a = S @ Aj
    C = torch.einsum("gab,b->ga", AG, Aj) @ A
    t = float(beta[j] / np.sqrt(adj * float(((sG @ Aj) ** 2).sum())))
    blocks, enumerated = draws(weights_type, int(AG.shape[0]), reps, seed)
    out = []
    for V in blocks:
        Vt = torch.as_tensor(V.T, **f64)
        num = Vt @ a
        U = Vt * a - (Vt @ S) @ C.T
        out.append(num / torch.sqrt(adj * (U * U).sum(dim=1)))
    return t, torch.cat(out).cpu().numpy(), enumerated


def wildboottest(est, param: int, reps=9999, weights_type="rademacher", impose_null=True,
                 seed=None):
    """core/results.py:245-307 `wildboottest` for an `inference.estimate`
    result made with `bootcluster`: {"param", "t value", "Pr(>|t|)", "reps",
    "weights_type", "impose_null", "cluster"}; a draw at least as extreme as
    t, ties to rounding included, counts (core/results.py:863-867)."""
    boot = est.get("boot")
    if boot is None:
        raise ValueError("wildboottest needs the per-cluster sums, which the fit keeps only "
                         "when asked: estimate with bootcluster=<cluster>")
    t, tstar, _ = bootstrap_t(boot["AG"], boot["sG"], est["beta"], int(param), boot["adj"],
                              reps, weights_type, impose_null, seed)
    return {"param": param, "t value": t,
            "Pr(>|t|)": float(np.mean(np.abs(tstar) >= np.abs(t) * (1 - 1e-9))),
            "reps": int(tstar.shape[0]), "weights_type": weights_type,
            "impose_null": impose_null, "cluster": boot["cluster"]}

"""Seeded employer-employee panels, and pass 0's row layout for them.

The panels are the synthetic inputs of the fixed-effects solve path: workers
observed over a run of consecutive years, moving between firms, with
log earnings = worker effect + firm effect + year effect + an age profile +
noise.  The generator follows this specification (it is not the reference's
own `simulate_akm`, whose panels differ in shape):

* worker effect alpha ~ N(0, 1), firm effect psi ~ N(0, 0.5^2), year effect
  ~ N(0, 0.1^2), noise ~ N(0, 0.5^2);
* each worker is present for a spell of consecutive years (a fixed length, or
  uniform on a range), starting uniformly within the panel's years;
* the first firm, and the firm after each move (yearly probability p_move),
  is the firm at quantile Phi(rho * alpha + sqrt(1 - rho^2) * e) of the
  firms ranked by psi (rho = 0.3), so better workers sort into better firms;
* age is uniform on 25-60 over the spell; the covariates are
  age_squared = age^2 / 100 and age_cubed = age^3 / 1000, the reference's
  scaling (simulate.py:136-137);
* int32 ids, float64 values; optional analytic weights uniform on [0.5, 2].

`pass0_layout` then lays the rows out as the reference's pass 0 does for a
fit that keeps its intermediates (core/passes.py:285-294, 359-373, with
n_buckets = 1): every fixed effect's codes are the ranks of its levels in
sorted order, the streamed dimension (the workers: the highest cardinality,
core/estimator.py:371-385) becomes the dense group code `gcode`, and the rows
are sorted by (gcode, the other codes, the variables).
"""

from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

from math import sqrt

from scipy.special import ndtr


@dataclass
class Panel:
    """Raw rows of a simulated panel (one row per worker-year)."""

    worker: np.ndarray          # int32
    firm: np.ndarray            # int32
    year: np.ndarray            # int32
    log_earn: np.ndarray        # float64
    age_squared: np.ndarray     # float64
    age_cubed: np.ndarray       # float64
    weight: np.ndarray | None = None
    truth: dict = field(default_factory=dict)

    @property
    def n_rows(self) -> int:
        return len(self.worker)


def simulate_panel(n_workers: int, n_firms: int, n_years: int, spell=(8, 8),
                   p_move: float = 0.1, sd_firm: float = 0.5, sd_year: float = 0.1,
                   sd_noise: float = 0.5, rho: float = 0.3, weights: bool = False,
                   seed: int = 0) -> Panel:
    """A panel per the specification in the module docstring.

    `spell` is (shortest, longest) years a worker is present, drawn uniformly;
    (8, 8) gives every worker 8 consecutive years, (5, 12) about 8.5.
    """
    lo, hi = int(spell[0]), int(spell[1])
    if not 1 <= lo <= hi <= n_years:
        raise ValueError("spell lengths must lie within 1..n_years")
    rng = np.random.default_rng(seed)
    alpha = rng.standard_normal(n_workers)
    psi = rng.normal(0.0, sd_firm, n_firms)
    year_eff = rng.normal(0.0, sd_year, n_years)
    by_quality = np.argsort(psi, kind="stable")
    length = rng.integers(lo, hi + 1, n_workers)
    first = rng.integers(0, n_years - length + 1)
    age0 = rng.integers(25, 60 - length + 2)        # last age <= 60

    n = int(length.sum())
    worker = np.repeat(np.arange(n_workers, dtype=np.int64), length)
    begin = np.concatenate(([0], np.cumsum(length)[:-1]))
    t = np.arange(n) - np.repeat(begin, length)     # year within the spell
    year = np.repeat(first, length) + t
    age = (np.repeat(age0, length) + t).astype(np.float64)

    # firm spells: a fresh draw at each worker's first year and at each move
    a = alpha[worker]
    score = rho * a + sqrt(1.0 - rho * rho) * rng.standard_normal(n)
    cand = by_quality[np.minimum((ndtr(score) * n_firms).astype(np.int64),
                                 n_firms - 1)]
    moves = rng.random(n) < p_move
    start_of_spell = (t == 0) | moves
    last = np.maximum.accumulate(np.where(start_of_spell, np.arange(n), 0))
    firm = cand[last]

    age_sq = age * age / 100.0
    age_cu = age * age * age / 1000.0
    noise = rng.normal(0.0, sd_noise, n)
    y = (10.0 + a + psi[firm] + year_eff[year] + 0.08 * age_sq - 0.012 * age_cu + noise)
    w = rng.uniform(0.5, 2.0, n) if weights else None
    return Panel(worker=worker.astype(np.int32), firm=firm.astype(np.int32),
                 year=year.astype(np.int32), log_earn=y, age_squared=age_sq,
                 age_cubed=age_cu, weight=w,
                 truth={"alpha": alpha, "psi": psi, "year": year_eff})


@dataclass
class Rows:
    """Pass 0's output layout: rows sorted by group, with codes.

    gcode (N,) uint32     dense code of the streamed dimension (the workers)
    codes (N, D) uint32   codes of the other dimensions (firm, year), sorted-
                          level ranks, in the formula's order
    V     (N, m) float64  the design variables: outcome, then covariates
    w     (N,) float64    analytic weights, or None
    n_levels              levels per non-streamed dimension, and n_groups
    names                 the variables' names
    """

    gcode: np.ndarray
    codes: np.ndarray
    V: np.ndarray
    w: np.ndarray | None
    n_levels: list
    n_groups: int
    names: list
    ids: dict = field(default_factory=dict)

    @property
    def n_rows(self) -> int:
        return len(self.gcode)

    @property
    def offs(self) -> np.ndarray:
        return np.concatenate(([0], np.cumsum(self.n_levels)[:-1])).astype(np.int64)

    @property
    def n_total_levels(self) -> int:
        return int(sum(self.n_levels))


def _rank_codes(values: np.ndarray):
    """Codes = rank of each value among the sorted distinct values
    (core/passes.py:285-294: unique().sort() then a row index).  Ids are
    small non-negative integers here, so a presence table does it in O(n)."""
    values = np.asarray(values)
    if len(values) and values.min() >= 0 and values.max() < 4 * len(values) + 1024:
        present = np.zeros(int(values.max()) + 1, bool)
        present[values] = True
        rank = np.cumsum(present) - 1
        return rank[values].astype(np.uint32), np.flatnonzero(present)
    levels, codes = np.unique(values, return_inverse=True)
    return codes.astype(np.uint32), levels


def pass0_layout(panel: Panel, keep: np.ndarray | None = None, year_fe: bool = True) -> Rows:
    """Rows of `panel` (optionally only those where `keep`) in pass 0's
    layout, sorted by (worker, firm, year, variables).  year_fe False: the
    model has worker and firm effects only (codes (N, 1))."""
    sel = slice(None) if keep is None else np.asarray(keep, bool)
    g, wlev = _rank_codes(panel.worker[sel])
    c1, flev = _rank_codes(panel.firm[sel])
    c2, ylev = _rank_codes(panel.year[sel])
    V = np.column_stack([panel.log_earn[sel], panel.age_squared[sel],
                         panel.age_cubed[sel]]).astype(np.float64)
    w = None if panel.weight is None else panel.weight[sel].astype(np.float64)
    key = (g.astype(np.int64) * len(flev) + c1) * len(ylev) + c2
    order = np.argsort(key, kind="stable")
    sk = key[order]
    if len(sk) > 1 and bool(np.any(sk[1:] == sk[:-1])):
        # rows sharing (worker, firm, year): the variables break the tie
        order = np.lexsort((V[:, 2], V[:, 1], V[:, 0], c2, c1, g))
    codes = np.column_stack([c1[order], c2[order]]) if year_fe else c1[order][:, None]
    return Rows(gcode=np.ascontiguousarray(g[order]), codes=np.ascontiguousarray(codes),
                V=np.ascontiguousarray(V[order]),
                w=None if w is None else np.ascontiguousarray(w[order]),
                n_levels=[len(flev), len(ylev)] if year_fe else [len(flev)],
                n_groups=len(wlev), names=["log_earn", "age_squared", "age_cubed"],
                ids={"worker": wlev, "firm": flev, "year": ylev})


def restrict_connected(panel: Panel, min_degree=(1, 1)) -> np.ndarray:
    """Rows kept by pass 0's `connected="largest"` restriction of the
    (worker, firm) graph, after `min_degree` pruning: core/passes.py:780-857
    `_connected_restriction` with core/connected.py:378-493
    `_find_components` -- levels with fewer than k distinct partners are
    removed until none is left, then the largest component by rows is kept
    (ties to the component holding the smallest worker).  This is input
    preparation on the host (pass 0), not a device kernel."""
    from scipy.sparse import coo_matrix
    from scipy.sparse.csgraph import connected_components

    _, wlev = _rank_codes(panel.worker)
    a, _ = _rank_codes(panel.worker)
    b, flev = _rank_codes(panel.firm)
    n0, n1 = len(wlev), len(flev)
    key = a.astype(np.int64) * n1 + b
    run = np.concatenate(([True], key[1:] != key[:-1]))
    keys, inv = np.unique(key[run], return_inverse=True)
    counts = np.bincount(inv, weights=np.diff(np.append(np.flatnonzero(run), len(key))))
    pa, pb = keys // n1, keys % n1
    alive0, alive1 = np.ones(n0, bool), np.ones(n1, bool)
    k0, k1 = (min_degree, min_degree) if np.isscalar(min_degree) else min_degree
    if (k0, k1) != (1, 1):
        while True:
            e = alive0[pa] & alive1[pb]
            d0 = np.bincount(pa[e], minlength=n0)
            d1 = np.bincount(pb[e], minlength=n1)
            drop0 = alive0 & (d0 < k0)
            drop1 = alive1 & (d1 < k1)
            if not (drop0.any() or drop1.any()):
                break
            alive0 &= ~drop0
            alive1 &= ~drop1
    e = alive0[pa] & alive1[pb]
    nv = n0 + n1
    adj = coo_matrix((np.ones(int(e.sum())), (pa[e], n0 + pb[e])), shape=(nv, nv))
    nc, lab = connected_components(adj, directed=False)
    alive = np.concatenate([alive0, alive1])
    rows = np.bincount(lab[pa[e]], weights=counts[e], minlength=nc)
    first = np.full(nc, nv, np.int64)
    np.minimum.at(first, lab, np.where(alive, np.arange(nv), nv))
    order = np.lexsort((first, -rows))
    best = order[0]
    ok0 = alive0 & (lab[:n0] == best)
    ok1 = alive1 & (lab[n0:] == best)
    return ok0[a] & ok1[b]


def restrict_leave_one_out(panel: Panel, keep: np.ndarray | None = None) -> np.ndarray:
    """Rows of the leave-one-out connected set of the (worker, firm) network
    (core/connected.py:503-557 `_leave_one_out`, which the reference's
    `leave_out_kss` applies), among the rows where `keep`: found on the
    device by `connected.leave_one_out` from the rows' codes in (worker,
    firm) order."""
    import torch
    from .connected import leave_one_out
    sel = np.ones(panel.n_rows, bool) if keep is None else np.asarray(keep, bool)
    idx = np.flatnonzero(sel)
    a, _ = _rank_codes(panel.worker[idx])
    b, flev = _rank_codes(panel.firm[idx])
    n0, n1 = int(a.max()) + 1, len(flev)
    order = np.lexsort((b, a))
    dev = torch.device("cuda", torch.cuda.current_device())
    alive, _ = leave_one_out(torch.as_tensor(a[order].astype(np.int32), device=dev),
                             torch.as_tensor(b[order].astype(np.int32), device=dev), n0, n1)
    alive = alive.cpu().numpy()
    out = np.zeros(panel.n_rows, bool)
    out[idx] = alive[a] & alive[n0 + b.astype(np.int64)]
    return out


# The panels the solve path is measured on, by what they are.
PANELS = {
    # 20k workers, 2k firms, 10 years, 8 consecutive years each (160k rows)
    "akm_20k": dict(n_workers=20_000, n_firms=2_000, n_years=10, spell=(8, 8),
                    p_move=0.1),
    # 5M workers, 500k firms, 15 years, ~8.5 rows per worker (~42M rows)
    "akm_5m": dict(n_workers=5_000_000, n_firms=500_000, n_years=15, spell=(5, 12),
                   p_move=0.08),
    # 2M workers, 200k firms, 15 years: the 5M-worker panel's shape at 2/5 of
    # the size (S and the vectors still larger than L2), for kernel profiles
    "akm_2m": dict(n_workers=2_000_000, n_firms=200_000, n_years=15, spell=(5, 12),
                   p_move=0.08),
    # 1M workers, 100k firms, 10 years, ~8.5 rows per worker (~8.5M rows)
    "kss_1m": dict(n_workers=1_000_000, n_firms=100_000, n_years=10, spell=(7, 10),
                   p_move=0.1),
    # 100k workers, 10k firms, 10 years (~850k rows): the 1M-worker panel's
    # shape at a tenth of the size, for kernel profiles
    "kss_100k": dict(n_workers=100_000, n_firms=10_000, n_years=10, spell=(7, 10),
                     p_move=0.1),
    # 400k workers, 40k firms, 10 years (~3.4M rows), weights U[0.5, 2]
    "akm_400k_w": dict(n_workers=400_000, n_firms=40_000, n_years=10, spell=(7, 10),
                       p_move=0.1, weights=True),
}


def prepare(name: str, seed: int = 0):
    """The named panel's rows in pass 0's layout, restricted as its
    specification says: akm_5m the largest connected set after min_degree 2;
    kss_1m the leave-one-out connected set (found on the device: kss_1m
    needs a GPU), with worker and firm effects only (log_earn ~ age_squared +
    age_cubed | worker_id + firm_id)."""
    spec = dict(PANELS[name])
    panel = simulate_panel(seed=seed, **spec)
    if name in ("akm_5m", "akm_2m"):
        return pass0_layout(panel, restrict_connected(panel, (2, 2)))
    if name.startswith("kss_"):
        return pass0_layout(panel, restrict_leave_one_out(panel), year_fe=False)
    return pass0_layout(panel)

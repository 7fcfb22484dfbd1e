"""The oracle: a CPU restatement of hdfe-stream's fixed-effects solve path.

TEST INFRASTRUCTURE ONLY.  tests/, `__graft_entry__.smoke()` and bench.py's
CPU-baseline leg use this as the checker and as the timed CPU baseline; the
product (hdfe_stream_b200/) never imports it.

The numba kernels of the reference are restated in C (hdfe_oracle.c, built by
the Makefile beside it, bit-identical to the numba kernels); the numpy glue
around them here restates the reference's own Python driver code, each
function citing the reference file:line it follows.  Parity against the
reference itself is pinned by tests/test_oracle.py on the golden vectors of
tests/golden/, which tests/golden/make_golden.py produced by running the
reference's kernels and mixins on the same panels.
"""

from __future__ import annotations

import ctypes
import os
import subprocess
from dataclasses import dataclass, field
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "libhdfe_oracle.so"

# core/solve.py:44 and :49; core/passes.py:48
RHS_ZERO_TOL = 1e-11
CG_BLOCKS = 256

_lib = None


def build() -> Path:
    """Compile the oracle's C kernels (make), if not built already."""
    src = HERE / "hdfe_oracle.c"
    if not LIB_PATH.exists() or LIB_PATH.stat().st_mtime < src.stat().st_mtime:
        subprocess.run(["make", "-s", "-C", str(HERE)], check=True)
    return LIB_PATH


def lib():
    global _lib
    if _lib is None:
        build()
        _lib = ctypes.CDLL(str(LIB_PATH))
        for name in ("orc_peel", "orc_dense_labels", "orc_bfs_components"):
            getattr(_lib, name).restype = ctypes.c_int64
    return _lib


def _p(a):
    """ctypes pointer of a numpy array (None for None)."""
    if a is None:
        return None
    return ctypes.c_void_p(a.ctypes.data)


def _i(x):
    return ctypes.c_int64(int(x))


def set_threads(n: int) -> None:
    lib().orc_set_threads(ctypes.c_int(int(n)))


def num_threads() -> int:
    return int(lib().orc_num_threads())


# ---------------------------------------------------------------- pass 1

@dataclass
class Cells:
    """Pass 1's output (core/passes.py:397-531, the plain case):
    identifying cells and the level bookkeeping built with them."""

    starts: np.ndarray          # (G'+1,) int64, groups with more than one cell
    codes: np.ndarray           # (M, D) uint32
    n: np.ndarray               # (M,) float64 cell weight
    sums: np.ndarray            # (M, m) float64 centred sums
    obs: np.ndarray             # (L,) weight per level, all cells
    cnt: np.ndarray             # (L,) rows per level, all cells
    diag: np.ndarray            # (L,) diagonal of S
    rhs: np.ndarray             # (L, m) D_o' M_0 V
    offs: np.ndarray            # (D,) int64
    n_levels: list
    n_cells: int
    fe0_rank: int
    means: np.ndarray
    raw_ss: np.ndarray
    pair_components: dict = field(default_factory=dict)

    @property
    def L(self) -> int:
        return int(sum(self.n_levels))


def cell_runs(rows):
    """Cells of sorted rows (core/passes.py:533-589 `_cell_chunks`): runs of
    equal (gcode, codes); cnt, n and the sums of the centred variables
    (`_nb_run_sums`, core/kernels_base.py:375-422)."""
    g = rows.gcode
    n_rows = len(g)
    same = g[1:] == g[:-1]
    for d in range(rows.codes.shape[1]):
        c = rows.codes[:, d]
        same &= c[1:] == c[:-1]
    cs = np.flatnonzero(np.concatenate(([True], ~same)))
    bounds = np.append(cs, n_rows).astype(np.int64)
    run = np.diff(bounds)
    means = rows.V.mean(axis=0) if n_rows else np.zeros(rows.V.shape[1])
    w = rows.w
    weighted = w is not None
    out = {"g": g[cs], "codes": rows.codes[cs], "cnt": run.astype(np.float64)}
    out["n"] = np.add.reduceat(w, cs) if weighted else out["cnt"]
    m = rows.V.shape[1]
    ZT = np.empty((m, n_rows))
    for j in range(m):
        np.subtract(rows.V[:, j], means[j], out=ZT[j])
    ST = np.empty((m, len(cs)))
    lib().orc_run_sums(_p(bounds), _i(len(cs)), _p(ZT), _i(m), _i(n_rows),
                       _p(np.ascontiguousarray(w) if weighted else None), _p(ST))
    out["S"] = np.ascontiguousarray(ST.T)
    return out, means


def segments(g):
    """core/utils.py:62-69 `_segments`: segment starts and local index."""
    brk = np.flatnonzero(g[1:] != g[:-1]) + 1
    starts = np.concatenate(([0], brk))
    local = np.zeros(len(g), dtype=np.int64)
    local[brk] = 1
    np.cumsum(local, out=local)
    return starts, local


def pass1(rows) -> Cells:
    """`_pass1_cells` (core/passes.py:397-531) over one chunk holding every
    row: cells, obs/cnt per level, identifying cells (groups of more than one
    cell), the Jacobi diagonal and the right-hand side D_o' M_0 V, and the
    pair union-find for the degrees of freedom."""
    ch, means = cell_runs(rows)
    nl = list(rows.n_levels)
    D = len(nl)
    offs = np.concatenate(([0], np.cumsum(nl)[:-1])).astype(np.int64)
    L = int(sum(nl))
    m = rows.V.shape[1]
    obs = np.zeros(L)
    cnt = np.zeros(L)
    diag = np.zeros(L)
    rhs = np.zeros((L, m))
    for d in range(D):
        sl = slice(offs[d], offs[d] + nl[d])
        obs[sl] += np.bincount(ch["codes"][:, d], weights=ch["n"], minlength=nl[d])
        cnt[sl] += np.bincount(ch["codes"][:, d], weights=ch["cnt"], minlength=nl[d])
    uf = {(i, j): np.arange(nl[i] + nl[j], dtype=np.int64)
          for i in range(D) for j in range(i + 1, D)}
    for (i, j), parent in uf.items():
        a = np.ascontiguousarray(ch["codes"][:, i])
        b = np.ascontiguousarray(ch["codes"][:, j])
        lib().orc_union_pairs(_p(parent), _p(a), _p(b), _i(len(a)), _i(nl[i]))
    starts, local = segments(ch["g"])
    ncells = np.diff(np.append(starts, len(local)))
    keep = ncells[local] > 1
    fe0_rank = len(starts)
    kept = ncells[ncells > 1]
    kstarts = np.concatenate(([0], np.cumsum(kept))).astype(np.int64)
    kcodes = np.ascontiguousarray(ch["codes"][keep]).astype(np.uint32)
    kn = np.ascontiguousarray(ch["n"][keep]).astype(np.float64)
    ksums = np.ascontiguousarray(ch["S"][keep])
    G = len(kstarts) - 1
    lib().orc_diag(_p(kstarts), _i(G), _p(kcodes), _i(D), _p(kn), _p(offs), _p(diag))
    lib().orc_rhs(_p(kstarts), _i(G), _p(kcodes), _i(D), _p(kn), _p(ksums), _i(m),
                  _p(offs), _p(rhs))
    n_obs = rows.n_rows
    raw_ss = (rows.V.var(axis=0, ddof=1) * max(n_obs - 1, 1)) if n_obs > 1 else np.zeros(m)
    pair = {(i, j): int(np.count_nonzero(p == np.arange(len(p)))) for (i, j), p in uf.items()}
    return Cells(starts=kstarts, codes=kcodes, n=kn, sums=ksums, obs=obs, cnt=cnt,
                 diag=diag, rhs=rhs, offs=offs, n_levels=nl, n_cells=len(ch["g"]),
                 fe0_rank=fe0_rank, means=means, raw_ss=raw_ss, pair_components=pair)


# ------------------------------------------------------------ components

def components(cells: Cells, col: int = 0):
    """Union-find over dimension `col` (`_nb_components`,
    core/kernels_base.py:156-174): the root of each level's component."""
    nl = cells.n_levels[col]
    parent = np.empty(nl, np.int64)
    G = len(cells.starts) - 1
    lib().orc_components(_p(cells.starts), _i(G), _p(cells.codes), _i(cells.codes.shape[1]),
                         _i(col), _i(nl), _p(parent))
    return parent


def rank_components(root: np.ndarray, cnt_first: np.ndarray):
    """core/passes.py:933-950 `_rank_components`: labels 0, 1, ... by rows,
    ties to the component with the smallest level (a stable sort)."""
    nl = len(root)
    is_root = root == np.arange(nl)
    dense = (np.cumsum(is_root) - 1)[root]
    rows = np.bincount(dense, weights=cnt_first, minlength=int(is_root.sum()))
    order = np.argsort(-rows, kind="stable")
    rank = np.empty(len(order), np.int64)
    rank[order] = np.arange(len(order))
    return rank[dense], len(order)


def component_labels(cells: Cells):
    """(comp, n_components) for the first non-streamed dimension, as
    `_components` (core/passes.py:952-979) computes them."""
    root = components(cells, 0)
    return rank_components(root, cells.cnt[cells.offs[0]:cells.offs[0] + cells.n_levels[0]])


# ------------------------------------------------------------- explicit S

def build_explicit(cells: Cells, n_threads: int | None = None):
    """`_build_explicit` (core/solve.py:148-194) for the plain case:
    S = D_o' M_0 D_o in CSR with sorted columns (indptr int64, indices
    int32, data float64)."""
    D = cells.codes.shape[1]
    L = cells.L
    G = len(cells.starts) - 1
    lptr = np.empty(L + 1, np.int64)
    lib().orc_level_groups(_p(cells.starts), _i(G), _p(cells.codes), _i(D), _p(cells.offs),
                           _i(L), _p(lptr), None)
    lgrp = np.empty(int(lptr[L]), np.int32)
    lib().orc_level_groups(_p(cells.starts), _i(G), _p(cells.codes), _i(D), _p(cells.offs),
                           _i(L), _p(lptr), _p(lgrp))
    work = np.empty(L, np.int64)
    lib().orc_row_work(_p(cells.starts), _p(lptr), _p(lgrp), _i(L), _p(work))
    wide = max(L // (4 * D), 1)
    rnnz = np.empty(L, np.int64)
    lib().orc_row_nnz(_p(cells.starts), _p(cells.codes), _i(D), _p(cells.offs), _p(lptr),
                      _p(lgrp), _p(work), _i(wide), _i(L), _p(rnnz))
    nnz = int(rnnz.sum())
    indptr = np.zeros(L + 1, np.int64)
    np.cumsum(rnnz, out=indptr[1:])
    indices = np.empty(nnz, np.int32)
    data = np.empty(nnz)
    ng = np.add.reduceat(cells.n, cells.starts[:-1]) if G else np.zeros(0)
    ng = np.ascontiguousarray(ng)
    lib().orc_row_fill(_p(cells.starts), _p(cells.codes), _i(D), _p(cells.n), _p(ng),
                       _p(cells.offs), _i(D), _p(lptr), _p(lgrp), _p(work), _i(wide), _i(L),
                       _p(indptr), _p(indices), _p(data))
    return indptr, indices, data


def jacobi(diag: np.ndarray) -> np.ndarray:
    """core/solve.py:142-146 `_jacobi`."""
    pos = diag > 1e-12
    return np.where(pos, 1.0 / np.where(pos, diag, 1.0), 0.0)


# ---------------------------------------------------------------- PCG

def csr_matmat(S, X):
    indptr, indices, data = S
    X = np.ascontiguousarray(X, dtype=np.float64)
    out = np.empty_like(X)
    lib().orc_csr_matmat(_p(indptr), _p(indices), _p(data), _i(len(indptr) - 1), _p(X),
                         _i(X.shape[1]), _p(out))
    return out


def pcg(S, dinv, b, zero=None, x0=None, tol=1e-10, maxiter=5000):
    """`_SolveMixin._pcg` (core/solve.py:66-140) with the Jacobi
    preconditioner: block PCG, one CG per column in lockstep, column sums over
    256 fixed row blocks.  Returns (X, iterations, converged, max rel)."""
    b = np.asarray(b, dtype=np.float64)
    bnorm = np.linalg.norm(b, axis=0)
    bnorm[bnorm == 0] = 1.0
    if x0 is None:
        X = np.zeros_like(b)
        R = b.copy()
    else:
        X = np.array(x0, dtype=np.float64, order="C")
        R = b - csr_matmat(S, X)
    if zero is not None and zero.any():
        X[:, zero] = 0.0
        R[:, zero] = 0.0
        if zero.all():
            return X, 0, True, 0.0
    active = np.ones(b.shape[1], bool) if zero is None else ~zero
    rel = np.zeros(b.shape[1])
    if x0 is not None:
        rel = np.linalg.norm(R, axis=0) / bnorm
        active &= rel > tol
        if not active.any():
            return X, 0, True, float(rel.max())
    X, R = np.ascontiguousarray(X), np.ascontiguousarray(R)
    L, k = X.shape
    dinv = np.ascontiguousarray(dinv, dtype=np.float64)
    nblk = max(1, min(CG_BLOCKS, L))
    parts = np.empty((nblk, 2, k))
    dots = np.empty((nblk, k))
    P = np.ascontiguousarray(R * dinv[:, None])
    lib().orc_cg_dot(_p(R), _p(P), _i(L), _i(k), _i(nblk), _p(dots))
    rz = dots.sum(axis=0)
    it = 0
    for it in range(1, maxiter + 1):
        AP = csr_matmat(S, P)
        lib().orc_cg_dot(_p(P), _p(AP), _i(L), _i(k), _i(nblk), _p(dots))
        pAp = dots.sum(axis=0)
        alpha = np.where(active & (pAp > 0), rz / np.where(pAp > 0, pAp, 1), 0.0)
        alpha = np.ascontiguousarray(alpha)
        lib().orc_cg_step(_p(X), _p(R), _p(P), _p(AP), _p(alpha), _p(dinv), _i(L), _i(k),
                          _i(nblk), _p(parts))
        sums = parts.sum(axis=0)
        rel = np.sqrt(sums[0]) / bnorm
        active = rel > tol
        if not active.any():
            break
        rz_new = sums[1]
        beta = np.ascontiguousarray(np.where(active, rz_new / np.where(rz != 0, rz, 1), 0.0))
        lib().orc_cg_direction(_p(P), _p(R), _p(dinv), _p(beta), _i(L), _i(k))
        rz = rz_new
    return X, it, bool(not active.any()), float(rel.max())


def normalize(Gamma, cells: Cells, comp):
    """core/solve.py:383-399 `_normalize`: first dimension's effects have
    obs-weighted mean zero within each component, further dimensions global
    obs-weighted mean zero."""
    nl, o = cells.n_levels[0], cells.offs[0]
    w = cells.obs[o:o + nl]
    cw = np.bincount(comp, weights=w, minlength=nl)
    cw[cw == 0] = 1.0
    mean = scatter(comp, w[:, None] * Gamma[o:o + nl], nl) / cw[:, None]
    Gamma[o:o + nl] -= mean[comp]
    for d in range(1, len(cells.n_levels)):
        nl, o = cells.n_levels[d], cells.offs[d]
        w = cells.obs[o:o + nl]
        Gamma[o:o + nl] -= (w @ Gamma[o:o + nl]) / max(w.sum(), 1.0)
    return Gamma


def scatter(idx, vals, n):
    """core/utils.py `_scatter`: column-wise bincount of `vals` (rows) by `idx`."""
    out = np.zeros((n, vals.shape[1]))
    for j in range(vals.shape[1]):
        out[:, j] = np.bincount(idx, weights=vals[:, j], minlength=n)
    return out


def solve(cells: Cells, S, tol=1e-10, maxiter=5000, rhs_block=8, comp=None, x0=None):
    """`_SolveMixin._solve` (core/solve.py:294-368) for the estimator's own
    variables, whose right-hand side pass 1 built: zero-column detection
    against each variable's total sum of squares, block PCG per rhs_block
    columns, then `_normalize`.  Returns (Gamma, info)."""
    L = cells.L
    m = cells.rhs.shape[1]
    if comp is None:
        comp, _ = component_labels(cells)
    dinv = jacobi(cells.diag)
    gamma = np.empty((L, m))
    its, conv, rel = [], True, 0.0
    for j0 in range(0, m, rhs_block):
        j1 = min(m, j0 + rhs_block)
        b = cells.rhs[:, j0:j1]
        scale = np.sqrt(np.maximum(cells.raw_ss[j0:j1], 0.0))
        zero = np.linalg.norm(b, axis=0) <= RHS_ZERO_TOL * scale
        X, it, c, r = pcg(S, dinv, b, zero, None if x0 is None else x0[:, j0:j1], tol, maxiter)
        gamma[:, j0:j1] = normalize(X, cells, comp)
        its.append(it)
        conv &= c
        rel = max(rel, r)
    return gamma, {"iterations": its if len(its) > 1 else its[0], "converged": conv,
                   "max_rel_residual": rel}


# ---------------------------------------------------- random draws, rows

def rademacher(ordinal, n_rows, draws, seed, first_draw=0):
    """core/kernels_groups.py:53-76 `_nb_rademacher`."""
    out = np.empty((n_rows, draws))
    lib().orc_rademacher(_i(ordinal), _i(n_rows), _i(draws), ctypes.c_uint64(seed & (2**64 - 1)),
                         _i(first_draw), _p(out))
    return out


def row_starts(gcode):
    """Group boundaries of sorted rows (inverse.py:139-142 `_chunk_layout`)."""
    n = len(gcode)
    return np.concatenate(([0], np.flatnonzero(gcode[1:] != gcode[:-1]) + 1, [n])).astype(np.int64)


def center_rows(starts, codes, offs, w, X, R, L, nt=1):
    """kernels_inverse.py:35-71 `_nb_center_rows` with `nt` accumulator
    copies; returns (acc.sum(0), acc_x.sum(0))."""
    codes = np.ascontiguousarray(codes, dtype=np.int64)
    G = len(starts) - 1
    m = R.shape[1]
    k = X.shape[1]
    acc = np.zeros((nt, L, m))
    acc_x = np.zeros((nt, k, m))
    lib().orc_center_rows(_p(starts), _i(G), _p(codes), _i(codes.shape[1]), _p(offs),
                          _p(np.ascontiguousarray(w, dtype=np.float64)),
                          _p(np.ascontiguousarray(X, dtype=np.float64)), _i(k),
                          _p(np.ascontiguousarray(R, dtype=np.float64)), _i(m), _i(nt), _i(L),
                          _p(acc), _p(acc_x))
    return acc.sum(axis=0), acc_x.sum(axis=0)


def project_rows_kernel(starts, codes, offs, w, X, C, R, U):
    """kernels_inverse.py:75-107 `_nb_project_rows`."""
    codes = np.ascontiguousarray(codes, dtype=np.int64)
    R = np.ascontiguousarray(R, dtype=np.float64)
    out = np.empty_like(R)
    lib().orc_project_rows(_p(starts), _i(len(starts) - 1), _p(codes), _i(codes.shape[1]),
                           _p(offs), _p(np.ascontiguousarray(w, dtype=np.float64)),
                           _p(np.ascontiguousarray(X, dtype=np.float64)), _i(X.shape[1]),
                           _p(np.ascontiguousarray(C, dtype=np.float64)), _p(R), _i(R.shape[1]),
                           _p(np.ascontiguousarray(U, dtype=np.float64)), _p(out))
    return out


def reduce_rows(starts, codes, offs, w, X, R, L, nt=1):
    """kernels_inverse.py:112-130 `_nb_reduce_rows`."""
    codes = np.ascontiguousarray(codes, dtype=np.int64)
    G = len(starts) - 1
    m = R.shape[1]
    k = X.shape[1]
    acc = np.zeros((nt, L, m))
    acc_x = np.zeros((nt, k, m))
    lib().orc_reduce_rows(_p(starts), _i(G), _p(codes), _i(codes.shape[1]), _p(offs),
                          _p(np.ascontiguousarray(w, dtype=np.float64)),
                          _p(np.ascontiguousarray(X, dtype=np.float64)), _i(k),
                          _p(np.ascontiguousarray(R, dtype=np.float64)), _i(m), _i(nt), _i(L),
                          _p(acc), _p(acc_x))
    return acc.sum(axis=0), acc_x.sum(axis=0)


def spread_groups(starts, w, group_values):
    """kernels_inverse.py:134-152 `_nb_spread_groups`."""
    gv = np.ascontiguousarray(group_values, dtype=np.float64)
    out = np.empty((int(starts[-1]), gv.shape[1]))
    lib().orc_spread_groups(_p(starts), _i(len(starts) - 1),
                            _p(np.ascontiguousarray(w, dtype=np.float64)), _p(gv),
                            _i(gv.shape[1]), _p(out))
    return out


def project_coef(starts, codes, offs, w, X, C, RHO, U):
    """kernels_inverse.py:157-188 `_nb_project_coef`: (rows, groups)."""
    codes = np.ascontiguousarray(codes, dtype=np.int64)
    RHO = np.ascontiguousarray(RHO, dtype=np.float64)
    G = len(starts) - 1
    rows = np.empty_like(RHO)
    groups = np.empty((G, RHO.shape[1]))
    lib().orc_project_coef(_p(starts), _i(G), _p(codes), _i(codes.shape[1]), _p(offs),
                           _p(np.ascontiguousarray(w, dtype=np.float64)),
                           _p(np.ascontiguousarray(X, dtype=np.float64)), _i(X.shape[1]),
                           _p(np.ascontiguousarray(C, dtype=np.float64)), _p(RHO),
                           _i(RHO.shape[1]), _p(np.ascontiguousarray(U, dtype=np.float64)),
                           _p(rows), _p(groups))
    return rows, groups


def group_sums(starts, w, R):
    """core/kernels_groups.py:17-27 `_nb_group_sums`."""
    R = np.ascontiguousarray(R, dtype=np.float64)
    out = np.empty((len(starts) - 1, R.shape[1]))
    lib().orc_group_sums(_p(starts), _i(len(starts) - 1),
                         _p(np.ascontiguousarray(w, dtype=np.float64)), _p(R), _i(R.shape[1]),
                         _p(out))
    return out


def trace_moments(starts, codes, psi_column, psi_offset, w, Zl, Zg, Ul, Ug, nt=1):
    """kernels_inverse.py:192-231 `_nb_trace_moments`: acc (nt, m, 8)."""
    codes = np.ascontiguousarray(codes, dtype=np.int64)
    m = Zg.shape[1]
    acc = np.zeros((nt, m, 8))
    lib().orc_trace_moments(_p(starts), _i(len(starts) - 1), _p(codes), _i(codes.shape[1]),
                            _i(psi_column), _i(psi_offset),
                            _p(np.ascontiguousarray(w, dtype=np.float64)),
                            *[_p(np.ascontiguousarray(a, dtype=np.float64))
                              for a in (Zl, Zg, Ul, Ug)], _i(m), _i(nt), _p(acc))
    return acc


# -------------------------------------------------- bipartite network

def distinct_pairs(a, b, n1):
    """core/connected.py:656-687 `_DistinctPairs` in one batch: sorted
    distinct keys a * n1 + b and the rows behind each."""
    key = a.astype(np.uint64) * np.uint64(max(n1, 1)) + b.astype(np.uint64)
    k, c = np.unique(key, return_counts=True)
    return k, c.astype(np.uint32)


def peel(keys, n1, k0, k1, alive0, alive1):
    """core/kernels_graph.py:188-221 `_nb_peel` (in place); returns rounds."""
    return int(lib().orc_peel(_p(keys), _i(len(keys)), ctypes.c_uint64(max(n1, 1)), _i(k0),
                              _i(k1), _p(alive0), _i(len(alive0)), _p(alive1),
                              _i(len(alive1))))


def largest_connected(a, b, n0, n1, min_degree=(1, 1)):
    """`_find_components` (core/connected.py:378-493) on coded pairs, for
    `connected="largest"` with pruning: returns (alive levels of each
    dimension in the largest component, labels (n0+n1), sizes by rows)."""
    lib_ = lib()
    alive = np.ones(n0 + n1, np.uint8)
    keys, counts = distinct_pairs(a, b, n1)
    n1u = max(n1, 1)
    if tuple(min_degree) != (1, 1):
        a0 = np.ascontiguousarray(alive[:n0])
        a1 = np.ascontiguousarray(alive[n0:])
        peel(keys, n1, min_degree[0], min_degree[1], a0, a1)
        alive[:n0], alive[n0:] = a0, a1
    parent = np.arange(n0 + n1, dtype=np.int64)
    a0 = np.ascontiguousarray(alive[:n0])
    a1 = np.ascontiguousarray(alive[n0:])
    lib_.orc_union_keys(_p(parent), _p(keys), _i(len(keys)), ctypes.c_uint64(n1u), _p(a0),
                        _i(n0), _p(a1))
    nc = int(lib_.orc_dense_labels(_p(parent), _i(n0 + n1), _p(alive)))
    rows = np.zeros(nc, np.int64)
    lib_.orc_pair_rows(_p(keys), _p(counts), _i(len(keys)), ctypes.c_uint64(n1u), _p(parent),
                       _i(n0 + n1), _p(rows))
    order = np.argsort(-rows, kind="stable")
    rank = np.empty(nc, np.int64)
    rank[order] = np.arange(nc)
    # core/kernels_graph.py `_nb_relabel`: negative labels (pruned) stay
    labels = np.where(parent >= 0, rank[np.maximum(parent, 0)] if nc else -1, -1)
    return labels == 0, labels, rows[order]


def leave_one_out(a, b, n0, n1, min_degree=(1, 1)):
    """core/connected.py:503-557 `_leave_one_out` (after `_nb_peel` when
    min_degree is given, as `_find_components` does at :429-447): the largest
    component by rows, workers (first dimension) seen once removed, then
    every worker that is an articulation point removed, the largest piece
    kept, until none is left.  Returns (alive (n0 + n1) bool, rows alive,
    counts dict)."""
    lib_ = lib()
    keys, counts = distinct_pairs(a, b, n1)
    n1u = ctypes.c_uint64(max(n1, 1))
    nv = n0 + n1
    alive = np.ones(nv, np.uint8)
    if tuple(min_degree) != (1, 1):
        a0, a1 = np.ones(n0, np.uint8), np.ones(n1, np.uint8)
        peel(keys, n1, min_degree[0], min_degree[1], a0, a1)
        alive[:n0], alive[n0:] = a0, a1
    indptr = np.zeros(nv + 1, np.int64)
    lib_.orc_pairs_csr(_p(keys), _i(len(keys)), n1u, _i(n0), _p(alive), _i(nv), _p(indptr), None)
    indices = np.empty(max(int(indptr[-1]), 1), np.int64)
    lib_.orc_pairs_csr(_p(keys), _i(len(keys)), n1u, _i(n0), _p(alive), _i(nv), _p(indptr),
                       _p(indices))
    label = np.empty(nv, np.int64)

    def keep_largest():
        nc = int(lib_.orc_bfs_components(_p(indptr), _p(indices), _i(nv), _p(alive), _p(label)))
        if nc == 0:
            return 0
        size = np.zeros(nc, np.int64)
        lib_.orc_pair_rows(_p(keys), _p(counts), _i(len(keys)), n1u, _p(label), _i(nv),
                           _p(size))
        alive[:] = alive & (label == int(np.argmax(size)))
        return nc

    out = {"components_before": keep_largest()}
    rows0 = np.zeros(n0, np.int64)
    lib_.orc_level_rows(_p(keys), _p(counts), _i(len(keys)), n1u, _p(alive), _i(n0), _p(rows0))
    single = (rows0 == 1) & (alive[:n0] != 0)
    out["single_observation"] = int(single.sum())
    if out["single_observation"]:
        alive[:n0] &= ~single
        keep_largest()
    cut_total, rounds = 0, 0
    is_cut = np.zeros(nv, np.uint8)
    while True:
        is_cut[:] = 0
        lib_.orc_articulation_points(_p(indptr), _p(indices), _i(nv), _p(is_cut), _p(alive))
        cut = (is_cut[:n0] != 0) & (alive[:n0] != 0)
        n_cut = int(cut.sum())
        if not n_cut:
            break
        cut_total += n_cut
        rounds += 1
        alive[:n0] &= ~cut
        keep_largest()
    out.update(cut=cut_total, rounds=rounds)
    lab = np.where(alive != 0, 0, -1).astype(np.int64)
    rows = np.zeros(1, np.int64)
    lib_.orc_pair_rows(_p(keys), _p(counts), _i(len(keys)), n1u, _p(lab), _i(nv), _p(rows))
    return alive != 0, int(rows[0]), out



# ------------------------------------------------ steps 3-4 of a fit

def residual_moments(starts, codes, offs, w, V, Gamma):
    """core/kernels_base.py:114-146 `_nb_residualize_rows` then
    core/inference.py:109-135 `_assemble` (row assembly): V' W V of the
    variables less their fixed-effect projections and weighted group means."""
    V = np.array(V, dtype=np.float64)
    codes = np.asarray(codes, dtype=np.int64)
    for d in range(codes.shape[1]):
        V -= Gamma[offs[d] + codes[:, d]]
    sizes = np.diff(starts)
    Wg = np.add.reduceat(w, starts[:-1])
    q = np.add.reduceat(w[:, None] * V, starts[:-1], axis=0) / Wg[:, None]
    V -= np.repeat(q, sizes, axis=0)
    Vs = V * np.sqrt(w)[:, None]
    return Vs.T @ Vs


def row_effects(starts, codes, offs, w, V, Gamma, beta):
    """core/inference.py:454-456 and core/kernels_base.py:544-615 `_nb_pass2`
    for y = V[:, 0], X = V[:, 1:]: (residual per row, the streamed effect per
    group, the first non-streamed effect per row, gam_y)."""
    codes = np.asarray(codes, dtype=np.int64)
    gam_y = Gamma[:, 0] - Gamma[:, 1:] @ beta
    u = V[:, 0] - V[:, 1:] @ beta
    for d in range(codes.shape[1]):
        u = u - gam_y[offs[d] + codes[:, d]]
    Wg = np.add.reduceat(w, starts[:-1])
    alpha = np.add.reduceat(w * u, starts[:-1]) / Wg
    e = u - np.repeat(alpha, np.diff(starts))
    return e, alpha, gam_y[offs[0] + codes[:, 0]], gam_y


def variance_sums(starts, codes, offs, w, V, Gamma, beta):
    """core/kernels_base.py:544-615 `_nb_pass2` with the sums
    core/inference.py:566-578 takes of its output (OLS, analytic weights):
    (bread sum w h h', meat sum (w e)^2 h h', meat of the streamed groups'
    scores sum_g s_g s_g' with s_g the group's sum of w e h, rss), h the
    residualised covariates."""
    codes = np.asarray(codes, dtype=np.int64)
    X = np.asarray(V[:, 1:], dtype=np.float64)
    H = X.copy()
    for d in range(codes.shape[1]):
        H -= Gamma[offs[d] + codes[:, d], 1:]
    Wg = np.add.reduceat(w, starts[:-1])
    mh = np.add.reduceat(w[:, None] * H, starts[:-1], axis=0) / Wg[:, None]
    H -= np.repeat(mh, np.diff(starts), axis=0)
    e, _, _, _ = row_effects(starts, codes, offs, w, V, Gamma, beta)
    sw = np.sqrt(w)
    B = (H * sw[:, None]).T @ (H * sw[:, None])
    he = H * (w * e)[:, None]
    sg = np.add.reduceat(he, starts[:-1], axis=0)
    return B, he.T @ he, sg.T @ sg, float(w @ (e * e))


def row_scores(starts, codes, offs, w, V, Gamma, beta, with_h=False):
    """The per-row scores w e h of core/inference.py:594-603 (`he`), the
    rows pass 2 sums per cluster; with_h: (he, h)."""
    codes = np.asarray(codes, dtype=np.int64)
    H = np.asarray(V[:, 1:], dtype=np.float64).copy()
    for d in range(codes.shape[1]):
        H -= Gamma[offs[d] + codes[:, d], 1:]
    Wg = np.add.reduceat(w, starts[:-1])
    H -= np.repeat(np.add.reduceat(w[:, None] * H, starts[:-1], axis=0) / Wg[:, None],
                   np.diff(starts), axis=0)
    e, _, _, _ = row_effects(starts, codes, offs, w, V, Gamma, beta)
    he = H * (w * e)[:, None]
    return (he, H) if with_h else he


def crv3_jack(code, w, H, he, B):
    """core/kernels_base.py:658-680 `_nb_crv3_scatter` and `_nb_crv3_finish`:
    the sum over clusters of d_g d_g', d_g = pinv(B - A_g) s_g with A_g the
    cluster's sum of w h h' and s_g its sum of w e h."""
    code = np.asarray(code, np.int64)
    G, k = int(code.max()) + 1, H.shape[1]
    AG = np.zeros((G, k, k))
    np.add.at(AG, code, w[:, None, None] * H[:, :, None] * H[:, None, :])
    sG = np.zeros((G, k))
    np.add.at(sG, code, he)
    acc = np.zeros((k, k))
    for g in range(G):
        d = np.linalg.pinv(B - AG[g]) @ sG[g]
        acc += np.outer(d, d)
    return acc


def cluster_variances(he, gcode, codes, n_levels, Binv, requests, names, pair_components,
                      extra=None):
    """CRV1 variances of beta for cluster requests (core/inference.py:176-240
    `_resolve_clusters`: "a" one term, "a^b" one term of the combinations,
    "a+b" the terms a, b, a^b with signs + + -; :242-269 `_nested_dims`;
    :886-906 the variance with G the smallest one-way count, K less the
    nested dimensions' levels plus one each, core/estimator.py:446-464
    `_k_fe` "exact" skipping pairs of two nested dimensions).  names: the
    streamed dimension first, then the others; pair_components keyed by
    (name, name); extra: name -> per-row integer codes.  Returns
    {request: (V, G list, adj, nested)}."""
    from itertools import combinations
    N, k = he.shape
    codes = np.asarray(codes, np.int64)
    g0 = names[0]
    col = {g0: np.asarray(gcode, np.int64)}
    for d in range(codes.shape[1]):
        col[names[d + 1]] = codes[:, d]
    for name, c in (extra or {}).items():
        col[name] = np.asarray(c, np.int64)
    params = {g0: int(col[g0].max()) + 1}
    for d in range(codes.shape[1]):
        params[names[d + 1]] = int(n_levels[d])

    def term(cols):
        cs = set(cols)
        if len(cols) == 1 and cols[0] in params:
            code = col[cols[0]]
            G = params[cols[0]]
            kind = "seg" if cols[0] == g0 else "fe"
        else:
            key = np.zeros(N, np.int64)
            for c in cols:
                key = key * (int(col[c].max()) + 1) + col[c]
            _, code = np.unique(key, return_inverse=True)
            G = int(code.max()) + 1
            kind = "segsub" if g0 in cs else "extra"
        sums = np.zeros((G, k))
        np.add.at(sums, code, he)
        nested = []
        for d in params:
            if cs <= {d}:
                nested.append(d)
            elif kind != "segsub":
                lo = np.full(params[d], np.iinfo(np.int64).max)
                hi = np.full(params[d], -1)
                np.minimum.at(lo, col[d], code)
                np.maximum.at(hi, col[d], code)
                if np.all(lo == hi):
                    nested.append(d)
        return G, sums.T @ sums, nested

    def k_fe(nest):
        comps = max((c for (a, b), c in pair_components.items()
                     if a not in nest or b not in nest), default=1)
        return sum(params.values()) - (comps + len(params) - 2)

    out = {}
    for req in requests:
        parts = [[c.strip() for c in p_.split("^")] for p_ in req.split("+")]
        terms = []
        for r in range(1, len(parts) + 1):
            for combo in combinations(range(len(parts)), r):
                cols = list(dict.fromkeys(c for i in combo for c in parts[i]))
                terms.append((term(cols), (-1) ** (r + 1), r == 1))
        Gs = [t[0] for t, _, single in terms if single]
        nest = list(dict.fromkeys(d for t, _, _ in terms for d in t[2]))
        Kc = k + k_fe(nest) - sum(params[d] for d in nest) + len(nest)
        adj = min(Gs) / (min(Gs) - 1) * (N - 1) / (N - Kc)
        V = sum(sign * adj * (Binv @ t[1] @ Binv) for t, sign, _ in terms)
        out[req] = (V, Gs, adj, nest)
    return out


def variances(B, meat_hc, meat_g, rss, n_obs, n_groups, n_levels, pair_components):
    """The iid, HC1 and CRV1 (clustered on the streamed dimension) variances
    of beta: core/inference.py:886-912 (pyfixest's small-sample factors) with
    core/estimator.py:446-464 `_k_fe` (fe_dof "exact": the fixed-effect
    parameters less the largest pair's components and one per further
    dimension; the streamed dimension's levels nested in its own clusters,
    so CRV1 counts one parameter for them)."""
    k = B.shape[0]
    G, N = int(n_groups), float(n_obs)
    k_fe = G + int(sum(n_levels)) - (max(pair_components) + len(n_levels) - 1)
    K = k + k_fe
    Binv = np.linalg.inv(B)
    Kc = k + k_fe - G + 1
    adj = G / (G - 1) * (N - 1) / (N - Kc)
    return {"iid": rss / (N - K) * Binv, "hetero": N / (N - K) * Binv @ meat_hc @ Binv,
            "CRV1": adj * Binv @ meat_g @ Binv, "k_fe": k_fe, "df_resid": N - K,
            "df_cluster": G - 1}


def leave_out_match(rows, n_draws, block, seed, tol=1e-12, se=False, se_variance="person_year",
                    se_draws=None, smooth_bins=None):
    """leaveout_match.py:156-214 `leave_out_match`, point estimates: the
    row-level fit's partialled outcome y~ = fe_alpha + fe_psi + resid
    (:76-77), collapsed to one row per (streamed level, psi level) match with
    its weighted mean and total weight (:63-88), the weighted match-level fit
    y~ ~ 1 | alpha + psi, and leaveout.py:634-805 on it with centering
    "reference" (:949-1016: (sqrt(w) ybar - its mean over matches) sqrt(w) e
    / M times the JLA factor), the stayers' matches given
    `sigma_for_stayers` (:91-132) and the n - 1 divisor counting
    person-years.  psi = the first non-streamed dimension."""
    c = pass1(rows)
    S = build_explicit(c)
    Gamma, _ = solve(c, S, tol=tol)
    starts = row_starts(rows.gcode)
    codes = np.asarray(rows.codes, np.int64)
    N = rows.n_rows
    w = rows.w if rows.w is not None else np.ones(N)
    A = residual_moments(starts, codes, c.offs, w, rows.V, Gamma)
    beta = np.linalg.solve(A[1:, 1:], A[1:, 0]) if A.shape[0] > 1 else np.zeros(0)
    e, alpha_g, psi_row, _ = row_effects(starts, codes, c.offs, w, rows.V, Gamma, beta)
    y_t = np.repeat(alpha_g, np.diff(starts)) + psi_row + e
    g, f = rows.gcode.astype(np.int64), codes[:, 0]
    head = np.concatenate(([True], (g[1:] != g[:-1]) | (f[1:] != f[:-1])))
    match = np.cumsum(head) - 1
    W_m = np.bincount(match, weights=w)
    Y_m = np.bincount(match, weights=w * y_t) / W_m
    first = np.flatnonzero(head)
    mrows = type(rows)(gcode=rows.gcode[first], codes=np.ascontiguousarray(rows.codes[first, :1]),
                       V=Y_m[:, None], w=W_m, n_levels=[int(rows.n_levels[0])],
                       n_groups=rows.n_groups, names=[rows.names[0]])
    cm = pass1(mrows)
    Sm = build_explicit(cm)
    gm, _ = solve(cm, Sm, tol=tol)
    des = Design(mrows, cm, Sm, tol=tol)
    sm_ = des.starts
    cm_codes = np.asarray(mrows.codes, np.int64)
    e_m, alpha_m, psi_m, _ = row_effects(sm_, cm_codes, cm.offs, W_m, mrows.V, gm, np.zeros(0))
    a_m = np.repeat(alpha_m, np.diff(sm_))
    T = W_m.sum()
    R = float(N)
    scale = T / (T * (R - 1.0) / R) if R > 1 else 1.0
    ma, mb = (W_m @ psi_m) / T, (W_m @ a_m) / T
    plug_in = np.array([scale * ((W_m @ (psi_m * psi_m)) / T - ma * ma),
                        scale * ((W_m @ (a_m * a_m)) / T - mb * mb),
                        scale * ((W_m @ (psi_m * a_m)) / T - ma * mb)])
    lev, comp, factor = des.jla_leverages(n_draws, block, seed)
    root = np.sqrt(W_m)
    yt = root * Y_m
    with np.errstate(divide="ignore", invalid="ignore"):     # stayers: replaced below
        sigma2 = (yt - yt.mean()) * root * e_m / comp * factor
    # the stayers' matches: leaveout_match.py:91-132 `stayer_sigma2`
    gm_codes = mrows.gcode.astype(np.int64)
    stayer = np.bincount(gm_codes)[gm_codes] == 1
    fitted = Y_m - e_m
    worker_w = np.bincount(g, weights=w)
    y_mean = (w @ y_t) / w.sum()
    r = (y_t - y_mean) * (y_t - fitted[match]) / (1.0 - w / worker_w[g])
    stay = np.bincount(match, weights=w * w * r) / W_m
    sigma2 = np.where(stayer, stay, sigma2)
    bias = des.hutchinson_trace(sigma2, n_draws, block, seed + 1_000_003, person_years=R)
    out = {"plug_in": plug_in, "bias": bias, "leave_out": plug_in - bias, "sigma2": sigma2,
           "n_matches": len(W_m), "stayer_matches": int(stayer.sum()), "person_years": N,
           "max_leverage": float(lev[~stayer].max()) if (~stayer).any() else 0.0}
    if not se:
        return out
    # leaveout.py:848-894 `_match_se_sigma2`: the weighted-centred
    # leave-match-out sigma2 of the movers' matches (:949-1016)
    movers = ~stayer
    y_bar = (W_m @ Y_m) / W_m.sum()
    with np.errstate(divide="ignore", invalid="ignore"):
        block_s2 = np.where(movers, W_m * (Y_m - y_bar) * e_m / comp * factor, np.nan)
    if se_variance == "match":
        sigma2_se = np.where(stayer, stay, block_s2)
    elif se_variance == "person_year":
        if rows.w is not None:
            raise ValueError("se_variance='person_year' has no user weights; use 'match'")
        # leaveout_match.py:135-153 `within_match_variance`
        within = np.bincount(match, weights=(y_t - Y_m[match]) ** 2) / np.bincount(match)
        sigma2_se = np.where(movers, within + block_s2 / W_m, within)
    else:
        raise ValueError("se_variance must be 'match' or 'person_year'")
    # leaveout.py:760-772: component_variances on the match rows, seed +
    # 5_500_011, stayers' b zeroed, reference centring, var(alpha) unreported
    des.person_years = R
    se_seed = seed + 5_500_011
    draws = n_draws if se_draws is None else int(se_draws)
    b_ii = des.bii_rows(draws, block, se_seed)
    out["se"] = des.component_variances(sigma2_se, lev, comp, factor, b_ii, draws, block,
                                        se_seed, smooth_bins, stayer_rows=stayer,
                                        centering="reference", reported=(0, 2))
    out["sigma2_se"] = sigma2_se
    out["b_ii"] = b_ii
    return out


# ------------------------------------------------ KSS standard-error pieces

def readout(starts, codes, offs, X, U_l, U_c, U_g):
    """kernels_se.py:19-43 `_nb_readout`: (A u)_i = u_g(i) + sum_d
    u_levels[level_d(i)] + x_i' u_cov, rows (N, m)."""
    codes = np.asarray(codes, np.int64)
    out = np.repeat(np.asarray(U_g, float), np.diff(starts), axis=0)
    for d in range(codes.shape[1]):
        out = out + U_l[offs[d] + codes[:, d]]
    for c in range(X.shape[1]):
        out = out + X[:, c:c + 1] * U_c[c][None, :]
    return out


def cov_cross(starts, codes, psi_column, psi_offset, w, U_l, U_g, L):
    """kernels_se.py:46-77 `_nb_cov_cross`: (acc (L, m): per psi level the sum
    of w_i u_streamed[g(i)]; out_groups (G, m): per group the sum of w_i
    u_levels[psi(i)])."""
    lev = psi_offset + np.asarray(codes, np.int64)[:, psi_column]
    ug = np.repeat(np.asarray(U_g, float), np.diff(starts), axis=0)
    m = ug.shape[1]
    acc = np.zeros((L, m))
    for j in range(m):
        acc[:, j] = np.bincount(lev, weights=w * ug[:, j], minlength=L)
    return acc, np.add.reduceat(w[:, None] * U_l[lev], starts[:-1], axis=0)


SMOOTH_QUANTILE_SAMPLE = 2_000_000


def _smooth_bins(n, dims):
    """leaveout_se.py:955-964 `_auto_bins`: n^(1/6) bins per axis in two
    dimensions (n^(1/3) in one), clipped to 2..500."""
    power = 1.0 / 6.0 if dims == 2 else 1.0 / 3.0
    return int(np.clip(round(n ** power), 2, 500))


def _smooth_knots(values, n_bins, take):
    """leaveout_se.py:967-973 `_knots`: strictly increasing quantile knots."""
    q = np.quantile(np.asarray(values[take], dtype=np.float64),
                    np.linspace(0.0, 1.0, n_bins + 1))
    q = np.maximum.accumulate(q)
    span = max(float(q[-1] - q[0]), 1e-300)
    return q + np.arange(len(q)) * span * 1e-12


def _smooth_rank(knots, values):
    """leaveout_se.py:976-979 `_rank`: piecewise-linear map to [0, 1]."""
    return np.interp(np.asarray(values, dtype=np.float64), knots,
                     np.linspace(0.0, 1.0, len(knots)))


def fit_smoother(sigma2, leverage, b_ii=None, n_bins=None):
    """leaveout_se.py:982-1035 `fit_smoother`: sigma2 averaged over a grid of
    cells in the empirical quantiles of (P_ii, B_ii); (knots, means, bins)."""
    n = len(sigma2)
    dims = 1 if b_ii is None else 2
    n_bins = _smooth_bins(n, dims) if n_bins is None else int(n_bins)
    if n_bins < 1:
        return None
    rng = np.random.default_rng(0)
    take = (np.arange(n) if n <= SMOOTH_QUANTILE_SAMPLE
            else np.sort(rng.choice(n, SMOOTH_QUANTILE_SAMPLE, replace=False)))
    knots = (_smooth_knots(leverage, n_bins, take),
             None if b_ii is None else _smooth_knots(b_ii, n_bins, take))
    shape = (n_bins,) * dims
    cells = [np.minimum((_smooth_rank(knots[0], leverage) * n_bins).astype(np.int64),
                        n_bins - 1)]
    if b_ii is not None:
        cells.append(np.minimum((_smooth_rank(knots[1], b_ii) * n_bins).astype(np.int64),
                                n_bins - 1))
    flat = np.ravel_multi_index(cells, shape)
    totals = np.bincount(flat, weights=np.asarray(sigma2, float),
                         minlength=int(np.prod(shape))).reshape(shape)
    counts = np.bincount(flat, minlength=int(np.prod(shape))).reshape(shape)
    overall = float(totals.sum() / max(counts.sum(), 1.0))
    means = np.where(counts > 0, totals / np.maximum(counts, 1.0), overall)
    return knots, means, n_bins


def smooth_eval(table, leverage, b_ii=None):
    """leaveout_se.py:1038-1054 `smooth_eval`: bilinear between cell centres."""
    knots, means, n_bins = table

    def weights(values, k):
        f = _smooth_rank(knots[k], values) * n_bins - 0.5
        j0 = np.clip(np.floor(f).astype(np.int64), 0, n_bins - 2)
        return j0, np.clip(f - j0, 0.0, 1.0)
    i0, a = weights(leverage, 0)
    if knots[1] is None:
        return (1.0 - a) * means[i0] + a * means[i0 + 1]
    j0, b = weights(b_ii, 1)
    return ((1.0 - a) * (1.0 - b) * means[i0, j0] + a * (1.0 - b) * means[i0 + 1, j0]
            + (1.0 - a) * b * means[i0, j0 + 1] + a * b * means[i0 + 1, j0 + 1])


# ------------------------------------------------- inverse operator, JLA

class Design:
    """Row-level view the inverse operator needs: group boundaries of the
    rows, their level codes, weights (ones when unweighted) and covariates
    (inverse.py:105-160 `_chunks`, `_covariate_matrix`)."""

    def __init__(self, rows, cells, S, X=None, tol=1e-10, nt=1):
        self.rows, self.cells, self.S, self.tol, self.nt = rows, cells, S, tol, nt
        self.starts = row_starts(rows.gcode)
        self.codes = rows.codes
        self.w = rows.w if rows.w is not None else np.ones(rows.n_rows)
        self.X = np.zeros((rows.n_rows, 0)) if X is None else np.ascontiguousarray(X, np.float64)
        self.dinv = jacobi(cells.diag)
        self._border = None
        # leaveout_se.py:216-220 `_person_years`: the rows behind the fit when
        # each row is a match (None: the rows themselves)
        self.person_years = None

    def solve_reduced(self, rhs, scale):
        """inverse.py:86-103 `_solve_reduced`: zero columns, then the PCG."""
        rhs = np.ascontiguousarray(rhs)
        zero = np.linalg.norm(rhs, axis=0) <= RHS_ZERO_TOL * np.asarray(scale)
        U, *_ = pcg(self.S, self.dinv, rhs, zero, None, self.tol)
        return U

    def border(self):
        """inverse.py:182-218 `_border` (and `_reduce_design`)."""
        if self._border is None:
            c = self.X.shape[1]
            if c == 0:
                self._border = (None, None)
            else:
                T_dx, T_xx = center_rows(self.starts, self.codes, self.cells.offs, self.w,
                                         self.X, self.X, self.cells.L, self.nt)
                scale = np.sqrt(self.w @ (self.X * self.X))
                Z = self.solve_reduced(T_dx, scale)
                schur = T_xx - T_dx.T @ Z
                self._border = (Z, np.linalg.pinv(schur, hermitian=True))
        return self._border

    def project_rows(self, n_vec, seed, first_draw=0, sqrt_weights=False):
        """inverse.py:240-309 `project_rows` for Rademacher vectors: the rows'
        (A S^- A' r_j)_i, all rows in one chunk."""
        N = self.rows.n_rows
        R = rademacher(0, N, n_vec, seed, first_draw)
        if sqrt_weights:
            root = np.sqrt(self.w)
            inv = np.divide(1.0, root, out=np.zeros_like(root), where=root > 0)
            R = R * inv[:, None]
        Z, schur_inv = self.border()
        rhs, rhs_x = center_rows(self.starts, self.codes, self.cells.offs, self.w, self.X, R,
                                 self.cells.L, self.nt)
        scale = np.sqrt(self.w @ (R * R))
        U = self.solve_reduced(rhs, scale)
        if Z is not None:
            C = schur_inv @ (rhs_x - Z.T @ rhs)
            U = U - Z @ C
        else:
            C = np.zeros((0, n_vec))
        out = project_rows_kernel(self.starts, self.codes, self.cells.offs, self.w, self.X, C,
                                  R, U)
        return out * root[:, None] if sqrt_weights else out

    # ---- coefficient-space right-hand sides (inverse.py:311-460)

    def null_space(self):
        """inverse.py:376-428 `_null_space`: an orthonormal basis of S's null
        space in (streamed, levels) blocks -- per connected component, +1 on
        its groups and -1 on its levels of the first non-streamed dimension;
        per further dimension, +1 across the first and -1 across it."""
        if getattr(self, "_null", None) is None:
            cells, starts = self.cells, self.starts
            G, L = len(starts) - 1, cells.L
            D = len(cells.n_levels)
            comp, _ = component_labels(cells)
            n_comp = int(comp.max()) + 1 if len(comp) else 0
            # inverse.py:430-437 `_group_components`: the component of each
            # group's first row's first-dimension level
            gcomp = comp[self.codes[starts[:-1], 0].astype(np.int64)]
            off = cells.offs
            vecs = []
            for c in range(n_comp):
                lv = np.zeros(L)
                lv[off[0]:off[0] + cells.n_levels[0]] = -(comp == c).astype(float)
                vecs.append(np.concatenate([(gcomp == c).astype(float), lv]))
            for d in range(1, D):
                lv = np.zeros(L)
                lv[off[0]:off[0] + cells.n_levels[0]] = 1.0
                lv[off[d]:off[d] + cells.n_levels[d]] = -1.0
                vecs.append(np.concatenate([np.zeros(G), lv]))
            if vecs:
                q, _ = np.linalg.qr(np.column_stack(vecs))
            else:
                q = np.zeros((G + L, 0))
            self._null = (q[:G], q[G:])
        return self._null

    def drop_null(self, levels, streamed):
        """inverse.py:445-460 `_drop_null_component`."""
        qs, ql = self.null_space()
        if ql.shape[1] == 0:
            return levels, streamed
        overlap = qs.T @ streamed + ql.T @ levels
        return levels - ql @ overlap, streamed - qs @ overlap

    def apply_inverse(self, levels, cov_values, streamed, row_weights=None):
        """inverse.py:311-374 `apply_inverse`: (U_levels, C, U_streamed, rows)
        for a coefficient-space right-hand side; rows = (A u)_i.  With
        row_weights, also the collect sink of leaveout.py:423-431: v = A' Omega
        rows as (v_levels, v_cov, v_groups)."""
        cells, starts = self.cells, self.starts
        B = levels.shape[1]
        Z, schur_inv = self.border()
        levels, streamed = self.drop_null(np.asarray(levels, float), np.asarray(streamed, float))
        scale = np.sqrt((levels * levels).sum(axis=0) + (streamed * streamed).sum(axis=0))
        rho = spread_groups(starts, self.w, streamed)
        acc, acc_x = reduce_rows(starts, self.codes, cells.offs, self.w, self.X, rho, cells.L,
                                 self.nt)
        rhs = levels - acc
        rhs_x = np.asarray(cov_values, float) - acc_x
        U = self.solve_reduced(rhs, scale)
        if Z is not None:
            C = schur_inv @ (rhs_x - Z.T @ rhs)
            U = U - Z @ C
        else:
            C = np.zeros((0, B))
        rows, groups = project_coef(starts, self.codes, cells.offs, self.w, self.X, C, rho, U)
        out = (U, C, groups, rows)
        if row_weights is not None:
            weighted = rows * np.asarray(row_weights, float)[:, None]
            v, v_x = reduce_rows(starts, self.codes, cells.offs, self.w, self.X, weighted,
                                 cells.L, self.nt)
            out = out + ((v, v_x, group_sums(starts, self.w, weighted)),)
        return out

    def hutchinson_trace(self, sigma2, n_draws, block, seed, psi_column=0, person_years=None):
        """leaveout.py:321-391 `hutchinson_trace` with :393-448
        `_trace_block`: the bias terms (var(psi), var(alpha), cov);
        person_years the divisor's count when the rows are matches
        (leaveout_se.py:216-220 `_person_years`)."""
        cells, starts = self.cells, self.starts
        G, L, c = len(starts) - 1, cells.L, self.X.shape[1]
        totals = np.zeros(8)
        drawn = 0
        while drawn < n_draws:
            size = min(block, n_draws - drawn)
            Zall = rademacher(0, L + G + c, size, seed, drawn)
            Zl, Zg, Zc = Zall[:L], Zall[L:L + G], Zall[L + G:]
            *_, (vl, vx, vg) = self.apply_inverse(Zl, Zc, Zg, row_weights=sigma2)
            Ul, _, Ug, _ = self.apply_inverse(vl, vx, vg)
            totals += trace_moments(starts, self.codes, psi_column, int(cells.offs[psi_column]),
                                    self.w, Zl, Zg, Ul, Ug, self.nt).sum(axis=(0, 1))
            drawn += size
        weight, a1a2, b1b2, cross, a1, a2, b1, b2 = totals / n_draws
        var_psi = a1a2 / weight - (a1 / weight) * (a2 / weight)
        var_alpha = b1b2 / weight - (b1 / weight) * (b2 / weight)
        cov = 0.5 * (cross / weight - (a1 / weight) * (b2 / weight) - (b1 / weight) * (a2 / weight))
        # leaveout_se.py:202-214 `_moment_divisor`: n - 1 person-years
        R = float(self.rows.n_rows if person_years is None else person_years)
        scale = weight / (weight * (R - 1.0) / R) if R > 1 else 1.0
        return np.array([scale * var_psi, scale * var_alpha, scale * cov])

    def leave_out_components(self, Gamma, n_draws, block, seed):
        """leaveout.py:634-805 `leave_out_components` (point estimates;
        stayers "own", weighted centring): the plug-in var(psi), var(alpha),
        cov(psi, alpha) (:807-833), sigma2 from the leverages and residuals
        (:949-1016), the Hutchinson bias (seed + 1_000_003) and their
        difference.  psi = the first non-streamed dimension."""
        rows, cells, starts = self.rows, self.cells, self.starts
        w = self.w
        A = residual_moments(starts, self.codes, cells.offs, w, rows.V, Gamma)
        beta = np.linalg.solve(A[1:, 1:], A[1:, 0])
        e, alpha_g, psi_row, _ = row_effects(starts, self.codes, cells.offs, w, rows.V, Gamma,
                                             beta)
        alpha_row = np.repeat(alpha_g, np.diff(starts))
        T = w.sum()
        R = float(rows.n_rows)
        scale = T / (T * (R - 1.0) / R) if R > 1 else 1.0
        ma, mb = (w @ psi_row) / T, (w @ alpha_row) / T
        plug_in = np.array([scale * ((w @ (psi_row * psi_row)) / T - ma * ma),
                            scale * ((w @ (alpha_row * alpha_row)) / T - mb * mb),
                            scale * ((w @ (psi_row * alpha_row)) / T - ma * mb)])
        lev, comp, factor = self.jla_leverages(n_draws, block, seed)
        y = rows.V[:, 0]
        ybar = float(w @ y / T)
        sigma2 = w * (y - ybar) * e / comp * factor
        bias = self.hutchinson_trace(sigma2, n_draws, block, seed + 1_000_003)
        return {"plug_in": plug_in, "bias": bias, "leave_out": plug_in - bias, "beta": beta,
                "sigma2": sigma2, "max_leverage": float(lev.max()), "leverage": lev,
                "complement": comp, "factor": factor}

    # ---- KSS standard errors (leaveout_se.py), weighted centring

    def se_layout(self):
        """leaveout_se.py:135-180 `_level_weight_totals` / `_se_layout`:
        (per-level weight totals, per-group totals, total, the n - 1 divisor
        `_moment_divisor`, the psi dimension's slice of the levels)."""
        cells, starts = self.cells, self.starts
        L = cells.L
        codes = np.asarray(self.codes, np.int64)
        lw = np.zeros(L)
        for d in range(codes.shape[1]):
            lw += np.bincount(cells.offs[d] + codes[:, d], weights=self.w, minlength=L)
        gw = np.add.reduceat(self.w, starts[:-1])
        total = float(gw.sum())
        R = float(self.rows.n_rows if self.person_years is None else self.person_years)
        norm = total * (R - 1.0) / R if R > 1 else total
        psi = slice(int(cells.offs[0]), int(cells.offs[0]) + int(cells.n_levels[0]))
        return lw, gw, total, norm, psi

    def _roots(self):
        root = np.sqrt(self.w)
        return root, np.divide(1.0, root, out=np.zeros_like(root), where=root > 0)

    def _to_coef(self, R):
        """A' W R as (levels, covariates, groups): `_nb_reduce_rows` and
        `_nb_group_sums` on explicit rows."""
        cells, starts = self.cells, self.starts
        acc, acc_x = reduce_rows(starts, self.codes, cells.offs, self.w, self.X, R, cells.L,
                                 self.nt)
        return acc, acc_x, group_sums(starts, self.w, R)

    def bii_rows(self, n_draws, block, seed):
        """leaveout_se.py:228-327 `bii_rows`: B_ii of var(psi), var(alpha)
        and cov per row, (3, N), by random projection (one pair of solves per
        draw)."""
        lw, gw, total, norm, psi = self.se_layout()
        N, L, G, c = self.rows.n_rows, self.cells.L, len(self.starts) - 1, self.X.shape[1]
        root, inv = self._roots()
        root_total = np.sqrt(norm)
        out = np.zeros((3, N))
        drawn = 0
        while drawn < n_draws:
            size = min(block, n_draws - drawn)
            q = rademacher(0, N, size, seed, drawn) * inv[:, None]
            levels, _, gsum = self._to_coef(q)
            grand = levels[psi].sum(axis=0) / total
            rhs_l = np.zeros((L, 2 * size))
            rhs_l[psi, :size] = (levels[psi] - np.outer(lw[psi], grand)) / root_total
            rhs_g = np.zeros((G, 2 * size))
            rhs_g[:, size:] = (gsum - np.outer(gw, grand)) / root_total
            U_l, U_c, U_g, _ = self.apply_inverse(rhs_l, np.zeros((c, 2 * size)), rhs_g)
            rows = readout(self.starts, self.codes, self.cells.offs, self.X, U_l, U_c, U_g)
            x, y = root[:, None] * rows[:, :size], root[:, None] * rows[:, size:]
            out[0] += (x * x).sum(axis=1)
            out[1] += (y * y).sum(axis=1)
            out[2] += (x * y).sum(axis=1)
            drawn += size
        return out / n_draws

    def apply_q(self, k, U_l, U_g, layout):
        """leaveout_se.py:339-385 `_apply_q`: Q_k u in coefficient space
        (k = 0 var(psi), 1 var(alpha), 2 cov, the last with a row sweep)."""
        lw, gw, total, norm, psi = layout
        L, G = self.cells.L, len(self.starts) - 1
        m = U_l.shape[1]
        out_l, out_g = np.zeros((L, m)), np.zeros((G, m))
        level_w, base = lw[psi], U_l[psi]
        psi_mean = (level_w @ base) / total
        alpha_mean = (gw @ U_g) / total
        if k == 0:
            out_l[psi] = level_w[:, None] * (base - psi_mean) / norm
        elif k == 1:
            out_g[:] = gw[:, None] * (U_g - alpha_mean) / norm
        else:
            cross_l, cross_g = cov_cross(self.starts, self.codes, 0, int(self.cells.offs[0]),
                                         self.w, U_l, U_g, L)
            out_l[psi] = (cross_l[psi] - level_w[:, None] * alpha_mean) / (2 * norm)
            out_g[:] = (cross_g - gw[:, None] * psi_mean) / (2 * norm)
        return out_l, out_g

    def m_times(self, b):
        """leaveout_se.py:387-424 `_m_times`: u_k = M b_k for the three
        rows of b (3, N), one solve for all three."""
        root, inv = self._roots()
        levels, cov_block, gsum = self._to_coef(np.ascontiguousarray(b.T) * inv[:, None])
        U_l, U_c, U_g, _ = self.apply_inverse(levels, cov_block, gsum)
        base = readout(self.starts, self.codes, self.cells.offs, self.X, U_l, U_c, U_g)
        return b - (root[:, None] * base).T

    def apply_c(self, v, b, per_component, layout, rank_two=None, deflate=None):
        """leaveout_se.py:426-597 `_apply_c`: C v = B v - (b .* M v +
        M (b .* v)) / 2 for each component, v (N, size) shared or (N, 3, size)
        one per component; (N, 3, size).  rank_two = (u (3, N), scale) adds
        scale (1 u_k' + u_k 1') v (:536-543, :591-595); deflate = (lambda (3,),
        x1 (N, 3)) takes lambda_k x1_k x1_k' v off B v (:532-535, :580-582)."""
        N, L, G, c = self.rows.n_rows, self.cells.L, len(self.starts) - 1, self.X.shape[1]
        n_in = 3 if per_component else 1
        size = v.shape[-1]
        root, inv = self._roots()

        def part(k):
            return v[:, k, :] if per_component else v

        def in_cols(k):
            j = k if per_component else 0
            return slice(j * size, (j + 1) * size)

        def b_cols(k):
            return slice((n_in + k) * size, (n_in + k + 1) * size)
        stack = np.empty((N, (n_in + 3) * size))
        for k in range(n_in):
            stack[:, k * size:(k + 1) * size] = part(k)
        for k in range(3):
            stack[:, b_cols(k)] = part(k) * b[k][:, None]
        levels, cov_block, gsum = self._to_coef(stack * inv[:, None])
        U0_l, U0_c, U0_g, _ = self.apply_inverse(levels, cov_block, gsum)
        q_l, q_g = np.zeros((L, 3 * size)), np.zeros((G, 3 * size))
        for k in range(3):
            cols = slice(k * size, (k + 1) * size)
            q_l[:, cols], q_g[:, cols] = self.apply_q(k, U0_l[:, in_cols(k)],
                                                      U0_g[:, in_cols(k)], layout)
        U1_l, U1_c, U1_g, _ = self.apply_inverse(q_l, np.zeros((c, 3 * size)), q_g)
        offs = self.cells.offs
        base = readout(self.starts, self.codes, offs, self.X, U0_l, U0_c, U0_g)
        through_q = readout(self.starts, self.codes, offs, self.X, U1_l, U1_c, U1_g)
        cv = np.empty((N, 3, size))
        for k in range(3):
            vk = part(k)
            Mv = vk - root[:, None] * base[:, in_cols(k)]
            Bv = root[:, None] * through_q[:, k * size:(k + 1) * size]
            if deflate is not None:
                lams, x1 = deflate
                Bv = Bv - lams[k] * np.outer(x1[:, k], x1[:, k] @ vk)
            M_bv = vk * b[k][:, None] - root[:, None] * base[:, b_cols(k)]
            cv[:, k, :] = Bv - 0.5 * (b[k][:, None] * Mv + M_bv)
            if rank_two is not None:
                u, scale = rank_two
                cv[:, k, :] += scale * ((u[k] @ vk)[None, :] + np.outer(u[k], vk.sum(axis=0)))
        return cv

    def component_variances(self, sigma2, leverage, complement, factor, b_ii, n_draws,
                            block, seed, smooth_bins=None, stayer_rows=None,
                            centering="weighted", reported=(0, 1, 2), weak_id=None,
                            weak_components=None, sigma2_point=None):
        """leaveout_se.py:599-784 `component_variances` (trace included, no
        weak-identification pieces): per component the first term
        4 sum s~ (C y~)^2, the trace term 2 tr(C Om~ C Om~) by Hutchinson
        draws (seed + 7_700_017), theta = y~' C y~, and variance = first -
        trace term; s~ the smoothed sigma2.  Leaving out matches (:616-636):
        b is zero on `stayer_rows`; centering "reference" applies
        K = C + (1 u' + u 1') / (2 R), u = M b, R the rows, to the uncentred
        sqrt(w) y; components not in `reported` are NaN."""
        layout = self.se_layout()
        with np.errstate(divide="ignore", invalid="ignore"):   # stayers' M_ii = 0
            b = b_ii * (factor / complement)[None, :]
        if stayer_rows is not None:
            b[:, np.asarray(stayer_rows, bool)] = 0.0
        rank_two = None
        if centering == "reference":
            rank_two = (self.m_times(b), 0.5 / self.rows.n_rows)
        elif centering != "weighted":
            raise ValueError("centering must be 'reference' or 'weighted'")
        tables = [fit_smoother(sigma2, leverage, b_ii[k], smooth_bins) for k in range(3)]
        sig = [smooth_eval(t, leverage, b_ii[k]) if t is not None else np.asarray(sigma2)
               for k, t in enumerate(tables)]
        y = self.rows.V[:, 0]
        w = self.w
        y_bar = float(w @ y / w.sum()) if centering == "weighted" else 0.0
        shifted = np.sqrt(w) * (y - y_bar)
        cv = self.apply_c(shifted[:, None], b, False, layout, rank_two)
        first = np.array([4.0 * float(sig[k] @ (cv[:, k, 0] ** 2)) for k in range(3)])
        theta = np.array([float(shifted @ cv[:, k, 0]) for k in range(3)])
        trace = np.zeros(3)
        N = self.rows.n_rows
        drawn = 0
        while drawn < n_draws:
            size = min(block, n_draws - drawn)
            z = rademacher(0, N, size, seed + 7_700_017, drawn)
            v = np.stack([z * np.sqrt(np.maximum(sig[k], 0.0))[:, None] for k in range(3)],
                         axis=1)
            cvt = self.apply_c(v, b, True, layout, rank_two)
            for k in range(3):
                trace[k] += float(sig[k] @ (cvt[:, k, :] ** 2).sum(axis=1))
            drawn += size
        trace /= n_draws
        # :737-759: the q = 1 pieces for the components the diagnostic flags
        weak = None
        if weak_id is not None:
            if weak_components is None:
                weak_components = [k for k in range(3) if weak_id["q"][k] >= 1]
            weak_components = [k for k in weak_components
                               if k in reported and (stayer_rows is None or k == 0)]
            if weak_components:
                weak = self.weak_moments(sigma2 if sigma2_point is None else sigma2_point,
                                         sig, b_ii, complement, factor, weak_id,
                                         weak_components, n_draws, block, seed + 8_800_021,
                                         layout, stayer_rows, centering)
        variance = first - 2.0 * trace
        for k in range(3):
            if k not in reported:
                variance[k] = first[k] = trace[k] = theta[k] = np.nan
        return {"variance": variance, "first_term": first,
                "trace_term": 2.0 * trace, "theta": theta, "weak": weak}

    def weak_moments(self, sigma2, sig, b_ii, complement, factor, weak_id, components, n_draws,
                     block, seed, layout, stayer_rows=None, centering="weighted"):
        """leaveout_se.py:786-888 `_weak_moments`: per flagged component the
        leading direction's estimate b1 = x1' y~ (x1 = sqrt(w) A u1), its raw
        variance sum x1^2 sigma2, and the 2x2 covariance of (b1, theta1) from
        the deflated kernel C2 (B2 = B - lambda_1 x1 x1', b2 from diag(B2)),
        sigma2 smoothed and floored at zero; the first term alone when the
        trace leaves it indefinite."""
        N = self.rows.n_rows
        lams = np.array([float(e[0]) if len(e) else 0.0 for e in weak_id["eigenvalues"]])
        U = weak_id["lead_vectors"]
        root = np.sqrt(self.w)
        x1 = root[:, None] * readout(self.starts, self.codes, self.cells.offs, self.X, U[0],
                                     U[1], U[2])
        y = self.rows.V[:, 0]
        y_bar = float(self.w @ y / self.w.sum())
        yt = root * (y - y_bar)
        flo = [np.maximum(sk, 0.0) for sk in sig]
        b1 = x1.T @ yt
        v_raw = (x1 ** 2).T @ np.asarray(sigma2, float)
        s11 = np.array([(x1[:, k] ** 2) @ flo[k] for k in range(3)])
        with np.errstate(divide="ignore", invalid="ignore"):
            inv_m = factor / complement
        b2 = np.stack([(b_ii[k] - lams[k] * x1[:, k] ** 2) * inv_m for k in range(3)])
        if stayer_rows is not None:
            b2[:, np.asarray(stayer_rows, bool)] = 0.0
        rank_two = (self.m_times(b2), 0.5 / N) if centering == "reference" else None
        shift = y_bar if centering == "weighted" else 0.0
        y_c = root * (y - shift)
        deflate = (lams, x1)
        cv = self.apply_c(y_c[:, None], b2, False, layout, rank_two, deflate)
        s12 = np.array([2.0 * float((x1[:, k] * flo[k]) @ cv[:, k, 0]) for k in range(3)])
        first = np.array([4.0 * float(flo[k] @ (cv[:, k, 0] ** 2)) for k in range(3)])
        quad = np.array([float(y_c @ cv[:, k, 0]) for k in range(3)])
        # :890-930 `_cc_trace` with clamp and only the flagged components drawn
        trace = np.zeros(3)
        drawn = 0
        while drawn < n_draws:
            size = min(block, n_draws - drawn)
            z = rademacher(0, N, size, seed, drawn)
            v = np.zeros((N, 3, size))
            for k in components:
                v[:, k, :] = z * np.sqrt(flo[k])[:, None]
            cvt = self.apply_c(v, b2, True, layout, rank_two, deflate)
            for k in components:
                trace[k] += float(flo[k] @ (cvt[:, k, :] ** 2).sum(axis=1))
            drawn += size
        trace /= n_draws
        out = {}
        for k in components:
            s22 = first[k] - 2.0 * trace[k]
            conservative = not (s22 > 0 and s12[k] ** 2 < s11[k] * s22)
            if conservative:
                s22 = first[k]
            out[k] = {"lambda_1": float(lams[k]), "b1": float(b1[k]), "v_raw": float(v_raw[k]),
                      "sigma": np.array([[s11[k], s12[k]], [s12[k], s22]]),
                      "conservative": bool(conservative), "trace": float(trace[k]),
                      "quadratic": float(quad[k])}
        return out

    def jla_leverages(self, n_draws, block, seed):
        """leaveout.py:130-198 `jla_leverages` and :210-282
        `_combine_moments`: (leverage, complement, factor)."""
        N = self.rows.n_rows
        mom = np.zeros((5, N))
        drawn = 0
        sq = self.rows.w is not None
        while drawn < n_draws:
            size = min(block, n_draws - drawn)
            proj = self.project_rows(size, seed, drawn, sqrt_weights=sq)
            r = rademacher(0, N, size, seed, drawn)
            P = proj ** 2
            M = (r - proj) ** 2
            mom[0] += P.sum(axis=1)
            mom[1] += M.sum(axis=1)
            mom[2] += (P ** 2).sum(axis=1)
            mom[3] += (M ** 2).sum(axis=1)
            mom[4] += (P * M).sum(axis=1)
            drawn += size
        P, M, m_PP, m_MM, m_PM = (m / n_draws for m in mom)
        total = P + M
        P_bar = np.divide(P, total, out=np.zeros_like(P), where=total > 0)
        M_bar = 1.0 - P_bar
        V = (M_bar ** 2 * m_PP + P_bar ** 2 * m_MM - 2 * P_bar * M_bar * m_PM) / n_draws
        B = (M_bar * m_PP - P_bar * m_MM + (M_bar - P_bar) * m_PM) / n_draws
        usable = M_bar > 0
        factor = np.ones_like(M_bar)
        np.divide(V, M_bar ** 2, out=factor, where=usable)
        factor = np.where(usable, 1.0 - factor + np.divide(B, M_bar, out=np.zeros_like(B),
                                                             where=usable), 1.0)
        return P_bar, M_bar, factor


# ------------------------------------------- the weak-identification diagnostic

WEAK_ID_THRESHOLD = 0.1             # leaveout_weakid.py:64 (KSS Section 6.2)


def ritz_top(alpha, beta, top):
    """leaveout_weakid.py:386-434 `_ritz_top`: the leading genuine Ritz values
    of the tridiagonal (alpha, beta[:-1]), their error bounds |beta[-1] s_m|
    and vectors; copies within 1e-8 of the largest merge (the one with the
    smaller bound kept), and a lone value that is also an eigenvalue of the
    tridiagonal without its first row and column (to 1e-11) is spurious
    (Cullum-Willoughby)."""
    from scipy.linalg import eigh_tridiagonal, eigvalsh_tridiagonal
    m = len(alpha)
    if m == 0:
        return np.array([]), np.array([]), np.zeros((0, 0))
    off = np.asarray(beta[:m - 1], float)
    theta, S = eigh_tridiagonal(np.asarray(alpha, float), off)
    bounds = np.abs(beta[m - 1] * S[-1, :])
    scale = max(float(np.abs(theta).max()), 1e-300)
    order = np.argsort(theta)
    kept = []
    for i in order:
        if kept and abs(theta[i] - theta[kept[-1]]) <= 1e-8 * scale:
            if bounds[i] < bounds[kept[-1]]:
                kept[-1] = i
            continue
        kept.append(i)
    copies = {}
    for i in order:
        head = min(kept, key=lambda h: abs(theta[h] - theta[i]))
        copies[head] = copies.get(head, 0) + 1
    if m > 1:
        hat = eigvalsh_tridiagonal(alpha[1:], off[1:]) if m > 2 else np.asarray(alpha[1:])
        kept = [h for h in kept
                if copies[h] > 1 or np.min(np.abs(hat - theta[h])) > 1e-11 * scale]
    kept = sorted(kept, key=lambda h: -abs(theta[h]))[:top]
    return theta[kept], bounds[kept], S[:, kept]


def weak_id_diagnostics(des, sigma2, leverage, n_draws=64, block=32, seed=0, max_iter=150,
                        tol=1e-4, top=3, smooth_bins=None, scratch_mb=32):
    """leaveout_weakid.py:565-713 `weak_id_diagnostics`: per component the
    leading eigenvalues of S^- Q by Lanczos in the S^- inner product (three
    components in lockstep, one solve of three columns a step; :217-383),
    sum lambda^2 by deflated Hutchinson (:467-555, seed + 3_300_007), the
    ratios, q, and the first-stage F of the leading direction (:715-744).
    No covariates in the design."""
    layout = des.se_layout()
    lw, gw, total, norm, psi = layout
    L, G, c = des.cells.L, len(des.starts) - 1, des.X.shape[1]
    n_psi = psi.stop - psi.start
    if n_draws < 2:
        raise ValueError("n_draws must be at least 2")

    def q_block(comps, U_l, U_g):
        out_l, out_g = np.zeros_like(U_l), np.zeros_like(U_g)
        comps = np.asarray(comps)
        for k in range(3):
            cols = np.flatnonzero(comps == k)
            if len(cols):
                ql, qg = des.apply_q(k, U_l[:, cols], U_g[:, cols], layout)
                out_l[:, cols], out_g[:, cols] = ql, qg
        return out_l, out_g

    def solve(t):
        U_l, U_c, U_g, _ = des.apply_inverse(t[0], t[1], t[2])
        return [U_l, U_c, U_g]

    def dot(a, b):
        return sum((x * y).sum(axis=0) for x, y in zip(a, b))

    # :185-215 `_krylov_plan`
    dims = [max(n_psi - 1, 0), max(L + c + 1, 1), max(2 * (n_psi - 1), 0)]
    support_rows = [n_psi, G, n_psi + G]
    budget = int(scratch_mb) << 20
    caps = [min(max_iter, d) for d in dims]
    reorth = [cap * 2 * r * 8 <= budget for cap, r in zip(caps, support_rows)]

    def support(k, t):
        parts = []
        if k in (0, 2):
            parts.append(t[0][psi, k])
        if k in (1, 2):
            parts.append(t[2][:, k])
        return np.concatenate(parts) if len(parts) > 1 else parts[0].copy()

    def scatter(k, flat, t):
        at = 0
        if k in (0, 2):
            t[0][psi, k] -= flat[:n_psi]
            at = n_psi
        if k in (1, 2):
            t[2][:, k] -= flat[at:]

    def project(t):
        for k in (0, 2):
            t[0][psi, k] -= t[0][psi, k].mean()
        for k in (1, 2):
            t[2][:, k] -= t[2][:, k].mean()

    shapes = [(L, 3), (c, 3), (G, 3)]

    def lanczos(n_iter, ritz=None, check=None, every=20):
        r = [rademacher(pos, s[0], 3, seed, 0) for pos, s in zip((0, L, L + c), shapes)]
        ql, qg = q_block([0, 1, 2], r[0], r[2])
        x = [ql, np.zeros(shapes[1]), qg]
        project(x)
        y = solve(x)
        nrm = np.sqrt(np.maximum(dot(x, y), 0.0))
        live = (nrm > 0) & (np.array(caps) > 0)
        for t in (*x, *y):
            t[:, live] /= nrm[live]
            t[:, ~live] = 0.0
        x_prev = [np.zeros(s) for s in shapes]
        beta_prev = np.zeros(3)
        basis = [([], []) for _ in range(3)]
        alphas, betas = [[], [], []], [[], [], []]
        lengths = np.zeros(3, dtype=int)
        acc = None
        if ritz is not None:
            kk = ritz[0].shape[1]
            acc = ([np.zeros((s[0], 3 * kk)) for s in shapes],
                   [np.zeros((s[0], 3 * kk)) for s in shapes])
        beta_max = np.zeros(3)
        steps = 0
        for j in range(n_iter):
            if not live.any():
                break
            if (check is not None and j > 0 and j % every == 0
                    and check([np.array(a) for a in alphas], [np.array(b) for b in betas],
                              lengths, j)):
                break
            steps = j + 1
            if acc is not None:
                for k in np.flatnonzero(live):
                    if j < len(ritz[k]):
                        cols = slice(k * kk, (k + 1) * kk)
                        for ax, ay, xb, yb in zip(acc[0], acc[1], x, y):
                            ax[:, cols] += np.outer(xb[:, k], ritz[k][j])
                            ay[:, cols] += np.outer(yb[:, k], ritz[k][j])
            for k in np.flatnonzero(live):
                if reorth[k]:
                    basis[k][0].append(support(k, x))
                    basis[k][1].append(support(k, y))
            ql, qg = q_block([0, 1, 2], y[0], y[2])
            w = [ql, np.zeros(shapes[1]), qg]
            for wb, xp in zip(w, x_prev):
                wb -= beta_prev * xp
            alpha = dot(w, y)
            for wb, xb in zip(w, x):
                wb -= alpha * xb
            fix = dot(w, y)
            for wb, xb in zip(w, x):
                wb -= fix * xb
            alpha = alpha + fix
            project(w)
            for k in np.flatnonzero(live):
                if not reorth[k] or not basis[k][0]:
                    continue
                for _ in range(2):
                    wk = support(k, w)
                    Xs, Ys = np.column_stack(basis[k][0]), np.column_stack(basis[k][1])
                    scatter(k, Xs @ (Ys.T @ wk), w)
            project(w)
            z = solve(w)
            beta = np.sqrt(np.maximum(dot(w, z), 0.0))
            beta_max = np.maximum(beta_max, beta)
            for k in np.flatnonzero(live):
                alphas[k].append(float(alpha[k]))
                betas[k].append(float(beta[k]))
                lengths[k] = j + 1
            live = (live & (beta > 1e-8 * np.maximum(beta_max, 1e-300))
                    & (lengths < np.array(caps)))
            x_prev = x
            x = [wb.copy() for wb in w]
            y = z
            for t in (*x, *y):
                t[:, live] /= beta[live]
                t[:, ~live] = 0.0
            beta_prev = np.where(live, beta, 0.0)
        if acc is not None:
            return acc
        return [np.array(a) for a in alphas], [np.array(b) for b in betas], lengths, steps

    def converged_all(alphas, betas, lengths, steps):
        for k in range(3):
            if lengths[k] < steps:
                continue
            theta, bounds, _ = ritz_top(alphas[k], betas[k], top)
            lead = float(np.abs(theta[0])) if len(theta) else 0.0
            if np.any(bounds[:2] > tol * max(lead, 1e-300)):
                return False
        return True

    alphas, betas, lengths, n_iter = lanczos(max_iter, check=converged_all, every=10)
    checked = [ritz_top(alphas[k], betas[k], top) for k in range(3)]
    n_coef = L + c + G
    kk = top if 2 * 3 * top * n_coef * 8 <= budget else 1
    ritz = []
    for _, _, S in checked:
        coef = np.zeros((S.shape[0], kk))
        coef[:, :min(kk, S.shape[1])] = S[:, :kk]
        ritz.append(coef)
    X, Y = lanczos(n_iter, ritz=ritz)
    # :436-465 `_s_orthonormalize`: modified Gram-Schmidt in <x, y> = x' S^- y
    for k in range(3):
        base = k * kk
        for a in range(kk):
            ca = base + a
            for p in range(a):
                cp = base + p
                co = sum(xb[:, ca] @ yb[:, cp] for xb, yb in zip(X, Y))
                for xb, yb in zip(X, Y):
                    xb[:, ca] -= co * xb[:, cp]
                    yb[:, ca] -= co * yb[:, cp]
            n2 = sum(xb[:, ca] @ yb[:, ca] for xb, yb in zip(X, Y))
            lead = sum(xb[:, base] @ yb[:, base] for xb, yb in zip(X, Y))
            if n2 <= 1e-20 * max(lead, 1e-300) or n2 <= 0:
                for t in (*X, *Y):
                    t[:, ca] = 0.0
                continue
            for t in (*X, *Y):
                t[:, ca] *= 1.0 / np.sqrt(n2)
    u = [t[:, ::kk].copy() for t in Y]
    leading = [theta for theta, _, _ in checked]

    # :467-555 `_sum_sq_eigenvalues`
    comps = [k for k in range(3) for _ in range(kk)]
    ql, qg = q_block(comps, Y[0], Y[2])
    zq = solve([ql, np.zeros((c, 3 * kk)), qg])
    exact = ((ql * zq[0]).sum(0) + (qg * zq[2]).sum(0)).reshape(3, kk).sum(axis=1)
    N = des.rows.n_rows
    _, inv = des._roots()
    draws, drawn = [], 0
    size = max(1, block // 3)

    def summarize(values):
        n = values.shape[1]
        se = values.std(axis=1, ddof=1) / np.sqrt(n) if n > 1 else np.full(3, np.nan)
        return exact + values.mean(axis=1), se

    def settled(est, se):
        for k in range(3):
            if not est[k] > 0 or not np.isfinite(se[k]):
                return False
            r = leading[k] ** 2 / est[k]
            if np.any(np.abs(r - WEAK_ID_THRESHOLD) < 2.0 * (se[k] / est[k]) * r):
                return False
        return True

    while drawn < n_draws:
        m = min(size, n_draws - drawn)
        xi = rademacher(0, N, m, seed + 3_300_007, drawn) * inv[:, None]
        zeta = list(des._to_coef(xi))
        yv = solve(zeta)
        y_def = [np.empty((t.shape[0], 3 * m)) for t in yv]
        for k in range(3):
            cols = slice(k * kk, (k + 1) * kk)
            proj = sum(zb.T @ Yb[:, cols] for zb, Yb in zip(zeta, Y))
            for yd, yb, Yb in zip(y_def, yv, Y):
                yd[:, k * m:(k + 1) * m] = yb - Yb[:, cols] @ proj.T
        ql, qg = q_block([k for k in range(3) for _ in range(m)], y_def[0], y_def[2])
        bq = solve([ql, np.zeros((c, 3 * m)), qg])
        draws.append(((ql * bq[0]).sum(axis=0) + (qg * bq[2]).sum(axis=0)).reshape(3, m))
        drawn += m
        if drawn >= 16 and drawn < n_draws and settled(*summarize(np.hstack(draws))):
            break
    sum_sq, sum_sq_se = summarize(np.hstack(draws))

    # :715-744 `_first_stage_f`, sigma2 smoothed on the leverage alone
    table = fit_smoother(sigma2, leverage, None, smooth_bins)
    smooth = smooth_eval(table, leverage, None) if table is not None else np.asarray(sigma2)
    rows_u = readout(des.starts, des.codes, des.cells.offs, des.X, u[0], u[1], u[2])
    root = np.sqrt(des.w)
    x1 = rows_u * root[:, None]
    y = des.rows.V[:, 0]
    y_t = root * (y - float(des.w @ y / des.w.sum()))
    num, den = x1.T @ y_t, (x1 ** 2).T @ smooth
    f_stat = np.where(den > 0, num ** 2 / np.where(den > 0, den, 1.0), np.nan)

    out = {"eigenvalues": [], "bounds": [], "ratios": [], "q": [], "q_capped": [],
           "q_borderline": [], "converged": [], "sum_sq": sum_sq, "sum_sq_se": sum_sq_se,
           "f_stat": f_stat, "steps": n_iter, "lengths": lengths, "n_draws": drawn,
           "deflated": kk, "caps": caps, "reorth": reorth, "lead_vectors": u}
    for k in range(3):
        theta, bnd, _ = checked[k]
        lead = float(np.abs(theta[0])) if len(theta) else 0.0
        r = theta ** 2 / sum_sq[k] if sum_sq[k] > 0 else np.zeros_like(theta)
        q = 0
        for v in r:
            if v < WEAK_ID_THRESHOLD:
                break
            q += 1
        rel_se = sum_sq_se[k] / sum_sq[k] if sum_sq[k] > 0 else np.inf
        out["eigenvalues"].append(theta)
        out["bounds"].append(bnd)
        out["ratios"].append(r)
        out["q"].append(q)
        out["q_capped"].append(bool(q == len(r) and q > 0))
        out["q_borderline"].append(bool(np.any(np.abs(r - WEAK_ID_THRESHOLD) < 2.0 * rel_se * r)))
        out["converged"].append(bool(lengths[k] < n_iter or lengths[k] >= caps[k]
                                     or np.all(bnd[:2] <= tol * max(lead, 1e-300))))
    return out


# ------------------------------------------------ the wild cluster bootstrap

def wild_bootstrap(AG, sG, beta, j, adj, reps, weights_type, impose_null, seed):
    """core/wildboot.py:65-102 (`_draws`, `_Test`) and core/results.py:
    296-307, 863-867: (t, t*, p-value) of the restricted (or unrestricted)
    wild cluster bootstrap of beta_j = 0 from the clusters' sums."""
    from itertools import product
    G = AG.shape[0]
    A = np.linalg.inv(AG.sum(axis=0))
    Aj = A[:, j]
    S = sG + np.einsum("gab,b->ga", AG, Aj * (beta[j] / A[j, j])) if impose_null else sG
    a, C = S @ Aj, np.einsum("gab,b->ga", AG, Aj) @ A
    t = beta[j] / np.sqrt(adj * np.sum((sG @ Aj) ** 2))
    if weights_type == "rademacher" and 2 ** G < reps:
        blocks = [np.array(list(product([-1, 1], repeat=G)), dtype=float).T]
    else:
        rng = np.random.default_rng(seed)
        r5 = np.sqrt(5)
        gen = {"rademacher": lambda n: rng.choice([-1, 1], size=n, replace=True),
               "mammen": lambda n: rng.choice(np.array([-1, 1]) * (r5 + np.array([-1, 1])) / 2,
                                              size=n, replace=True,
                                              p=(r5 + np.array([1, -1])) / (2 * r5)),
               "webb": lambda n: rng.choice(np.concatenate([-np.sqrt(np.array([3, 2, 1]) / 2),
                                                            np.sqrt(np.array([1, 2, 3]) / 2)]),
                                            replace=True, size=n),
               "norm": lambda n: rng.normal(size=n)}[weights_type]
        per = reps if G * reps <= (1 << 25) else max(1, (1 << 25) // G)
        blocks, left = [], reps
        while left:
            b = min(per, left)
            blocks.append(np.asarray(gen(G * b), dtype=float).reshape(G, b))
            left -= b
    tstar = []
    for V in blocks:
        Vt = V.T
        U = Vt * a - (Vt @ S) @ C.T
        tstar.append((Vt @ a) / np.sqrt(adj * np.einsum("bg,bg->b", U, U)))
    tstar = np.concatenate(tstar)
    return t, tstar, float(np.mean(np.abs(tstar) >= np.abs(t) * (1 - 1e-9)))

"""Many independent fixed-effects regressions fitted together.

The systems' rows are laid end to end with disjoint codes (each system's
groups and levels shifted past the previous systems'), so ONE pass 1 and ONE
S build serve them all and the reduced matrix comes out block-diagonal.  Its
levels are renumbered so each system's are contiguous, and one persistent
launch (`hdfe_batch_pcg_solve`, csrc/batch.cu) runs the Jacobi block PCG of
every system with its own scalars -- the same algorithm, iteration rule and
tolerance as a single fit (core/solve.py:66-140) -- over warps that the host
assigns to the systems in proportion to their cost.  The launch shape (lanes
per row of the SpMV, the length at which long rows are cut into chunks, a
row's fixed cost in the warp split) is tuned on the batch itself
(`BatchSolver.tune`).  The normalisation
is the reference's per system (core/solve.py:383-399: the first non-streamed
dimension per connected component, the others per system).
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from . import _lib
from .fit import RHS_ZERO_TOL, DeviceRows, build_s, components, jacobi, pass1
from .simulate import Rows

LANE_CHOICES = (4, 8, 16, 32)
ROW_COST = 32           # a row's fixed cost in the warp split, in nonzeros
LONG_ROW = 1024         # rows with more nonzeros are cut into chunks of this size
LONG_ROW_CHOICES = (512, 1024, 4096)
ROW_COST_CHOICES = (16, 32, 64)


def _torch():
    import torch
    return torch


@dataclass
class Batch:
    """Systems laid end to end: `rows` and per system its rows, groups and,
    per dimension, level ranges (start, count) in the combined numbering."""

    rows: Rows
    row_ranges: list
    group_ranges: list
    level_ranges: list          # [system][dim] = (start within the dim, count)
    raw_ss: np.ndarray          # (systems, m) sums of squared deviations of V


def concat(systems) -> Batch:
    """Lay systems (pass 0's `Rows`, the same dimensions and variables) end
    to end with disjoint codes."""
    D = systems[0].codes.shape[1]
    m = systems[0].V.shape[1]
    weighted = systems[0].w is not None
    for r in systems:
        if r.codes.shape[1] != D or r.V.shape[1] != m or (r.w is not None) != weighted:
            raise ValueError("systems must share dimensions, variables and weighting")
    gcodes, codes, V, w = [], [], [], []
    row_ranges, group_ranges, level_ranges, raw_ss = [], [], [], []
    g0, r0 = 0, 0
    l0 = [0] * D
    for r in systems:
        gcodes.append(r.gcode.astype(np.int64) + g0)
        c = r.codes.astype(np.int64).copy()
        lv = []
        for d in range(D):
            c[:, d] += l0[d]
            lv.append((l0[d], int(r.n_levels[d])))
            l0[d] += int(r.n_levels[d])
        codes.append(c)
        V.append(r.V)
        raw_ss.append(((r.V - r.V.mean(axis=0)) ** 2).sum(axis=0) if r.n_rows
                      else np.zeros(m))
        if weighted:
            w.append(r.w)
        row_ranges.append((r0, r.n_rows))
        group_ranges.append((g0, r.n_groups))
        level_ranges.append(lv)
        g0 += r.n_groups
        r0 += r.n_rows
    rows = Rows(gcode=np.concatenate(gcodes).astype(np.uint32),
                codes=np.ascontiguousarray(np.concatenate(codes).astype(np.uint32)),
                V=np.ascontiguousarray(np.concatenate(V)),
                w=np.concatenate(w) if weighted else None, n_levels=list(l0), n_groups=g0,
                names=list(systems[0].names))
    return Batch(rows, row_ranges, group_ranges, level_ranges, np.asarray(raw_ss))


def split_work(indptr, sys_of_new, n_systems, W, long_row=LONG_ROW, fixed_cost=ROW_COST):
    """The warps' work for the batched PCG, from the renumbered CSR's indptr
    (host array): rows longer than `long_row` nonzeros are cut into chunks
    of `long_row`; each system gets one warp and then warps in proportion to
    its cost (largest remainders); the system's rows, then its chunks, are
    split over its warps by cumulative cost (nonzeros + `fixed_cost` per row
    or chunk, a long row counting `fixed_cost` for its vector work).  Returns
    a dict of the arrays `hdfe_batch_pcg_solve` takes."""
    long_row, fixed_cost = int(long_row), int(fixed_cost)
    if long_row < 1 or fixed_cost < 0:
        raise ValueError("split_work: long_row >= 1 and fixed_cost >= 0")
    indptr = np.asarray(indptr, np.int64)
    L = len(indptr) - 1
    rowlen = np.diff(indptr)
    long_ = rowlen > long_row
    nch = np.where(long_, (rowlen + long_row - 1) // long_row, 0)
    C = int(nch.sum())
    first = np.concatenate(([0], np.cumsum(nch)[:-1])).astype(np.int64)
    chunk_row = np.repeat(np.arange(L, dtype=np.int64), nch)
    j = np.arange(C, dtype=np.int64) - np.repeat(first, nch)
    chunk_lo = indptr[chunk_row] + j * long_row
    chunk_hi = np.minimum(chunk_lo + long_row, indptr[chunk_row + 1])
    row_chunk = np.where(long_, first, -1).astype(np.int32)
    row_cost = np.where(long_, 0, rowlen) + fixed_cost
    chunk_cost = (chunk_hi - chunk_lo) + fixed_cost
    if n_systems > W:
        raise ValueError(f"{n_systems} systems need more than the grid's {W} warps")
    rb = np.searchsorted(sys_of_new, np.arange(n_systems + 1))          # rows per system
    cb = np.searchsorted(chunk_row, rb)                                  # chunks per system
    sys_cost = (np.bincount(sys_of_new, weights=row_cost, minlength=n_systems)
                + np.bincount(sys_of_new[chunk_row], weights=chunk_cost, minlength=n_systems))
    share = sys_cost / max(sys_cost.sum(), 1) * (W - n_systems)
    nw = 1 + np.floor(share).astype(np.int64)
    order = np.argsort(-(share - np.floor(share)), kind="stable")
    for i in order[:W - int(nw.sum())]:
        nw[i] += 1
    warp_rows = np.empty(W + 1, np.int64)
    warp_chunks = np.empty(W + 1, np.int32)
    warp_sys = np.empty(W, np.int32)
    system_warps = np.zeros(n_systems + 1, np.int32)
    w = 0
    for i in range(n_systems):
        a, b, ca, cbb = int(rb[i]), int(rb[i + 1]), int(cb[i]), int(cb[i + 1])
        cost = np.concatenate((row_cost[a:b], chunk_cost[ca:cbb]))
        c = np.concatenate(([0], np.cumsum(cost)))
        targets = c[-1] * np.arange(nw[i]) / nw[i]
        t = np.searchsorted(c, targets, side="left")
        t = np.minimum(np.maximum.accumulate(t), len(cost))
        nrows = b - a
        system_warps[i] = w
        for k in range(nw[i]):
            warp_rows[w] = a + min(int(t[k]), nrows)
            warp_chunks[w] = ca + max(int(t[k]) - nrows, 0)
            warp_sys[w] = i
            w += 1
    system_warps[n_systems] = w
    while w < W:                  # any warps left over own no work
        warp_rows[w] = L
        warp_chunks[w] = C
        warp_sys[w] = n_systems - 1
        w += 1
    warp_rows[W] = L
    warp_chunks[W] = C
    return dict(warp_rows=warp_rows, warp_sys=warp_sys, system_warps=system_warps,
                warp_chunks=warp_chunks, chunk_row=chunk_row.astype(np.int32),
                chunk_lo=chunk_lo, chunk_hi=chunk_hi, row_chunk=row_chunk, n_chunks=C)


class BatchSolver:
    """The block-diagonal system of a `Batch` after pass 1 and the S build,
    renumbered system by system, with its warp split for the batched PCG."""

    def __init__(self, batch: Batch, tol=1e-10, maxiter=5000, lanes=None, drows=None):
        """drows: the batch's rows already on the device (`DeviceRows`), or
        None to upload them here."""
        torch = _torch()
        self.batch = batch
        self.tol, self.maxiter = float(tol), int(maxiter)
        rows = batch.rows
        self.drows = DeviceRows.from_rows(rows) if drows is None else drows
        self.cells = pass1(self.drows)
        self.S = build_s(self.cells)
        dev = self.S.indptr.device
        offs = np.concatenate(([0], np.cumsum(rows.n_levels)[:-1])).astype(np.int64)
        n = len(batch.level_ranges)
        perm = [np.arange(int(offs[d]) + s0, int(offs[d]) + s0 + cnt, dtype=np.int64)
                for lv in batch.level_ranges for d, (s0, cnt) in enumerate(lv)]
        self.perm = np.concatenate(perm) if perm else np.zeros(0, np.int64)
        self.sys_of = np.repeat(np.arange(n, dtype=np.int64),
                                [sum(cnt for _, cnt in lv) for lv in batch.level_ranges])
        L = len(self.perm)
        inv = np.empty(L, np.int64)
        inv[self.perm] = np.arange(L)
        self.perm_t = torch.as_tensor(self.perm, device=dev)
        self.inv_t = torch.as_tensor(inv, device=dev)
        # CSR of the renumbered matrix: row r of it is row perm[r] of S,
        # columns mapped through inv (entries keep their order)
        S = self.S
        rowlen = (S.indptr[1:] - S.indptr[:-1])[self.perm_t]
        indptr = torch.zeros(L + 1, dtype=torch.int64, device=dev)
        indptr[1:] = torch.cumsum(rowlen, 0)
        nnz = int(indptr[-1].item())
        src = torch.repeat_interleave(S.indptr[:-1][self.perm_t], rowlen) + (
            torch.arange(nnz, device=dev) - torch.repeat_interleave(indptr[:-1], rowlen))
        self.indptr = indptr
        self.indices = self.inv_t[S.indices[src].to(torch.int64)].to(torch.int32).contiguous()
        self.data = S.data[src].contiguous()
        self.dinv = jacobi(self.cells.diag)[self.perm_t].contiguous()
        self.m = int(self.cells.rhs.shape[1])
        self.B = self.cells.rhs[self.perm_t].contiguous()
        # per system zero right-hand sides (core/solve.py:44): ||b|| <= 1e-11 sqrt(raw ss)
        zero = np.zeros((n, self.m), np.uint8)
        bn = torch.zeros((n, self.m), dtype=torch.float64, device=dev).index_add_(
            0, torch.as_tensor(self.sys_of, device=dev), self.B * self.B).cpu().numpy()
        for i in range(n):
            zero[i] = np.sqrt(bn[i]) <= RHS_ZERO_TOL * np.sqrt(np.maximum(batch.raw_ss[i], 0.0))
        self.zero = torch.as_tensor(zero.reshape(-1), device=dev)
        self.n = n
        self.lanes = lanes
        self.shape = {}             # tuned long_row / row_cost (empty: the defaults)
        self.tuning = {}            # (lanes, long_row, row_cost) -> ms of the timed solves
        self._plans = {}
        self.root, _ = components(self.cells, 0)

    def plan(self, lanes, long_row=None, row_cost=None):
        """Grid and work split for a launch shape: lanes per row, the chunk
        length of long rows and a row's fixed cost in the split."""
        torch = _torch()
        long_row = int(long_row or self.shape.get("long_row", LONG_ROW))
        row_cost = int(self.shape.get("row_cost", ROW_COST) if row_cost is None else row_cost)
        key = (lanes, long_row, row_cost)
        if key not in self._plans:
            lib = _lib.lib()
            blocks = _lib._c.c_int32()
            wpb = _lib._c.c_int32()
            _lib.check(lib.hdfe_batch_pcg_grid(self.m, lanes, _lib._c.byref(blocks),
                                               _lib._c.byref(wpb)))
            W = blocks.value * wpb.value
            if not hasattr(self, "_indptr_host"):
                self._indptr_host = self.indptr.cpu().numpy()
            work = split_work(self._indptr_host, self.sys_of, self.n, W, long_row, row_cost)
            dev = self.indptr.device
            ws_bytes = int(lib.hdfe_batch_pcg_workspace_bytes(len(self.perm), self.m, W,
                                                              work["n_chunks"]))
            plan = {k: torch.as_tensor(v, device=dev) for k, v in work.items()
                    if k != "n_chunks"}
            plan.update(blocks=blocks.value, n_chunks=work["n_chunks"],
                        ws=torch.empty(ws_bytes, dtype=torch.uint8, device=dev))
            self._plans[key] = plan
        return self._plans[key]

    def solve(self, lanes=None, long_row=None, row_cost=None):
        """X (L, m) in the renumbered order and per-system info; the launch
        shape defaults to the tuned one."""
        torch = _torch()
        lanes = lanes or self.lanes or 8
        p = self.plan(lanes, long_row, row_cost)
        dev = self.indptr.device
        L = len(self.perm)
        X = torch.empty((L, self.m), dtype=torch.float64, device=dev)
        its = torch.empty(self.n, dtype=torch.int64, device=dev)
        rel = torch.empty(self.n, dtype=torch.float64, device=dev)
        conv = torch.empty(self.n, dtype=torch.int32, device=dev)
        status = torch.zeros(1, dtype=torch.int32, device=dev)
        _lib.check(_lib.lib().hdfe_batch_pcg_solve(
            self.indptr.data_ptr(), self.indices.data_ptr(), self.data.data_ptr(), L,
            self.dinv.data_ptr(), self.B.data_ptr(), self.m, self.zero.data_ptr(), self.n,
            p["warp_rows"].data_ptr(), p["warp_sys"].data_ptr(), p["system_warps"].data_ptr(),
            p["warp_chunks"].data_ptr(), p["chunk_row"].data_ptr(), p["chunk_lo"].data_ptr(),
            p["chunk_hi"].data_ptr(), p["row_chunk"].data_ptr(), p["n_chunks"], p["blocks"],
            lanes, self.tol, self.maxiter, X.data_ptr(), its.data_ptr(),
            rel.data_ptr(), conv.data_ptr(), status.data_ptr(), p["ws"].data_ptr(),
            p["ws"].numel(), _lib.stream_handle()))
        st = int(status.item())
        if st != _lib.HDFE_OK:
            raise _lib.HDFEError(st, "batched PCG stopped early")
        return X, {"iterations": its.cpu().numpy(), "max_rel_residual": rel.cpu().numpy(),
                   "converged": conv.cpu().numpy().astype(bool), "lanes": lanes,
                   "long_row": int(long_row or self.shape.get("long_row", LONG_ROW)),
                   "row_cost": int(self.shape.get("row_cost", ROW_COST) if row_cost is None
                                   else row_cost)}

    def _time(self, lanes, long_row, row_cost):
        """ms of one solve with this shape (CUDA events, after an untimed one)."""
        torch = _torch()
        key = (lanes, long_row, row_cost)
        if key not in self.tuning:
            self.solve(lanes, long_row, row_cost)
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record()
            self.solve(lanes, long_row, row_cost)
            b.record()
            torch.cuda.synchronize()
            self.tuning[key] = a.elapsed_time(b)
        return self.tuning[key]

    def tune(self):
        """The launch shape for this batch, one coordinate at a time: lanes
        per row (LANE_CHOICES) at the default split, then the long-row chunk
        length (LONG_ROW_CHOICES), then the row cost (ROW_COST_CHOICES), each
        choice timed once after an untimed solve and the fastest kept.
        Returns the lanes; the split is kept in `shape`."""
        long_row, row_cost = LONG_ROW, ROW_COST
        lanes = min(LANE_CHOICES, key=lambda v: self._time(v, long_row, row_cost))
        long_row = min(LONG_ROW_CHOICES, key=lambda v: self._time(lanes, v, row_cost))
        row_cost = min(ROW_COST_CHOICES, key=lambda v: self._time(lanes, long_row, v))
        self.lanes = lanes
        self.shape = {"long_row": long_row, "row_cost": row_cost}
        return lanes

    def normalize(self, X):
        """Gamma (L, m) in the combined numbering, normalised per system
        (core/solve.py:383-399)."""
        torch = _torch()
        rows = self.batch.rows
        dev = X.device
        G = torch.empty_like(X)
        G[self.perm_t] = X
        offs = np.concatenate(([0], np.cumsum(rows.n_levels)[:-1])).astype(np.int64)
        obs = self.cells.obs
        nl0 = int(rows.n_levels[0])
        w0 = obs[:nl0]
        root = self.root.to(torch.int64)
        cw = torch.zeros(nl0, dtype=torch.float64, device=dev).index_add_(0, root, w0)
        cw = torch.where(cw == 0, torch.ones_like(cw), cw)
        cs = torch.zeros((nl0, self.m), dtype=torch.float64, device=dev).index_add_(
            0, root, w0[:, None] * G[:nl0])
        G[:nl0] -= (cs / cw[:, None])[root]
        for d in range(1, rows.codes.shape[1]):
            o, nl = int(offs[d]), int(rows.n_levels[d])
            sys_d = torch.as_tensor(np.repeat(np.arange(self.n), [lv[d][1] for lv in
                                                                   self.batch.level_ranges]),
                                    device=dev)
            wd = obs[o:o + nl]
            sw = torch.zeros(self.n, dtype=torch.float64, device=dev).index_add_(0, sys_d, wd)
            ss = torch.zeros((self.n, self.m), dtype=torch.float64, device=dev).index_add_(
                0, sys_d, wd[:, None] * G[o:o + nl])
            G[o:o + nl] -= (ss / torch.clamp(sw, min=1.0)[:, None])[sys_d]
        return G

    def gammas(self, G):
        """Per system its effects (L_i, m), dimension by dimension."""
        torch = _torch()
        rows = self.batch.rows
        offs = np.concatenate(([0], np.cumsum(rows.n_levels)[:-1])).astype(np.int64)
        out = []
        for lv in self.batch.level_ranges:
            out.append(torch.cat([G[int(offs[d]) + s0:int(offs[d]) + s0 + cnt]
                                  for d, (s0, cnt) in enumerate(lv)], 0))
        return out


def fit_batch(systems, tol=1e-10, maxiter=5000, lanes=None, tune=False):
    """Fit every system of `systems` (pass 0's `Rows`): one pass 1, one S
    build, one batched PCG launch.  Returns (per-system gamma (L_i, m) on
    the device, info)."""
    solver = BatchSolver(concat(systems), tol, maxiter, lanes)
    if tune:
        solver.tune()
    X, info = solver.solve()
    return solver.gammas(solver.normalize(X)), info

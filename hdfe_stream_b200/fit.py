"""The fixed-effects solve path on the device, from pass 0's rows to Gamma.

This is the host side of libhdfe_b200 for a whole fit's step 1-2:

    rows (pass 0 layout, in HBM)
      -> pass1()        cells, identifying cells, obs/cnt, diag, rhs
                        (core/passes.py:397-589 `_pass1_cells`)
      -> build_s()      S = D_o' M_0 D_o in CSR (core/solve.py:148-194)
      -> BlockSolver    Jacobi block PCG (core/solve.py:66-140)
      -> normalize      (core/solve.py:383-399)

Every array lives in device memory as a torch tensor; the only host reads are
the data-dependent sizes between kernels (a few int64 each).
"""

from __future__ import annotations

import ctypes
from dataclasses import dataclass, field

import numpy as np

from . import _lib
from .gpu import BlockSolver, DeviceCSR, SmallSplit, small_levels

RHS_ZERO_TOL = 1e-11        # core/solve.py:44


def _torch():
    import torch
    return torch


@dataclass
class DeviceRows:
    """Pass 0's rows on the device.

    gcode (N,) uint32 (as int32), codes (N, D) uint32 (as int32), V (m, N)
    float64 one contiguous row per variable, w (N,) float64 or None."""

    gcode: object
    codes: object
    V: object
    w: object
    n_levels: list
    names: list = field(default_factory=list)

    @property
    def n_rows(self) -> int:
        return int(self.gcode.shape[0])

    @property
    def D(self) -> int:
        return int(self.codes.shape[1])

    @property
    def m(self) -> int:
        return int(self.V.shape[0])

    @classmethod
    def from_rows(cls, rows, device=None, pinned=False):
        """Upload a `simulate.Rows` (host arrays)."""
        torch = _torch()
        dev = device or torch.device("cuda", torch.cuda.current_device())

        def up(a, dtype):
            t = torch.from_numpy(np.ascontiguousarray(a).view(dtype))
            if pinned:
                t = t.pin_memory()
            return t.to(dev, non_blocking=pinned)
        gcode = up(rows.gcode.astype(np.uint32), np.int32)
        codes = up(rows.codes.astype(np.uint32), np.int32)
        V = up(np.ascontiguousarray(rows.V.T, dtype=np.float64), np.float64)
        w = None if rows.w is None else up(rows.w.astype(np.float64), np.float64)
        return cls(gcode, codes, V, w, list(rows.n_levels), list(rows.names))


@dataclass
class DeviceCells:
    """Pass 1's output on the device (sizes trimmed to the actual counts)."""

    starts: object          # (G'+1,) int64
    codes: object           # (M, D) int32 (uint32 values)
    n: object               # (M,) f64
    sums: object            # (M, m) f64 or None
    group_n: object         # (G',) f64
    lcount: object          # (L,) int32 identifying groups per level
    work: object            # (L,) int64 their cells
    obs: object
    cnt: object
    diag: object
    rhs: object             # (L, m)
    means: object
    raw_ss: object
    n_levels: list
    counts: dict

    @property
    def L(self) -> int:
        return int(sum(self.n_levels))

    @property
    def offs(self):
        return np.concatenate(([0], np.cumsum(self.n_levels)[:-1])).astype(np.int64)


def pass1(rows: DeviceRows, keep_sums: bool = False, stream=None) -> DeviceCells:
    torch = _torch()
    lib = _lib.lib()
    dev = rows.gcode.device
    N, D, m = rows.n_rows, rows.D, rows.m
    L = int(sum(rows.n_levels))
    f64 = dict(dtype=torch.float64, device=dev)
    nlev = np.asarray(rows.n_levels, dtype=np.int64)
    ws_bytes = lib.hdfe_pass1_workspace_bytes(N, m, int(keep_sums))
    ws = torch.empty(int(ws_bytes), dtype=torch.uint8, device=dev)
    # one slot at least: a structure-only pass (m = 0) still passes valid pointers
    means_buf, ss_buf = torch.empty(max(m, 1), **f64), torch.empty(max(m, 1), **f64)
    means, raw_ss = means_buf[:m], ss_buf[:m]
    starts = torch.empty(N + 1, dtype=torch.int64, device=dev)
    ccodes = torch.empty((N, D), dtype=torch.int32, device=dev)
    cn = torch.empty(N, **f64)
    csums = torch.empty((N, m), **f64) if keep_sums else None
    gn = torch.empty(N, **f64)
    obs, cnt, diag = torch.empty(L, **f64), torch.empty(L, **f64), torch.empty(L, **f64)
    rhs = torch.empty((L, m), **f64)
    lcount = torch.empty(L, dtype=torch.int32, device=dev)
    work = torch.empty(L, dtype=torch.int64, device=dev)
    counts = torch.zeros(6, dtype=torch.int64, device=dev)
    _lib.check(lib.hdfe_pass1(
        rows.gcode.data_ptr(), rows.codes.data_ptr(), D, rows.V.data_ptr(), m,
        None if rows.w is None else rows.w.data_ptr(), N, nlev.ctypes.data, means_buf.data_ptr(),
        ss_buf.data_ptr(), starts.data_ptr(), ccodes.data_ptr(), cn.data_ptr(),
        None if csums is None else csums.data_ptr(), gn.data_ptr(), obs.data_ptr(),
        cnt.data_ptr(), diag.data_ptr(), rhs.data_ptr(), lcount.data_ptr(), work.data_ptr(),
        counts.data_ptr(), ws.data_ptr(), ws.numel(), _lib.stream_handle(stream)))
    c = _lib.read_struct(_lib.Pass1Counts, counts)
    if c.status != _lib.HDFE_OK:
        raise _lib.HDFEError(c.status, "pass 1: a level code is out of range")
    G, M = int(c.n_ident_groups), int(c.n_ident_cells)
    return DeviceCells(starts=starts[:G + 1], codes=ccodes[:M], n=cn[:M],
                       sums=None if csums is None else csums[:M], group_n=gn[:G],
                       lcount=lcount, work=work, obs=obs,
                       cnt=cnt, diag=diag, rhs=rhs, means=means, raw_ss=raw_ss,
                       n_levels=list(rows.n_levels),
                       counts={k: int(getattr(c, k)) for k in
                               ("n_rows", "n_groups", "n_cells", "n_ident_groups",
                                "n_ident_cells")})


def build_s(cells: DeviceCells, stream=None) -> DeviceCSR:
    """S in CSR from the identifying cells: three launches (analyze, count,
    fill) with two size reads between them."""
    torch = _torch()
    lib = _lib.lib()
    dev = cells.starts.device
    G = int(cells.starts.shape[0]) - 1
    M = int(cells.codes.shape[0])
    D = len(cells.n_levels)
    L = cells.L
    nlev = np.asarray(cells.n_levels, dtype=np.int64)
    sh = _lib.stream_handle(stream)
    ws = torch.empty(int(lib.hdfe_sbuild_workspace_bytes(L, M, D)), dtype=torch.uint8, device=dev)
    info = torch.zeros(8, dtype=torch.int64, device=dev)
    lc = None if cells.lcount is None else cells.lcount.data_ptr()
    wk = None if cells.work is None else cells.work.data_ptr()
    args = (cells.starts.data_ptr(), G, cells.codes.data_ptr(), D, cells.n.data_ptr(),
            cells.group_n.data_ptr(), M, nlev.ctypes.data, lc, wk)
    _lib.check(lib.hdfe_sbuild_analyze(*args, ws.data_ptr(), ws.numel(), info.data_ptr(), sh))
    inf = _lib.read_struct(_lib.SbuildInfo, info)
    if inf.status != _lib.HDFE_OK:
        raise _lib.HDFEError(inf.status, "S build: a level code is out of range")
    W, T = int(inf.n_wide), int(inf.temp_len)
    wide = torch.empty(max(int(lib.hdfe_sbuild_wide_workspace_bytes(L, M, D, W)), 256),
                       dtype=torch.uint8, device=dev)
    temp = torch.empty(max(T * 12, 16), dtype=torch.uint8, device=dev)
    indptr = torch.empty(L + 1, dtype=torch.int64, device=dev)
    _lib.check(lib.hdfe_sbuild_count(*args, W, T, indptr.data_ptr(), ws.data_ptr(), ws.numel(),
                                     wide.data_ptr(), wide.numel(), temp.data_ptr(),
                                     temp.numel(), info.data_ptr(), sh))
    nnz = int(_lib.read_struct(_lib.SbuildInfo, info).nnz)
    indices = torch.empty(max(nnz, 1), dtype=torch.int32, device=dev)
    data = torch.empty(max(nnz, 1), dtype=torch.float64, device=dev)
    _lib.check(lib.hdfe_sbuild_fill(*args, W, T, indptr.data_ptr(), indices.data_ptr(),
                                    data.data_ptr(), ws.data_ptr(), ws.numel(), wide.data_ptr(),
                                    wide.numel(), temp.data_ptr(), temp.numel(),
                                    info.data_ptr(), sh))
    S = DeviceCSR(indptr, indices[:nnz], data[:nnz], L, nnz)
    S.info = {k: int(getattr(inf, k)) for k in ("n_wide", "n_warp_rows", "n_block_rows",
                                                "temp_len")}
    return S


def build_s_split(cells: DeviceCells, first: int, count: int, stream=None):
    """S in the split form (`gpu.SmallSplit`: the big levels' block in CSR,
    the dense cross and small blocks) built directly from the identifying
    cells, with the values `build_s` followed by `hdfe_small_split` would
    give; None when a big level is too wide for the build's narrow rows
    (then build S whole and split it)."""
    torch = _torch()
    lib = _lib.lib()
    dev = cells.starts.device
    G = int(cells.starts.shape[0]) - 1
    M = int(cells.codes.shape[0])
    D = len(cells.n_levels)
    L = cells.L
    nlev = np.asarray(cells.n_levels, dtype=np.int64)
    sh = _lib.stream_handle(stream)
    ws = torch.empty(int(lib.hdfe_sbuild_workspace_bytes(L, M, D)), dtype=torch.uint8, device=dev)
    info = torch.zeros(8, dtype=torch.int64, device=dev)
    lc = None if cells.lcount is None else cells.lcount.data_ptr()
    wk = None if cells.work is None else cells.work.data_ptr()
    args = (cells.starts.data_ptr(), G, cells.codes.data_ptr(), D, cells.n.data_ptr(),
            cells.group_n.data_ptr(), M, nlev.ctypes.data, lc, wk)
    _lib.check(lib.hdfe_sbuild_analyze_split(*args, first, count, ws.data_ptr(), ws.numel(),
                                             info.data_ptr(), sh))
    inf = _lib.read_struct(_lib.SbuildInfo, info)
    if inf.status == _lib.HDFE_ERR_CAPACITY:
        return None
    if inf.status != _lib.HDFE_OK:
        raise _lib.HDFEError(inf.status, "S build: a level code is out of range")
    W, T = int(inf.n_wide), int(inf.temp_len)
    wide = torch.empty(max(int(lib.hdfe_sbuild_wide_workspace_bytes(L, M, D, W)), 256),
                       dtype=torch.uint8, device=dev)
    temp = torch.empty(max(T * 12, 16), dtype=torch.uint8, device=dev)
    indptr = torch.empty(L + 1, dtype=torch.int64, device=dev)
    cross = torch.empty((first, _lib.SMALL_MAX_LEVELS), dtype=torch.float64, device=dev)
    small = torch.empty((count, count), dtype=torch.float64, device=dev)
    _lib.check(lib.hdfe_sbuild_count_split(*args, W, T, first, count, indptr.data_ptr(),
                                           cross.data_ptr(), small.data_ptr(), ws.data_ptr(),
                                           ws.numel(), wide.data_ptr(), wide.numel(),
                                           temp.data_ptr(), temp.numel(), info.data_ptr(), sh))
    nnz = int(_lib.read_struct(_lib.SbuildInfo, info).nnz)
    indices = torch.empty(max(nnz, 1), dtype=torch.int32, device=dev)
    data = torch.empty(max(nnz, 1), dtype=torch.float64, device=dev)
    _lib.check(lib.hdfe_sbuild_fill_split(*args, W, T, indptr.data_ptr(), indices.data_ptr(),
                                          data.data_ptr(), ws.data_ptr(), ws.numel(),
                                          wide.data_ptr(), wide.numel(), temp.data_ptr(),
                                          temp.numel(), info.data_ptr(), sh))
    return SmallSplit.from_parts(DeviceCSR(indptr, indices[:nnz], data[:nnz], L, nnz), cross,
                                 small, first, count)


def build_fit_s(cells: DeviceCells, m: int, small_block=True):
    """What the fit's solve takes: (S, split).  With a small trailing
    dimension and at most PCG_SMALL_MAX_K variables, only the split form
    (S None: `FitResult.S` builds the whole CSR when asked); else S whole."""
    small = small_levels(cells.n_levels) if small_block else None
    if small is not None and m <= _lib.PCG_SMALL_MAX_K:
        split = build_s_split(cells, *small)
        if split is not None:
            return None, split
    return build_s(cells), None


def jacobi(diag):
    """core/solve.py:142-146 `_jacobi` on the device."""
    torch = _torch()
    pos = diag > 1e-12
    return torch.where(pos, 1.0 / torch.where(pos, diag, torch.ones_like(diag)),
                       torch.zeros_like(diag))


def components(cells: DeviceCells, col: int = 0, stream=None):
    """Component root of each level of dimension `col` (its smallest level),
    and the number of components (core/kernels_base.py:156-174)."""
    torch = _torch()
    lib = _lib.lib()
    dev = cells.starts.device
    nl = int(cells.n_levels[col])
    root = torch.empty(nl, dtype=torch.int32, device=dev)
    out = torch.zeros(2, dtype=torch.int64, device=dev)
    ws = torch.empty(int(lib.hdfe_components_workspace_bytes()), dtype=torch.uint8, device=dev)
    G = int(cells.starts.shape[0]) - 1
    _lib.check(lib.hdfe_components(cells.starts.data_ptr(), G, cells.codes.data_ptr(),
                                   len(cells.n_levels), col, nl, root.data_ptr(), out.data_ptr(),
                                   ws.data_ptr(), ws.numel(), _lib.stream_handle(stream)))
    return root, out


_SIDE_STREAMS = {}


def components_async(cells: DeviceCells, col: int = 0):
    """`components` on a side stream, so that it runs beside the S build (it
    reads only pass 1's groups and codes).  Returns (root, out, event); wait
    on the event before reading root or out."""
    torch = _torch()
    dev = cells.starts.device
    main = torch.cuda.current_stream(dev)
    if dev.index not in _SIDE_STREAMS:
        _SIDE_STREAMS[dev.index] = torch.cuda.Stream(device=dev)
    side = _SIDE_STREAMS[dev.index]
    side.wait_stream(main)                  # pass 1's output is written
    for t in (cells.starts, cells.codes):
        t.record_stream(side)
    with torch.cuda.stream(side):
        root, out = components(cells, col, stream=side)
        done = torch.cuda.Event()
        done.record(side)
    for t in (root, out):
        t.record_stream(main)
    return root, out, done


def rank_components(root, cnt_first):
    """Labels 0, 1, ... by rows, ties to the smallest root (a stable sort):
    core/passes.py:933-950 `_rank_components`, on host arrays."""
    root = np.asarray(root, dtype=np.int64)
    nl = len(root)
    is_root = root == np.arange(nl)
    dense = (np.cumsum(is_root) - 1)[root]
    rows = np.bincount(dense, weights=cnt_first, minlength=int(is_root.sum()))
    order = np.argsort(-rows, kind="stable")
    rank = np.empty(len(order), np.int64)
    rank[order] = np.arange(len(order))
    return rank[dense], len(order)


def normalize(gamma, cells: DeviceCells, root, stream=None):
    """core/solve.py:383-399 `_normalize` on the device, Gamma (L, m) in place."""
    torch = _torch()
    lib = _lib.lib()
    m = int(gamma.shape[1])
    nlev = np.asarray(cells.n_levels, dtype=np.int64)
    ws = torch.empty(int(lib.hdfe_normalize_workspace_bytes(int(nlev[0]), m)), dtype=torch.uint8,
                     device=gamma.device)
    _lib.check(lib.hdfe_normalize(gamma.data_ptr(), m, len(nlev), nlev.ctypes.data,
                                  cells.obs.data_ptr(), root.data_ptr(), ws.data_ptr(),
                                  ws.numel(), _lib.stream_handle(stream)))
    return gamma


class FitResult:
    """Step 2's output for the estimator's own variables: gamma (L, m) on
    the device, normalised; info; the cells; S (the whole CSR: built on
    first use when the solve ran on the split form only); the first
    dimension's component roots; split (`gpu.SmallSplit`) or None."""

    def __init__(self, gamma, info, cells: DeviceCells, S, root, split=None):
        self.gamma, self.info, self.cells, self.root, self.split = gamma, info, cells, root, split
        self._S = S

    @property
    def S(self) -> DeviceCSR:
        if self._S is None:
            self._S = build_s(self.cells)
        return self._S


def solve(cells: DeviceCells, S: DeviceCSR, tol=1e-10, maxiter=5000, rhs_block=8,
          x0=None, normalize_fe=True, timer=None, precision="fp64", comps=None,
          solver="explicit", names=None, small_block=True, split=None) -> FitResult:
    """`_SolveMixin._solve` (core/solve.py:294-368) on the device: zero
    right-hand sides (norm <= 1e-11 sqrt(total sum of squares)) solved by
    zero, block PCG per `rhs_block` columns, then `_normalize`.  `comps`:
    the first dimension's components from `components_async`, else computed
    here.  `names`: the variables' names, for info["fe_spanned"].
    `small_block`: when the trailing dimensions have at most 16 levels in
    all (the years), the FP64 solve takes S with those levels' rows and
    columns stored densely (`gpu.SmallSplit`, `hdfe_pcg_solve_small`);
    `split`: that form already built (`build_fit_s`), S then may be None.  The info
    dict has the keys of core/solve.py:370-381 `_solve_info` (iterations,
    converged, blocks; max_rel_residual unless NaN; fe_spanned, the names
    of the variables the fixed effects span, only when there are any) and
    the device's own (solver, device, S_nnz, S_mb, n_components)."""
    torch = _torch()
    timer = timer or _NoTimer()
    m = int(cells.rhs.shape[1])
    dinv = jacobi(cells.diag)
    if solver == "stream_cg":
        from .gpu import StreamSolver
        solver = StreamSolver(cells, dinv, tol, maxiter)
    elif solver == "explicit":
        small = small_levels(cells.n_levels) if small_block and precision == "fp64" else None
        if split is not None or S is None:
            small = None
        if S is None and (split is None or precision != "fp64"):
            S = build_s(cells)
        solver = BlockSolver(S, dinv, tol, maxiter, precision=precision, small=small,
                             split=split if precision == "fp64" else None)
        solver.timer = timer
    else:
        raise ValueError("solver must be 'explicit' or 'stream_cg'")
    scale = torch.sqrt(torch.clamp(cells.raw_ss, min=0.0))
    zero_all = (torch.linalg.vector_norm(cells.rhs, dim=0) <= RHS_ZERO_TOL * scale).cpu().numpy()
    if comps is None:
        root, ncomp = components(cells, 0)
    else:
        root, ncomp, done = comps
        torch.cuda.current_stream(root.device).wait_event(done)
    gamma = torch.empty_like(cells.rhs)
    its, conv, rel = [], True, 0.0
    for j0 in range(0, m, rhs_block):
        j1 = min(m, j0 + rhs_block)
        X, it, c, r = solver.solve_device(cells.rhs[:, j0:j1], zero_all[j0:j1],
                                          None if x0 is None else x0[:, j0:j1])
        gamma[:, j0:j1] = X
        its.append(it)
        conv &= c
        rel = max(rel, r)
    if normalize_fe:
        normalize(gamma, cells, root)
    n_comp = ncomp.cpu().numpy()
    if int(n_comp[1]) != _lib.HDFE_OK:
        raise _lib.HDFEError(int(n_comp[1]), "components: union-find failed")
    explicit = not hasattr(solver, "matvec")
    sp = getattr(solver, "split", None)
    if explicit and S is not None:
        nnz, mb = S.nnz, round(S.nbytes / 1e6, 1)
    elif explicit:          # the split form only (its big block in info["small_block"])
        nnz, mb = None, round(sp.nbytes / 1e6, 1)
    else:
        nnz = mb = None
    info = {"solver": "explicit" if explicit else "stream_cg", "device": "cuda",
            "iterations": its if len(its) > 1 else its[0],
            "converged": conv, "blocks": len(its),
            "S_nnz": nnz, "S_mb": mb,
            "n_components": int(n_comp[0])}
    if not np.isnan(rel):
        info["max_rel_residual"] = rel
    if explicit and sp is not None:
        info["small_block"] = {"first": sp.first, "count": sp.count, "big_nnz": sp.S_big.nnz}
    names = list(names) if names else [f"v{j}" for j in range(m)]
    spanned = [names[j] for j in range(m) if zero_all[j]]
    if spanned:
        info["fe_spanned"] = spanned
    return FitResult(gamma=gamma, info=info, cells=cells, S=S, root=root, split=sp)


class PhaseTimer:
    """CUDA events around the phases of a fit, on the current stream:
    `with timer("pass1"): ...`; `totals()` gives milliseconds per phase."""

    def __init__(self):
        self.events = []

    def __call__(self, name):
        timer = self

        class _Phase:
            def __enter__(self_):
                torch = _torch()
                self_.a = torch.cuda.Event(enable_timing=True)
                self_.b = torch.cuda.Event(enable_timing=True)
                self_.a.record()

            def __exit__(self_, *exc):
                self_.b.record()
                timer.events.append((name, self_.a, self_.b))
        return _Phase()

    def totals(self):
        _torch().cuda.synchronize()
        out = {}
        for name, a, b in self.events:
            t = out.setdefault(name, [0.0, 0])
            t[0] += a.elapsed_time(b)
            t[1] += 1
        return out


class _NoTimer:
    def __call__(self, name):
        import contextlib
        return contextlib.nullcontext()


def fit(rows: DeviceRows, tol=1e-10, maxiter=5000, rhs_block=8, timer=None,
        precision="fp64", small_block=True) -> FitResult:
    """Pass 1, the S build and step 2 on the device, for device rows.
    precision "mixed": the PCG's inner iterations in FP32 with FP64
    refinement to the same FP64 tolerance.  small_block: with a trailing
    dimension of at most 16 levels (the years) and at most 4 variables, S
    is built in the split form the solve takes (`build_fit_s`)."""
    timer = timer or _NoTimer()
    with timer("pass1"):
        cells = pass1(rows)
    comps = components_async(cells)         # beside the S build
    with timer("sbuild"):
        S, split = build_fit_s(cells, rows.m, small_block and precision == "fp64")
    with timer("solve"):
        return solve(cells, S, tol, maxiter, rhs_block, timer=timer, precision=precision,
                     comps=comps, names=rows.names, split=split, small_block=small_block)


_COPY_STREAMS = {}


def _copy_stream(dev):
    torch = _torch()
    key = dev.index
    if key not in _COPY_STREAMS:
        _COPY_STREAMS[key] = torch.cuda.Stream(device=dev)
    return _COPY_STREAMS[key]


V_CHUNKS = (4, 3, 2, 1)     # relative sizes of the outcome's upload chunks, last smallest


def _group_cuts(gcode, weights):
    """Row offsets 0 < c_1 < ... < N cutting the sorted host `gcode` into
    pieces of about the given relative sizes, each cut at a group's first
    row (so no group is split)."""
    g = gcode.numpy() if hasattr(gcode, "numpy") else np.asarray(gcode)
    N = len(g)
    tot = float(sum(weights))
    cuts, acc = [0], 0.0
    for wgt in weights[:-1]:
        acc += wgt
        t = min(int(N * acc / tot), N - 1)
        c = int(np.searchsorted(g, g[t], side="left")) if N else 0
        if cuts[-1] < c < N:
            cuts.append(c)
    cuts.append(N)
    return cuts


@dataclass
class HostUpload:
    """Rows in flight to the device (`upload_host`): device tensors being
    filled on the copy stream and the events that say when."""

    gcode: object
    codes: object
    w: object
    chunks: list                # (first row, last row + 1, V chunk (m, rows), event)
    structure: object           # event: gcode, codes and w have landed
    m: int
    done: object = None         # event on the compute stream: the fit has read them all


def upload_host(gcode, codes, V, w=None, v_chunks=V_CHUNKS, reuse=None) -> HostUpload:
    """Start the upload of host rows in pass 0's layout -- gcode (N,) int32,
    codes (N, D) int32, V (m, N) float64, w (N,) float64 or None, pinned --
    on the copy stream, and return at once: the group and level structure
    (and the weights) first, then V in chunks of whole groups (relative sizes
    `v_chunks`, the last the smallest).  No wait on the compute stream: the
    copies write fresh blocks of the copy stream's own pool (the caching
    allocator never hands a block freed on one stream to another), so a
    caller can upload the next fit's rows while this one computes.  `reuse`:
    an earlier upload of rows of the same shape whose fit has returned; its
    device buffers are written again (after that fit's last read of them),
    so a pipeline of fits cycles two sets of buffers instead of allocating."""
    torch = _torch()
    dev = torch.device("cuda", torch.cuda.current_device())
    copy = _copy_stream(dev)
    m = int(V.shape[0])
    cuts = _group_cuts(gcode, list(v_chunks) or [1])
    same = (reuse is not None and reuse.done is not None and reuse.m == m and
            tuple(reuse.gcode.shape) == tuple(gcode.shape) and
            tuple(reuse.codes.shape) == tuple(codes.shape) and (reuse.w is None) == (w is None)
            and [(lo, hi) for lo, hi, _, _ in reuse.chunks] == list(zip(cuts[:-1], cuts[1:])))
    chunks = []
    with torch.cuda.stream(copy):
        if same:
            copy.wait_event(reuse.done)
            g_d, c_d, w_d = reuse.gcode, reuse.codes, reuse.w
            g_d.copy_(gcode, non_blocking=True)
            c_d.copy_(codes, non_blocking=True)
            if w_d is not None:
                w_d.copy_(w, non_blocking=True)
        else:
            g_d = gcode.to(dev, non_blocking=True)
            c_d = codes.to(dev, non_blocking=True)
            w_d = None if w is None else w.to(dev, non_blocking=True)
        structure = torch.cuda.Event()
        structure.record(copy)
        for q, (lo, hi) in enumerate(zip(cuts[:-1], cuts[1:])):
            Vc = reuse.chunks[q][2] if same else torch.empty((m, hi - lo), dtype=torch.float64,
                                                             device=dev)
            for j in range(m):
                Vc[j].copy_(V[j, lo:hi], non_blocking=True)
            ev = torch.cuda.Event()
            ev.record(copy)
            chunks.append((lo, hi, Vc, ev))
    return HostUpload(g_d, c_d, w_d, chunks, structure, m)


def fit_uploaded(up: HostUpload, n_levels, tol=1e-10, maxiter=5000, rhs_block=8, timer=None,
                 precision="fp64", names=None) -> FitResult:
    """The fit of rows `upload_host` is bringing over, overlapped with their
    arrival: pass 1 runs on the structure alone (m = 0: cells, counts,
    diag) as soon as it lands, then the components and S are built while V
    is still on the bus; as each V chunk lands, pass 1 runs on that chunk's
    rows for its right-hand sides (sums over its groups, so they add up
    across chunks; the variables' sums of squares combine by the
    parallel-variance rule).  After the last byte only the last chunk's
    pass and the solve remain."""
    torch = _torch()
    timer = timer or _NoTimer()
    dev = up.gcode.device
    compute = torch.cuda.current_stream(dev)
    compute.wait_event(up.structure)
    g_d, c_d, w_d, m = up.gcode, up.codes, up.w, up.m
    for t in (g_d, c_d, w_d):
        if t is not None:
            t.record_stream(compute)
    n_levels = list(n_levels)
    empty = torch.empty((0, int(g_d.shape[0])), dtype=torch.float64, device=dev)
    with timer("pass1"):
        shape = pass1(DeviceRows(g_d, c_d, empty, w_d, n_levels))
    comps = components_async(shape)         # the structure is all it reads
    with timer("sbuild"):
        S, split = build_fit_s(shape, m, precision == "fp64")
    rhs, n_tot, mean, m2 = None, 0, None, None
    with timer("pass1"):
        for lo, hi, Vc, ev in up.chunks:
            compute.wait_event(ev)
            Vc.record_stream(compute)
            part = pass1(DeviceRows(g_d[lo:hi], c_d[lo:hi], Vc,
                                    None if w_d is None else w_d[lo:hi], n_levels))
            nb = hi - lo
            if rhs is None:
                rhs, n_tot, mean, m2 = part.rhs, nb, part.means.clone(), part.raw_ss.clone()
            else:
                rhs = rhs + part.rhs
                delta = part.means - mean
                n_new = n_tot + nb
                m2 = m2 + part.raw_ss + delta * delta * (n_tot * nb / n_new)
                mean = mean + delta * (nb / n_new)
                n_tot = n_new
            del part
    up.done = torch.cuda.Event()        # every read of the upload's buffers is enqueued
    up.done.record(compute)
    import dataclasses
    cells = dataclasses.replace(shape, rhs=rhs, means=mean, raw_ss=m2)
    with timer("solve"):
        return solve(cells, S, tol, maxiter, rhs_block, timer=timer, precision=precision,
                     comps=comps, names=names, split=split)


def fit_host(gcode, codes, V, n_levels, w=None, tol=1e-10, maxiter=5000, rhs_block=8,
             timer=None, precision="fp64", names=None, v_chunks=V_CHUNKS) -> FitResult:
    """The fit from host tensors in pass 0's layout (pinned for the copies to
    overlap): `upload_host` then `fit_uploaded`.  S depends on the structure
    only and comes out identical to `fit`'s; the right-hand sides agree with
    `fit`'s to rounding (another grouping of the same sums).  A caller
    fitting one panel after another overlaps the next upload with this
    fit's work by calling `upload_host` for the next rows before
    `fit_uploaded` for these."""
    return fit_uploaded(upload_host(gcode, codes, V, w, v_chunks), n_levels, tol, maxiter,
                        rhs_block, timer, precision, names)


def fit_rows(rows, tol=1e-10, maxiter=5000, rhs_block=8):
    """The fit from host rows (pass 0's layout, `simulate.Rows`): upload,
    solve on the device, and the normalised fixed effects back on the host.
    Returns (gamma (L, m) numpy, info)."""
    res = fit(DeviceRows.from_rows(rows), tol, maxiter, rhs_block)
    return res.gamma.cpu().numpy(), res.info


BATCH_ROWS = 4_000_000      # rows per streamed batch (core/passes.py batch_rows)


def group_batches(rows, batch_rows=BATCH_ROWS):
    """Host rows (pass 0's layout, `simulate.Rows`) cut into batches of at
    most about `batch_rows` rows at group boundaries -- every group whole in
    one batch (core/passes.py:397-589 streams pass 1 the same way) -- as
    pinned tuples (gcode (n,) int32, codes (n, D) int32, V (m, n) float64, w
    (n,) float64 or None).  A group longer than `batch_rows` is a batch of
    its own."""
    import torch
    g = np.asarray(rows.gcode)
    N = len(g)
    heads = np.flatnonzero(np.concatenate(([True], g[1:] != g[:-1]))) if N else np.zeros(0, int)
    cuts, at = [0], 0
    while at < N:
        # the last group start at or below at + batch_rows, past `at`
        k = int(np.searchsorted(heads, at + int(batch_rows), side="right")) - 1
        nxt = int(heads[k]) if k >= 0 and heads[k] > at else None
        if at + int(batch_rows) >= N:
            nxt = N
        elif nxt is None:                       # one group longer than a batch
            j = int(np.searchsorted(heads, at, side="right"))
            nxt = int(heads[j]) if j < len(heads) else N
        cuts.append(nxt)
        at = nxt

    def pin(a, dtype):
        return torch.from_numpy(np.ascontiguousarray(a).view(dtype)).pin_memory()
    out = []
    for a, b in zip(cuts[:-1], cuts[1:]):
        out.append((pin(rows.gcode[a:b].astype(np.uint32), np.int32),
                    pin(rows.codes[a:b].astype(np.uint32), np.int32),
                    pin(np.ascontiguousarray(rows.V[a:b].T, dtype=np.float64), np.float64),
                    None if rows.w is None else pin(rows.w[a:b].astype(np.float64),
                                                    np.float64)))
    return out


def fit_stream(batches, n_levels, tol=1e-10, maxiter=5000, rhs_block=8, names=None,
               precision="fp64", timer=None) -> FitResult:
    """The fit from row batches streamed through the device (the reference's
    pass 1 over `batch_rows` batches, core/passes.py:397-589): the batches
    (`group_batches`' pinned tuples, every group whole in one batch) are
    uploaded on a copy stream one ahead of pass 1, so batch b + 1 crosses
    PCIe while pass 1 runs on batch b, and only one or two batches are on the
    device at a time.  Each batch's level arrays (obs, cnt, diag, rhs,
    identifying groups and their cells per level) are sums over its groups
    and add up across batches; its identifying cells append to the cell list
    (their starts shifted by the cells before them); the variables' raw sums
    of squares combine by the parallel-variance rule.  The S build and the
    solve then run on the whole cell list, as in `fit`."""
    torch = _torch()
    timer = timer or _NoTimer()
    dev = torch.device("cuda", torch.cuda.current_device())
    compute = torch.cuda.current_stream(dev)
    copy = _copy_stream(dev)
    n_levels = list(n_levels)

    def upload(b):              # no wait on compute: see fit_host
        with torch.cuda.stream(copy):
            ts = tuple(None if t is None else t.to(dev, non_blocking=True) for t in b)
            ev = torch.cuda.Event()
            ev.record(copy)
        return ts, ev

    if not batches:
        raise ValueError("fit_stream: no batches")
    level = None                            # obs, cnt, diag, rhs, lcount, work
    parts = []                              # per batch: starts, codes, n, group_n
    counts = {}
    n_tot, mean, m2 = 0, None, None
    ahead = upload(batches[0])
    with timer("pass1"):
        for i in range(len(batches)):
            (g, c, V, w), ev = ahead
            compute.wait_event(ev)
            for t in (g, c, V, w):
                if t is not None:
                    t.record_stream(compute)
            if i + 1 < len(batches):
                ahead = upload(batches[i + 1])
            cells = pass1(DeviceRows(g, c, V, w, n_levels))
            arrays = (cells.obs, cells.cnt, cells.diag, cells.rhs, cells.lcount, cells.work)
            level = list(arrays) if level is None else [a + b for a, b in zip(level, arrays)]
            parts.append((cells.starts.clone(), cells.codes.clone(), cells.n.clone(),
                          cells.group_n.clone()))
            for k, v in cells.counts.items():
                counts[k] = counts.get(k, 0) + v
            nb = int(g.shape[0])
            if mean is None:
                n_tot, mean, m2 = nb, cells.means.clone(), cells.raw_ss.clone()
            else:                           # Chan, Golub and LeVeque's pairwise update
                delta = cells.means - mean
                n_new = n_tot + nb
                m2 = m2 + cells.raw_ss + delta * delta * (n_tot * nb / n_new)
                mean = mean + delta * (nb / n_new)
                n_tot = n_new
            del cells, g, c, V, w
        starts, shift = [], 0
        for s, *_ in parts:
            starts.append(s[:-1] + shift)
            shift += int(s[-1].item())          # the batch's identifying cells
        starts.append(torch.tensor([shift], dtype=torch.int64, device=dev))
        cells = DeviceCells(starts=torch.cat(starts),
                            codes=torch.cat([p[1] for p in parts]),
                            n=torch.cat([p[2] for p in parts]),
                            sums=None, group_n=torch.cat([p[3] for p in parts]),
                            lcount=level[4].to(torch.int32), work=level[5], obs=level[0],
                            cnt=level[1], diag=level[2], rhs=level[3], means=mean,
                            raw_ss=m2, n_levels=n_levels, counts=counts)
        del parts
    comps = components_async(cells)
    with timer("sbuild"):
        S, split = build_fit_s(cells, int(cells.rhs.shape[1]), precision == "fp64")
    with timer("solve"):
        res = solve(cells, S, tol, maxiter, rhs_block, timer=timer, precision=precision,
                    comps=comps, names=names, split=split)
    res.info["batches"] = len(batches)
    return res

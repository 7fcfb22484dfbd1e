"""The drop-in for hdfe-stream's device solve seam.

hdfe-stream's step 2 reaches the GPU through one function,
`core/gpu.py:186-197 explicit_solver(S, dinv, tol, maxiter, debug) ->
(solve, device_name)`, called from core/solve.py:221-229 when
`device == "cuda"` and `solver == "explicit"`; `solve(b, zero, x0)` returns
`(X, iterations, converged, max_rel)` with host arrays in and out.  This
module provides the same two functions, and `cuda_backend()` (the seam the
reference's tests monkeypatch, core/gpu.py:33-51), backed by the persistent
CUDA block-PCG of libhdfe_b200 instead of CuPy:

* S and the preconditioner go to the device once per solver, as there;
* each call is one launch for up to 8 right-hand-side columns (wider blocks
  run as independent launches of 8: each column's CG is independent, so the
  result is the same as one lockstep solve), with no host round trip per
  iteration;
* errors follow the reference: ImportError naming what to build when the
  library is missing, RuntimeError when there is no device; non-convergence
  is reported in the return value (the caller warns), not raised.
"""

from __future__ import annotations

import ctypes
from types import SimpleNamespace

import numpy as np

from . import _lib

_HINT = ("device='cuda' needs libhdfe_b200.so built for sm_100a "
         "(`python -m hdfe_stream_b200.build`) and an NVIDIA B200 GPU")


def cuda_backend():
    """The device the solver runs on, as core/gpu.py:33-51 returns it: a
    namespace with the device `name` (and the torch device)."""
    try:
        import torch
    except ImportError as err:              # pragma: no cover - torch is a dependency
        raise ImportError(_HINT) from err
    try:
        _lib.lib()
    except ImportError as err:
        raise ImportError(f"{_HINT}: {err}") from err
    if not torch.cuda.is_available() or torch.cuda.device_count() < 1:
        raise RuntimeError("device='cuda': no CUDA device found")
    dev = torch.device("cuda", torch.cuda.current_device())
    return SimpleNamespace(name=torch.cuda.get_device_name(dev), device=dev)


class DeviceCSR:
    """S on the device: indptr int64 (L+1), indices int32 (nnz), data f64."""

    def __init__(self, indptr, indices, data, L: int, nnz: int):
        self.indptr, self.indices, self.data = indptr, indices, data
        self.L, self.nnz = int(L), int(nnz)

    @classmethod
    def from_host(cls, indptr, indices, data, device=None):
        import torch
        dev = device or torch.device("cuda", torch.cuda.current_device())
        ip = torch.as_tensor(np.ascontiguousarray(indptr, dtype=np.int64)).to(dev)
        ix = torch.as_tensor(np.ascontiguousarray(indices, dtype=np.int32)).to(dev)
        dt = torch.as_tensor(np.ascontiguousarray(data, dtype=np.float64)).to(dev)
        return cls(ip, ix, dt, len(indptr) - 1, len(data))

    @classmethod
    def from_scipy(cls, S, device=None):
        return cls.from_host(S.indptr, S.indices, S.data, device)

    @property
    def nbytes(self) -> int:
        return self.nnz * 12 + (self.L + 1) * 8


def small_levels(n_levels):
    """(first, count) of the dense small block for levels stacked by
    dimension (`n_levels`): the trailing dimensions whose levels total at
    most SMALL_MAX_LEVELS, behind at least one big level; None if none."""
    n = [int(v) for v in n_levels]
    count, d = 0, len(n)
    while d > 1 and count + n[d - 1] <= _lib.SMALL_MAX_LEVELS:
        count += n[d - 1]
        d -= 1
    first = sum(n[:d])
    return (first, count) if count > 0 and first > 0 else None


class SmallSplit:
    """S split for `hdfe_pcg_solve_small`: the big levels' block in CSR
    (`S_big`), cross (first, 16) = S[r, first + j] and small (count, count)
    (`hdfe_small_split`)."""

    @classmethod
    def from_parts(cls, S_big: DeviceCSR, cross, small, first: int, count: int):
        """The split form as built directly (`fit.build_s_split`)."""
        self = cls.__new__(cls)
        self.S_big, self.cross, self.small = S_big, cross, small
        self.first, self.count = int(first), int(count)
        return self

    def __init__(self, S: DeviceCSR, first: int, count: int, stream=None):
        import torch
        lib = _lib.lib()
        dev = S.indptr.device
        L = S.L
        self.first, self.count = int(first), int(count)
        indptr = torch.empty(L + 1, dtype=torch.int64, device=dev)
        indices = torch.empty(max(S.nnz, 1), dtype=torch.int32, device=dev)
        data = torch.empty(max(S.nnz, 1), dtype=torch.float64, device=dev)
        self.cross = torch.empty((self.first, _lib.SMALL_MAX_LEVELS), dtype=torch.float64,
                                 device=dev)
        self.small = torch.empty((self.count, self.count), dtype=torch.float64, device=dev)
        out = torch.zeros(2, dtype=torch.int64, device=dev)       # nnz, status
        ws = torch.empty(int(lib.hdfe_small_split_workspace_bytes(L)), dtype=torch.uint8,
                         device=dev)
        _lib.check(lib.hdfe_small_split(
            S.indptr.data_ptr(), S.indices.data_ptr(), S.data.data_ptr(), L, self.first,
            self.count, indptr.data_ptr(), indices.data_ptr(), data.data_ptr(),
            self.cross.data_ptr(), self.small.data_ptr(), out.data_ptr(),
            out.data_ptr() + 8, ws.data_ptr(), ws.numel(), _lib.stream_handle(stream)))
        nnz, status = (int(v) for v in out.cpu())
        if status & 0xFFFFFFFF:
            raise _lib.HDFEError(_lib.HDFE_ERR_BAD_CODE,
                                 "small split: a big row holds only small-level entries "
                                 "or a column is out of range")
        self.S_big = DeviceCSR(indptr, indices[:nnz], data[:nnz], L, nnz)

    @property
    def nbytes(self) -> int:
        return self.S_big.nbytes + (self.cross.numel() + self.small.numel()) * 8


class BlockSolver:
    """`solve(b, zero, x0) -> (X, iterations, converged, rel)` on the device.

    `solve_device` takes and returns device tensors (what the device-resident
    fit and the leave-out passes use); calling the object takes host arrays,
    exactly as the reference's `solve` (core/gpu.py:194-196)."""

    def __init__(self, S: DeviceCSR, dinv, tol: float, maxiter: int, debug=None,
                 precision: str = "fp64", inner_tol: float = 1e-6, small=None, split=None):
        """precision "fp64" is the reference's solve; "mixed" runs the inner
        CG in FP32 with FP64 iterative refinement (hdfe_pcg_solve_mixed),
        stopping on the same FP64 relative residual `tol`.  small: (first,
        count) of a dense small block (`small_levels`), used by the FP64
        solves of at most PCG_SMALL_MAX_K columns (`hdfe_pcg_solve_small`);
        split: that form already built (`SmallSplit`), in which case S may be
        None when no solve is wider than PCG_SMALL_MAX_K columns."""
        import torch
        if precision not in ("fp64", "mixed"):
            raise ValueError("precision must be 'fp64' or 'mixed'")
        self.precision, self.inner_tol = precision, float(inner_tol)
        self.S = S
        self._data32 = S.data.float() if precision == "mixed" else None
        self.dev = (S if S is not None else split.S_big).indptr.device
        self.dinv = torch.as_tensor(np.asarray(dinv, dtype=np.float64)).to(self.dev) \
            if not torch.is_tensor(dinv) else dinv.to(self.dev, torch.float64).contiguous()
        self.tol, self.maxiter, self.debug = float(tol), int(maxiter), debug
        self._ws = {}
        self._info = torch.zeros(3, dtype=torch.float64, device=self.dev)   # 24 bytes
        self._zero = torch.zeros(_lib.PCG_MAX_K, dtype=torch.uint8, device=self.dev)
        self.stats = {"launches": 0, "iterations": 0}     # solves so far (for the roofline)
        self.split = split if precision == "fp64" else None
        if self.split is None and small is not None and precision == "fp64":
            try:
                self.split = SmallSplit(S, *small)
            except _lib.HDFEError as e:
                # a level whose row of S meets only the small levels: solve
                # on the whole CSR instead
                if e.code != _lib.HDFE_ERR_BAD_CODE:
                    raise

    def _workspace(self, k):
        import torch
        if k not in self._ws:
            size = (_lib.lib().hdfe_pcg_mixed_workspace_bytes if self.precision == "mixed"
                    else _lib.lib().hdfe_pcg_workspace_bytes)
            A = self.S if self.S is not None else self.split.S_big
            nbytes = size(A.L, A.nnz, k)
            if nbytes < 0:
                raise _lib.HDFEError(_lib.HDFE_ERR_CUDA, "could not size the PCG workspace")
            self._ws[k] = torch.empty(int(nbytes), dtype=torch.uint8, device=self.dev)
        return self._ws[k]

    def launch(self, B, zero, X0, X, stream=None):
        """Enqueue one solve of at most 8 columns on `stream` (no sync)."""
        k = B.shape[1]
        ws = self._workspace(k)
        zp = None
        if zero is not None:
            import torch
            self._zero[:k].copy_(torch.from_numpy(np.asarray(zero, bool).astype(np.uint8)))
            zp = self._zero.data_ptr()
        x0p = None if X0 is None else X0.data_ptr()
        if self.split is not None and k <= _lib.PCG_SMALL_MAX_K:
            sp = self.split
            _lib.check(_lib.lib().hdfe_pcg_solve_small(
                sp.S_big.indptr.data_ptr(), sp.S_big.indices.data_ptr(),
                sp.S_big.data.data_ptr(), sp.S_big.L, sp.S_big.nnz, sp.first, sp.count,
                sp.cross.data_ptr(), sp.small.data_ptr(), self.dinv.data_ptr(), B.data_ptr(),
                k, zp, x0p, self.tol, self.maxiter, X.data_ptr(), ws.data_ptr(), ws.numel(),
                self._info.data_ptr(), _lib.stream_handle(stream)))
            return
        if self.S is None:
            raise ValueError(f"a {k}-column solve needs S's CSR; this solver holds only the "
                             "split form")
        if self.precision == "mixed":
            _lib.check(_lib.lib().hdfe_pcg_solve_mixed(
                self.S.indptr.data_ptr(), self.S.indices.data_ptr(), self.S.data.data_ptr(),
                self._data32.data_ptr(), self.S.L, self.S.nnz, self.dinv.data_ptr(),
                B.data_ptr(), k, zp, x0p, self.tol, self.inner_tol, self.maxiter,
                X.data_ptr(), ws.data_ptr(), ws.numel(), self._info.data_ptr(),
                _lib.stream_handle(stream)))
            return
        _lib.check(_lib.lib().hdfe_pcg_solve(
            self.S.indptr.data_ptr(), self.S.indices.data_ptr(), self.S.data.data_ptr(),
            self.S.L, self.S.nnz, self.dinv.data_ptr(), B.data_ptr(), k, zp, x0p, self.tol,
            self.maxiter, X.data_ptr(), ws.data_ptr(), ws.numel(), self._info.data_ptr(),
            _lib.stream_handle(stream)))

    def read_info(self):
        raw = self._info.cpu().numpy().tobytes()
        info = _lib.PcgInfo.from_buffer_copy(raw)
        if info.status != _lib.HDFE_OK:
            why = {_lib.HDFE_ERR_SPIN_LIMIT: "a grid-wide wait timed out",
                   _lib.HDFE_ERR_BAD_CODE: "a column index of S is out of range"}
            raise _lib.HDFEError(info.status, "the PCG kernel stopped early: "
                                 + why.get(info.status, "device error"))
        self.stats["launches"] += 1
        self.stats["iterations"] += max(int(info.iterations), 0)
        return int(info.iterations), bool(info.converged), float(info.max_rel)

    def solve_device(self, B, zero=None, X0=None):
        import torch
        B = B.to(self.dev, torch.float64).contiguous()
        L, k = B.shape
        X = torch.empty_like(B)
        its, conv, rel = 0, True, 0.0
        zero = None if zero is None else np.asarray(zero, bool)
        width = _lib.PCG_MIXED_MAX_K if self.precision == "mixed" else _lib.PCG_MAX_K
        for j0 in range(0, k, width):
            j1 = min(k, j0 + width)
            Bj = B[:, j0:j1].contiguous()
            Xj = torch.empty_like(Bj)
            X0j = None if X0 is None else X0[:, j0:j1].to(self.dev, torch.float64).contiguous()
            zj = None if zero is None else zero[j0:j1]
            timer = getattr(self, "timer", None)
            if timer is not None:
                with timer("pcg_kernel"):
                    self.launch(Bj, zj, X0j, Xj)
            else:
                self.launch(Bj, zj, X0j, Xj)
            it, c, r = self.read_info()
            X[:, j0:j1] = Xj
            its, conv, rel = max(its, it), conv and c, max(rel, r)
        if self.debug is not None:
            self.debug(f"  CG iter {its}: max rel. residual {rel:.2e}")
        return X, its, conv, rel

    def __call__(self, b, zero=None, x0=None):
        import torch
        b = np.ascontiguousarray(b, dtype=np.float64)
        B = torch.as_tensor(b).to(self.dev)
        X0 = None if x0 is None else torch.as_tensor(np.ascontiguousarray(x0, np.float64)).to(self.dev)
        X, it, conv, rel = self.solve_device(B, zero, X0)
        return X.cpu().numpy(), it, conv, rel


class StreamSolver:
    """The `stream_cg` solver (core/solve.py:251-266): the same Jacobi block
    PCG (core/solve.py:66-140, step for step: per-column alpha and beta, the
    active mask, `zero` columns, warm start, rel = ||R|| / ||B||) with S P
    computed from pass 1's identifying cells every iteration
    (`hdfe_stream_matvec`) instead of from an explicit S.  The reference
    falls back to it when S does not fit its memory budget; here it serves the
    same role for a caller that would rather not hold S.  The iteration is
    driven from the host (one read of the active mask per iteration), the
    product and the vector updates run on the device."""

    def __init__(self, cells, dinv, tol: float, maxiter: int, debug=None):
        import torch
        self.cells = cells
        self.dev = cells.starts.device
        self.dinv = dinv.to(self.dev, torch.float64).contiguous() if torch.is_tensor(dinv) \
            else torch.as_tensor(np.asarray(dinv, np.float64), device=self.dev)
        self.tol, self.maxiter, self.debug = float(tol), int(maxiter), debug
        self._nlev = np.asarray(cells.n_levels, dtype=np.int64)
        self._status = torch.zeros(1, dtype=torch.int32, device=self.dev)

    def matvec(self, P):
        """S P (P (L, k), k <= 32) from the cells."""
        import torch
        P = P.contiguous()
        out = torch.empty_like(P)
        c = self.cells
        _lib.check(_lib.lib().hdfe_stream_matvec(
            c.starts.data_ptr(), int(c.starts.shape[0]) - 1, c.codes.data_ptr(),
            len(self._nlev), self._nlev.ctypes.data, c.n.data_ptr(), P.data_ptr(), P.shape[1],
            out.data_ptr(), self._status.data_ptr(), _lib.stream_handle()))
        return out

    def _solve_block(self, B, zero, X0):
        import torch
        L, k = B.shape
        bnorm = torch.linalg.vector_norm(B, dim=0)
        bnorm = torch.where(bnorm == 0, torch.ones_like(bnorm), bnorm)
        if X0 is None:
            X = torch.zeros_like(B)
            R = B.clone()
        else:
            X = X0.clone()
            R = B - self.matvec(X)
        zero_t = torch.zeros(k, dtype=torch.bool, device=self.dev) if zero is None else \
            torch.as_tensor(np.asarray(zero, bool), device=self.dev)
        if bool(zero_t.any()):
            X[:, zero_t] = 0.0
            R[:, zero_t] = 0.0
            if bool(zero_t.all()):
                return X, 0, True, 0.0
        active = ~zero_t
        rel = torch.zeros(k, dtype=torch.float64, device=self.dev)
        if X0 is not None:
            rel = torch.linalg.vector_norm(R, dim=0) / bnorm
            active &= rel > self.tol
            if not bool(active.any()):
                return X, 0, True, float(rel.max())
        d = self.dinv[:, None]
        P = R * d
        rz = (R * P).sum(0)
        it = 0
        for it in range(1, self.maxiter + 1):
            AP = self.matvec(P)
            pAp = (P * AP).sum(0)
            alpha = torch.where(active & (pAp > 0), rz / torch.where(pAp > 0, pAp, 1.0),
                                torch.zeros_like(pAp))
            X += alpha * P
            R -= alpha * AP
            rel = torch.sqrt((R * R).sum(0)) / bnorm
            rz_new = (R * R * d).sum(0)
            active = rel > self.tol
            if not bool(active.any()):
                break
            beta = torch.where(active, rz_new / torch.where(rz != 0, rz, 1.0),
                               torch.zeros_like(rz))
            P = R * d + beta * P
            rz = rz_new
        if int(self._status.item()) != _lib.HDFE_OK:
            raise _lib.HDFEError(int(self._status.item()), "stream_cg: a level code is out of range")
        return X, it, not bool(active.any()), float(rel.max())

    def solve_device(self, B, zero=None, X0=None):
        import torch
        B = B.to(self.dev, torch.float64).contiguous()
        L, k = B.shape
        X = torch.empty_like(B)
        its, conv, rel = 0, True, 0.0
        zero = None if zero is None else np.asarray(zero, bool)
        for j0 in range(0, k, 32):
            j1 = min(k, j0 + 32)
            X0j = None if X0 is None else X0[:, j0:j1].to(self.dev, torch.float64)
            Xj, it, c, r = self._solve_block(B[:, j0:j1], None if zero is None else zero[j0:j1],
                                             X0j)
            X[:, j0:j1] = Xj
            its, conv, rel = max(its, it), conv and c, max(rel, r)
        if self.debug is not None:
            self.debug(f"  CG iter {its}: max rel. residual {rel:.2e}")
        return X, its, conv, rel

    def __call__(self, b, zero=None, x0=None):
        import torch
        B = torch.as_tensor(np.ascontiguousarray(b, dtype=np.float64)).to(self.dev)
        X0 = None if x0 is None else torch.as_tensor(np.ascontiguousarray(x0, np.float64)).to(self.dev)
        X, it, conv, rel = self.solve_device(B, zero, X0)
        return X.cpu().numpy(), it, conv, rel


def explicit_solver(S, dinv, tol, maxiter, debug=None):
    """(solve(b, zero, x0) -> (X, iterations, converged, rel), device name):
    S (scipy CSR) and the preconditioner are copied to the device here, once
    (core/gpu.py:186-197)."""
    be = cuda_backend()
    A = DeviceCSR.from_scipy(S, be.device)
    return BlockSolver(A, dinv, tol, maxiter, debug), be.name


def pcg(A: DeviceCSR, dinv, b, zero=None, x0=None, tol=1e-10, maxiter=5000, debug=None):
    """One block-PCG solve on a device matrix (core/gpu.py:199-253): host
    arrays in and out, `(X, iterations, converged, max_rel)`."""
    return BlockSolver(A, dinv, tol, maxiter, debug)(b, zero, x0)

"""The inverse operator and the JLA leverages on the device.

Host side of the row-pass kernels of libhdfe_b200 (rows.cu) with the block
PCG: the projection A S^- A' of regenerated Rademacher draws
(inverse.py:240-309 `project_rows`, with the covariate Schur border of
:182-218 `_border`) and the Johnson-Lindenstrauss leverages of
leaveout.py:130-198 `jla_leverages` / :210-282 `_combine_moments`.  The draws
are keyed on (seed, row ordinal, absolute draw index), so the results do not
depend on how the draws are blocked, exactly as in the reference.
"""

from __future__ import annotations

import numpy as np

from . import _lib
from .fit import DeviceCells, DeviceRows, RHS_ZERO_TOL, jacobi
from .gpu import BlockSolver, DeviceCSR

MAX_BLOCK = 32      # vectors per row pass (one lane each)


def _torch():
    import torch
    return torch


class InverseOperator:
    """A S^- A' for one fit's design: its rows (device), identifying cells
    and reduced matrix S, and optional covariates (N, c) joining the fixed
    effects in the design (leaveout.py:91-110 `_model_covariates`)."""

    def __init__(self, rows: DeviceRows, cells: DeviceCells, S: DeviceCSR, covariates=None,
                 tol=1e-10, maxiter=5000, precision="fp64"):
        torch = _torch()
        self.rows, self.cells, self.S = rows, cells, S
        self.dev = rows.gcode.device
        self.N = rows.n_rows
        self.L = cells.L
        self.nlev = np.asarray(cells.n_levels, dtype=np.int64)
        self.solver = BlockSolver(S, jacobi(cells.diag), tol, maxiter, precision=precision)
        self.X = None if covariates is None or covariates.shape[1] == 0 else \
            covariates.to(self.dev, torch.float64).contiguous()
        self.c = 0 if self.X is None else int(self.X.shape[1])
        self.w = rows.w
        self.starts, self.G = self._row_groups()
        self._border = None
        self._ws = torch.empty(256, dtype=torch.uint8, device=self.dev)

    def _row_groups(self):
        torch = _torch()
        lib = _lib.lib()
        starts = torch.empty(self.N + 1, dtype=torch.int64, device=self.dev)
        ng = torch.zeros(1, dtype=torch.int64, device=self.dev)
        ws = torch.empty(int(lib.hdfe_row_groups_workspace_bytes(self.N)), dtype=torch.uint8,
                         device=self.dev)
        _lib.check(lib.hdfe_row_groups(self.rows.gcode.data_ptr(), self.N, starts.data_ptr(),
                                       ng.data_ptr(), ws.data_ptr(), ws.numel(),
                                       _lib.stream_handle()))
        G = int(ng.item())
        return starts[:G + 1], G

    def _ptr(self, t):
        return None if t is None else t.data_ptr()

    def center(self, B, seed=0, first_draw=0, R=None, sqrt_weights=False):
        """(acc (L, B), acc_x (c, B), squares (B)): `_reduce` over all rows."""
        torch = _torch()
        f64 = dict(dtype=torch.float64, device=self.dev)
        acc = torch.empty((self.L, B), **f64)
        acc_x = torch.empty((max(self.c, 1), B), **f64)
        sq = torch.empty(B, **f64)
        _lib.check(_lib.lib().hdfe_rows_center(
            self.starts.data_ptr(), self.G, self.rows.codes.data_ptr(), len(self.nlev),
            self.nlev.ctypes.data, self._ptr(self.w), self._ptr(self.X), self.c, self._ptr(R), B,
            int(seed) & (2**64 - 1), int(first_draw), 0, int(bool(sqrt_weights)), acc.data_ptr(),
            acc_x.data_ptr(), sq.data_ptr(), self._ws.data_ptr(), self._ws.numel(),
            _lib.stream_handle()))
        return acc, acc_x[:self.c], sq

    def solve_reduced(self, rhs, scale):
        """inverse.py:86-103 `_solve_reduced`: columns negligible next to
        their scale are solved by zero, the rest by the block PCG."""
        torch = _torch()
        zero = (torch.linalg.vector_norm(rhs, dim=0) <= RHS_ZERO_TOL * scale).cpu().numpy()
        U, it, conv, rel = self.solver.solve_device(rhs, zero)
        return U, {"iterations": it, "converged": conv, "max_rel_residual": rel}

    def border(self):
        """(Z, pinv(Schur)) for the covariates, computed once."""
        torch = _torch()
        if self._border is None:
            if self.c == 0:
                self._border = (None, None)
            else:
                T_dx, T_xx, sq = self.center(self.c, R=self.X)
                Z, _ = self.solve_reduced(T_dx, torch.sqrt(sq))
                schur = (T_xx - T_dx.T @ Z).cpu().numpy()
                self._border = (Z, torch.as_tensor(np.linalg.pinv(schur, hermitian=True),
                                                   device=self.dev))
        return self._border

    def project(self, B, seed=0, first_draw=0, sqrt_weights=False, out=True, moments=None):
        """`project_rows` for B <= 32 Rademacher vectors: the rows' (A S^- A'
        r_j)_i as an (N, B) tensor (out=True), and/or the JLA sink's five
        running sums added into `moments` (5, N)."""
        torch = _torch()
        if not 1 <= B <= MAX_BLOCK:
            raise ValueError(f"project: 1 <= B <= {MAX_BLOCK}")
        Z, schur_inv = self.border()
        rhs, rhs_x, sq = self.center(B, seed, first_draw, sqrt_weights=sqrt_weights)
        U, info = self.solve_reduced(rhs, torch.sqrt(sq))
        if Z is not None:
            C = schur_inv @ (rhs_x - Z.T @ rhs)
            U = (U - Z @ C).contiguous()
        else:
            C = None
        res = torch.empty((self.N, B), dtype=torch.float64, device=self.dev) if out else None
        _lib.check(_lib.lib().hdfe_rows_project(
            self.starts.data_ptr(), self.G, self.rows.codes.data_ptr(), len(self.nlev),
            self.nlev.ctypes.data, self._ptr(self.w), self._ptr(self.X), self.c,
            self._ptr(None if C is None else C.contiguous()), U.data_ptr(), None, B,
            int(seed) & (2**64 - 1), int(first_draw), 0, int(bool(sqrt_weights)), self.N,
            self._ptr(res), self._ptr(moments), _lib.stream_handle()))
        return res, info

    def jla_leverages(self, n_draws=250, block=MAX_BLOCK, seed=0):
        """leaveout.py:130-198 `jla_leverages`: (leverage, complement, factor)
        per row (device tensors), in the square-root weight metric when the
        fit is weighted."""
        torch = _torch()
        block = int(block)
        if block < 1 or n_draws < 1:
            raise ValueError("n_draws and block must be at least 1")
        block = min(block, MAX_BLOCK)
        moments = torch.zeros((5, self.N), dtype=torch.float64, device=self.dev)
        drawn, blocks, info = 0, 0, {}
        while drawn < n_draws:
            size = min(block, n_draws - drawn)
            _, info = self.project(size, seed, drawn, sqrt_weights=self.w is not None,
                                   out=False, moments=moments)
            drawn += size
            blocks += 1
        _lib.check(_lib.lib().hdfe_jla_combine(moments.data_ptr(), self.N, n_draws,
                                               _lib.stream_handle()))
        self.jla_info = {**info, "blocks": blocks}
        return moments[0], moments[1], moments[2]

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

    # ---- coefficient-space right-hand sides (inverse.py:311-460)

    def null_space(self):
        """inverse.py:376-428 `_null_space`: an orthonormal basis of S's null
        space as (streamed (G, k), levels (L, k)) device blocks -- per
        connected component, +1 on its groups and -1 on its levels of the
        first non-streamed dimension; per further dimension, +1 across the
        first and -1 across it.  Built once (host QR of a (G + L) x k matrix
        of structured columns, as the reference does)."""
        if getattr(self, "_null", None) is None:
            torch = _torch()
            from .fit import components, rank_components
            cells = self.cells
            root, _ = components(cells, 0)
            nl0 = int(self.nlev[0])
            cnt_first = cells.cnt[:nl0].cpu().numpy()
            comp, n_comp = rank_components(root.cpu().numpy(), cnt_first)
            # inverse.py:430-437 `_group_components`: each group's first row
            first = self.rows.codes.view(-1, len(self.nlev))[self.starts[:-1], 0]
            gcomp = comp[first.cpu().numpy().astype(np.int64)]
            offs = np.concatenate(([0], np.cumsum(self.nlev)[:-1]))
            vecs = []
            for c in range(n_comp):
                lv = np.zeros(self.L)
                lv[offs[0]:offs[0] + nl0] = -(comp == c).astype(float)
                vecs.append(np.concatenate([(gcomp == c).astype(float), lv]))
            for d in range(1, len(self.nlev)):
                lv = np.zeros(self.L)
                lv[offs[0]:offs[0] + nl0] = 1.0
                lv[offs[d]:offs[d] + self.nlev[d]] = -1.0
                vecs.append(np.concatenate([np.zeros(self.G), lv]))
            q = np.linalg.qr(np.column_stack(vecs))[0] if vecs else np.zeros((self.G + self.L, 0))
            q = torch.as_tensor(q, device=self.dev)
            self._null = (q[:self.G].contiguous(), q[self.G:].contiguous())
        return self._null

    def drop_null(self, levels, streamed):
        """inverse.py:445-460 `_drop_null_component` (thin GEMMs)."""
        qs, ql = self.null_space()
        if ql.shape[1] == 0:
            return levels, streamed
        overlap = qs.T @ streamed + ql.T @ levels
        return (levels - ql @ overlap).contiguous(), (streamed - qs @ overlap).contiguous()

    def _status(self):
        torch = _torch()
        if getattr(self, "_st", None) is None:
            self._st = torch.zeros(1, dtype=torch.int32, device=self.dev)
        return self._st

    def apply_inverse(self, levels, cov_values, streamed, omega=None, rows=False):
        """inverse.py:311-374 `apply_inverse`: u = S^- v for v in coefficient
        space -- levels (L, B), cov_values (c, B), streamed (G, B), device
        tensors, B <= 32.  Returns (U (L, B), C (c, B), U_streamed (G, B),
        rows (N, B) or None).  With omega (N), also the Hutchinson trace's
        collect sink (leaveout.py:423-431), v = A' Omega A u, as a fifth item
        (v_levels, v_cov, v_groups)."""
        torch = _torch()
        lib = _lib.lib()
        B = int(levels.shape[1])
        if not 1 <= B <= MAX_BLOCK:
            raise ValueError(f"apply_inverse: 1 <= B <= {MAX_BLOCK}")
        f64 = dict(dtype=torch.float64, device=self.dev)
        Z, schur_inv = self.border()
        levels, streamed = self.drop_null(levels.to(**f64), streamed.to(**f64).contiguous())
        scale = torch.sqrt((levels * levels).sum(dim=0) + (streamed * streamed).sum(dim=0))
        acc = torch.zeros((self.L, B), **f64)
        acc_x = torch.zeros((max(self.c, 1), B), **f64)
        st, sh = self._status(), _lib.stream_handle()
        base = (self.starts.data_ptr(), self.G, self.rows.codes.data_ptr(), len(self.nlev),
                self.nlev.ctypes.data, self._ptr(self.w), self._ptr(self.X), self.c)
        _lib.check(lib.hdfe_rows_reduce(*base, streamed.data_ptr(), None, B, acc.data_ptr(),
                                        acc_x.data_ptr(), None, st.data_ptr(), sh))
        rhs = levels - acc
        U, info = self.solve_reduced(rhs.contiguous(), scale)
        if Z is not None:
            rhs_x = cov_values.to(**f64) - acc_x[:self.c]
            C = (schur_inv @ (rhs_x - Z.T @ rhs)).contiguous()
            U = (U - Z @ C).contiguous()
        else:
            C = None
        U_g = torch.empty((self.G, B), **f64)
        out_rows = torch.empty((self.N, B), **f64) if rows else None
        v = None
        if omega is not None:
            v = (torch.zeros((self.L, B), **f64), torch.zeros((max(self.c, 1), B), **f64),
                 torch.empty((self.G, B), **f64))
        _lib.check(lib.hdfe_rows_project_coef(
            *base, self._ptr(C), U.data_ptr(), streamed.data_ptr(), B, self._ptr(out_rows),
            U_g.data_ptr(), self._ptr(omega), self._ptr(None if v is None else v[0]),
            self._ptr(None if v is None else v[1]), self._ptr(None if v is None else v[2]),
            st.data_ptr(), sh))
        self.ainv_info = info
        res = (U, C, U_g, out_rows)
        if v is not None:
            res = res + ((v[0], v[1][:self.c], v[2]),)
        return res

    def hutchinson_trace(self, sigma2, n_draws=250, block=MAX_BLOCK, seed=0, psi_column=0,
                         person_years=None):
        """leaveout.py:321-391 `hutchinson_trace` and :393-448 `_trace_block`:
        the bias terms (var(psi), var(alpha), cov(psi, alpha)) from n_draws
        Rademacher vectors in coefficient space, two applications of the
        inverse per block; sigma2 (N) per-row variances.  Draws are keyed on
        (seed, position, draw), so the answer does not depend on blocking."""
        torch = _torch()
        lib = _lib.lib()
        block = int(block)
        if block < 1 or n_draws < 1:
            raise ValueError("n_draws and block must be at least 1")
        block = min(block, MAX_BLOCK)
        f64 = dict(dtype=torch.float64, device=self.dev)
        omega = torch.as_tensor(sigma2).to(**f64).contiguous()
        L, G, c = self.L, self.G, self.c
        totals = torch.zeros(8, **f64)
        ws = torch.empty(int(lib.hdfe_trace_moments_workspace_bytes(block)), dtype=torch.uint8,
                         device=self.dev)
        mom = torch.empty((block, 8), **f64)
        drawn, blocks = 0, 0
        sh = _lib.stream_handle()
        while drawn < n_draws:
            size = min(block, n_draws - drawn)
            Zall = torch.empty((L + G + c, size), **f64)
            _lib.check(lib.hdfe_rademacher(Zall.data_ptr(), L + G + c, 0, size,
                                           int(seed) & (2**64 - 1), drawn, sh))
            Zl, Zg, Zc = Zall[:L], Zall[L:L + G], Zall[L + G:]
            *_, (vl, vx, vg) = self.apply_inverse(Zl, Zc, Zg, omega=omega)
            Ul, _, Ug, _ = self.apply_inverse(vl, vx, vg)
            _lib.check(lib.hdfe_trace_moments(
                self.starts.data_ptr(), G, self.rows.codes.data_ptr(), len(self.nlev),
                self.nlev.ctypes.data, psi_column, self._ptr(self.w), Zl.data_ptr(),
                Zg.data_ptr(), Ul.data_ptr(), Ug.data_ptr(), size, mom.data_ptr(), ws.data_ptr(),
                ws.numel(), self._status().data_ptr(), sh))
            totals += mom[:size].sum(dim=0)
            drawn += size
            blocks += 1
        t = (totals / n_draws).cpu().numpy()
        weight, a1a2, b1b2, cross, a1, a2, b1, b2 = t
        var_psi = a1a2 / weight - (a1 / weight) * (a2 / weight)
        var_alpha = b1b2 / weight - (b1 / weight) * (b2 / weight)
        cov = 0.5 * (cross / weight - (a1 / weight) * (b2 / weight) - (b1 / weight) * (a2 / weight))
        # leaveout_se.py:202-214 `_moment_divisor`: n - 1 person-years
        R = float(self.N if person_years is None else person_years)
        scale = weight / (weight * (R - 1.0) / R) if R > 1 else 1.0
        self.trace_info = {"blocks": blocks, "n_obs": float(weight)}
        return np.array([scale * var_psi, scale * var_alpha, scale * cov])

    # ---- steps 3-4 and the KSS components (core/inference.py, leaveout.py:634-1016)

    def _assemble_ws(self, m):
        torch = _torch()
        return torch.empty(int(_lib.lib().hdfe_assemble_workspace_bytes(m)), dtype=torch.uint8,
                           device=self.dev)

    def residual_moments(self, gamma):
        """V' W V of the rows' variables less Gamma's projections and their
        weighted group means (`_nb_residualize_rows` + `_assemble`), (m, m)
        on the device."""
        torch = _torch()
        m = self.rows.m
        gamma = gamma.to(self.dev, torch.float64).contiguous()
        out = torch.empty((m, m), dtype=torch.float64, device=self.dev)
        ws = self._assemble_ws(m)
        _lib.check(_lib.lib().hdfe_resid_moments(
            self.starts.data_ptr(), self.G, self.rows.codes.data_ptr(), len(self.nlev),
            self.nlev.ctypes.data, self._ptr(self.w), self.rows.V.data_ptr(), m, self.N,
            gamma.data_ptr(), out.data_ptr(), ws.data_ptr(), ws.numel(),
            self._status().data_ptr(), _lib.stream_handle()))
        return out

    def row_effects(self, gamma, beta, psi_column=0):
        """`_nb_pass2` for y = V[0], X = V[1:]: (residual (N), streamed effect
        per group (G), gam_y (L), sums (7): w, w y, w a, w b, w a^2, w b^2,
        w a b with a the psi dimension's effect and b the streamed one)."""
        torch = _torch()
        m = self.rows.m
        f64 = dict(dtype=torch.float64, device=self.dev)
        gamma = gamma.to(**f64)
        beta = torch.as_tensor(np.asarray(beta, dtype=np.float64)).to(**f64).reshape(-1)
        beta = beta.contiguous()
        gam_y = (gamma[:, 0] - gamma[:, 1:] @ beta).contiguous() if m > 1 else \
            gamma[:, 0].contiguous()
        resid = torch.empty(self.N, **f64)
        alpha = torch.empty(max(self.G, 1), **f64)
        sums = torch.empty(7, **f64)
        ws = self._assemble_ws(m)
        _lib.check(_lib.lib().hdfe_row_effects(
            self.starts.data_ptr(), self.G, self.rows.codes.data_ptr(), len(self.nlev),
            self.nlev.ctypes.data, int(psi_column), self._ptr(self.w), self.rows.V.data_ptr(), m,
            self.N, beta.data_ptr() if m > 1 else None, gam_y.data_ptr(),
            resid.data_ptr(), alpha.data_ptr(), sums.data_ptr(), ws.data_ptr(), ws.numel(),
            self._status().data_ptr(), _lib.stream_handle()))
        return resid, alpha[:self.G], gam_y, sums

    def leave_out_components(self, gamma, n_draws=250, block=MAX_BLOCK, seed=0, psi_column=0,
                             timer=None):
        """leaveout.py:634-805 `leave_out_components` (point estimates;
        stayers "own", weighted centring): beta from the residual moments,
        the plug-in var(psi), var(alpha), cov(psi, alpha) (:807-833) with the
        n - 1 divisor, sigma2 from the JLA leverages and the residuals
        (:949-1016), the Hutchinson bias with seed + 1_000_003, and
        leave_out = plug_in - bias.  gamma (L, m) the fit's normalised
        effects for V's variables (y first).  timer: a `fit.PhaseTimer` for
        the phases "steps34", "leverages", "sigma2" and "trace"."""
        import contextlib
        torch = _torch()
        phase = timer or (lambda name: contextlib.nullcontext())
        with phase("steps34"):
            A = self.residual_moments(gamma).cpu().numpy()
            m = A.shape[0]
            beta = np.linalg.solve(A[1:, 1:], A[1:, 0]) if m > 1 else np.zeros(0)
            resid, _, _, sums = self.row_effects(gamma, beta, psi_column)
            s = sums.cpu().numpy()
        if int(self._status().item()) != _lib.HDFE_OK:
            raise _lib.HDFEError(int(self._status().item()), "a level code is out of range")
        T = s[0]
        R = float(self.N)
        scale = T / (T * (R - 1.0) / R) if R > 1 else 1.0
        ma, mb = s[2] / T, s[3] / T
        plug_in = np.array([scale * (s[4] / T - ma * ma), scale * (s[5] / T - mb * mb),
                            scale * (s[6] / T - ma * mb)])
        with phase("leverages"):
            lev, comp, factor = self.jla_leverages(n_draws, block, seed)
        with phase("sigma2"):
            sigma2 = torch.empty(self.N, dtype=torch.float64, device=self.dev)
            _lib.check(_lib.lib().hdfe_kss_sigma2(
                self.rows.V.data_ptr(), self._ptr(self.w), resid.data_ptr(), comp.data_ptr(),
                factor.data_ptr(), float(s[1] / T), self.N, sigma2.data_ptr(),
                _lib.stream_handle()))
        with phase("trace"):
            bias = self.hutchinson_trace(sigma2, n_draws, block, seed + 1_000_003, psi_column)
        return {"plug_in": plug_in, "bias": bias, "leave_out": plug_in - bias, "beta": beta,
                "sigma2": sigma2, "max_leverage": float(lev.max().item()), "leverage": lev,
                "complement": comp, "factor": factor}

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

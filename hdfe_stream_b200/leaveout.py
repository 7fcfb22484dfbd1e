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

from dataclasses import dataclass, field

import numpy as np

from . import _lib
from .fit import DeviceCells, DeviceRows, RHS_ZERO_TOL, jacobi
from .gpu import BlockSolver, DeviceCSR

MAX_BLOCK = 32      # vectors per row pass (one lane each)
COMPONENTS = ("var(psi)", "var(alpha)", "cov(psi, alpha)")
TRACE_SEED_OFFSET = 1_000_003       # leaveout.py:733 (the bias term's draws)
SE_SEED_OFFSET = 5_500_011          # leaveout.py:770
WEAK_ID_SEED_OFFSET = 9_900_019     # leaveout.py:751


def _torch():
    import torch
    return torch


@dataclass
class JLALeverages:
    """Per-row leverage estimates in the rows' order (leaveout.py:65-86
    `JLALeverages`), as device tensors (N,): the leverage P_ii in [0, 1],
    its complement M_ii = 1 - P_ii and the non-linearity correction factor
    for sigma^2; n_draws Rademacher draws; diagnostics: blocks, covariates,
    the last block's PCG iterations."""

    leverage: object
    complement: object
    factor: object
    n_draws: int
    diagnostics: dict = field(default_factory=dict)

    @property
    def n_rows(self) -> int:
        return int(self.leverage.shape[0])

    def summary(self) -> str:
        d = self.diagnostics
        lev, f = self.leverage, self.factor
        return (f"JLA leverages: {self.n_rows:,} rows, {self.n_draws} draws in "
                f"{d.get('blocks', '?')} block(s)\n"
                f"  leverage   min {float(lev.min()):.6f}  max {float(lev.max()):.6f}  "
                f"mean {float(lev.mean()):.6f}\n"
                f"  correction min {float(f.min()):.6f}  max {float(f.max()):.6f}  "
                f"mean {float(f.mean()):.6f}")


@dataclass
class TraceEstimate:
    """The bias terms of the three AKM variance components (leaveout.py:
    290-313 `TraceEstimate`)."""

    var_psi: float
    var_alpha: float
    cov: float
    n_draws: int
    diagnostics: dict = field(default_factory=dict)

    def as_dict(self) -> dict:
        return {"var(psi)": self.var_psi, "var(alpha)": self.var_alpha,
                "cov(psi, alpha)": self.cov}

    def as_array(self) -> np.ndarray:
        return np.array([self.var_psi, self.var_alpha, self.cov])

    def summary(self) -> str:
        d = self.diagnostics
        return (f"bias terms from {self.n_draws} Hutchinson draws in "
                f"{d.get('blocks', '?')} block(s)\n"
                f"  var(psi)        {self.var_psi:+.6f}\n"
                f"  var(alpha)      {self.var_alpha:+.6f}\n"
                f"  cov(psi, alpha) {self.cov:+.6f}")


@dataclass
class LeaveOutComponents:
    """KSS leave-out variance components with the plug-in ones beside them
    (leaveout.py:456-630 `LeaveOutComponents`).  plug_in, bias and
    leave_out are dicts keyed "var(psi)", "var(alpha)", "cov(psi, alpha)";
    n_obs the observations (person-years); n_movers the movers'
    observations (movers' matches when leaving out a match); leverages a
    `JLALeverages`; trace a `TraceEstimate`; se a
    `leaveout_se.ComponentSE` with se=True; weak_id the weak-identification
    diagnostic's dict when it ran; diagnostics settings and summary
    statistics (maximum leverage, mean sigma2, ...); fit the regression the
    components are from; match_fit the collapsed match-level regression
    when leaving out a match.  The per-row sigma2 is in diagnostics
    ["sigma2"] (a device tensor)."""

    plug_in: dict
    bias: dict
    leave_out: dict
    n_obs: int
    n_movers: int
    leverages: object
    trace: object
    se: object = None
    weak_id: object = None
    diagnostics: dict = field(default_factory=dict)
    pruning: dict | None = None
    fit: object = None
    match_fit: object = None

    def tidy(self):
        """The three components as a table (pandas DataFrame)."""
        import pandas as pd
        keys = list(self.plug_in)
        return pd.DataFrame({"component": keys,
                             "plug_in": [self.plug_in[k] for k in keys],
                             "bias": [self.bias[k] for k in keys],
                             "leave_out": [self.leave_out[k] for k in keys]})

    def summary(self) -> str:
        d = self.diagnostics
        lines = [f"leave-out variance components ({d.get('psi')} and {d.get('alpha')})",
                 f"  {self.n_obs:,} observations, {self.n_movers:,} of them movers'; "
                 f"{self.leverages.n_draws} draws",
                 f"  max leverage {d.get('max_leverage', float('nan')):.6f}   "
                 f"mean sigma2 {d.get('sigma2_mean', float('nan')):.6f}", "",
                 f"{'component':<20}{'plug-in':>12}{'bias':>12}{'leave-out':>12}"
                 + (f"{'se':>11}" if self.se is not None else ""),
                 "-" * (67 if self.se is not None else 56)]
        for key in self.plug_in:
            row = (f"{key:<20}{self.plug_in[key]:>12.6f}{self.bias[key]:>12.6f}"
                   f"{self.leave_out[key]:>12.6f}")
            if self.se is not None:
                row += f"{self.se.se[key]:>11.6f}"
            lines.append(row)
        return "\n".join(lines)


def trace_components(mean, person_years):
    """The three bias terms from the eight Hutchinson moments averaged over
    the draws (leaveout.py:380-391): var = E[a1 a2]/w - (E[a1]/w)(E[a2]/w)
    per component and the covariance's symmetrised form, times the n - 1
    divisor's correction (leaveout_se.py:202-214 `_moment_divisor`)."""
    weight, a1a2, b1b2, cross, a1, a2, b1, b2 = (float(x) for x in mean)
    var_psi = a1a2 / weight - (a1 / weight) * (a2 / weight)
    var_alpha = b1b2 / weight - (b1 / weight) * (b2 / weight)
    cov = 0.5 * (cross / weight - (a1 / weight) * (b2 / weight) - (b1 / weight) * (a2 / weight))
    R = float(person_years)
    scale = weight / (weight * (R - 1.0) / R) if R > 1 else 1.0
    return np.array([scale * var_psi, scale * var_alpha, scale * cov])


class InverseOperator:
    """A S^- A' for one fit's design: its rows (device), identifying cells
    and reduced matrix S, and optional covariates (N, c) joining the fixed
    effects in the design (leaveout.py:91-110 `_model_covariates`).
    `fe_names`: the fixed effects' names, the streamed dimension (alpha)
    first, then the non-streamed ones in the codes' column order (default
    "fe0", "fe1", ...); `psi` arguments name one of the latter."""

    def __init__(self, rows: DeviceRows, cells: DeviceCells, S: DeviceCSR, covariates=None,
                 tol=1e-10, maxiter=5000, precision="fp64", fe_names=None):
        torch = _torch()
        names = list(fe_names) if fe_names else [f"fe{d}" for d in range(len(cells.n_levels) + 1)]
        if len(names) != len(cells.n_levels) + 1:
            raise ValueError("fe_names: the streamed dimension and one name per column of codes")
        self.g_fe, self.o_fe = names[0], names[1:]
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
        self.timer = None       # a fit.PhaseTimer: CUDA events around each kernel launch

    def _phase(self, name):
        """The timer's phase `name`, or nothing when no timer is set."""
        import contextlib
        if self.timer is None:
            return contextlib.nullcontext()
        self.solver.timer = self.timer
        return self.timer(name)

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
        with self._phase("k_center"):
            _lib.check(_lib.lib().hdfe_rows_center(
                self.starts.data_ptr(), self.G, self.rows.codes.data_ptr(), len(self.nlev),
                self.nlev.ctypes.data, self._ptr(self.w), self._ptr(self.X), self.c,
                self._ptr(R), B, int(seed) & (2**64 - 1), int(first_draw), 0,
                int(bool(sqrt_weights)), acc.data_ptr(), acc_x.data_ptr(), sq.data_ptr(),
                self._ws.data_ptr(), self._ws.numel(), _lib.stream_handle()))
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
        with self._phase("k_project"):
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
        with self._phase("k_reduce"):
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
        with self._phase("k_project_coef"):
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

    def _psi_column(self, psi):
        """The codes' column of `psi` (a name of `o_fe`, a column index, or
        None for the first)."""
        if psi is None:
            return 0
        if isinstance(psi, (int, np.integer)):
            if not 0 <= int(psi) < len(self.o_fe):
                raise ValueError(f"psi column {psi} out of range")
            return int(psi)
        if psi not in self.o_fe:
            raise ValueError(f"psi must be a non-streamed dimension, one of {self.o_fe}; "
                             f"got {psi!r}")
        return self.o_fe.index(psi)

    def _check_covariates(self, covariates):
        """The design is fixed when the operator is built: covariates=None
        (the operator's own) or the same number of columns passes."""
        if covariates is None:
            return
        if len(tuple(covariates)) != self.c:
            raise ValueError(f"this operator's design has {self.c} covariate(s); build an "
                             "InverseOperator with the covariates wanted")

    def trace_totals(self, sigma2, first, last, block=None, seed=0, psi=None):
        """The eight Hutchinson moment sums (w, a1 a2, b1 b2, cross, a1, a2,
        b1, b2; leaveout.py:393-448 `_trace_block`) over the draws
        [first, last), a device tensor (8,), and the blocks run.  Draw j is
        keyed on (seed, position, j) whoever computes it, so sums over
        disjoint draw ranges add up to the sum over their union."""
        torch = _torch()
        lib = _lib.lib()
        psi_column = self._psi_column(psi)
        block = MAX_BLOCK if block is None else int(block)
        if block < 1:
            raise ValueError("block must be at least 1")
        block = min(block, MAX_BLOCK)
        f64 = dict(dtype=torch.float64, device=self.dev)
        omega = torch.as_tensor(sigma2).to(**f64).contiguous()
        L, G, c = self.L, self.G, self.c
        totals = torch.zeros(8, **f64)
        ws = torch.empty(int(lib.hdfe_trace_moments_workspace_bytes(block)), dtype=torch.uint8,
                         device=self.dev)
        mom = torch.empty((block, 8), **f64)
        drawn, blocks = int(first), 0
        sh = _lib.stream_handle()
        while drawn < last:
            size = min(block, last - drawn)
            Zall = torch.empty((L + G + c, size), **f64)
            _lib.check(lib.hdfe_rademacher(Zall.data_ptr(), L + G + c, 0, size,
                                           int(seed) & (2**64 - 1), drawn, sh))
            Zl, Zg, Zc = Zall[:L], Zall[L:L + G], Zall[L + G:]
            *_, (vl, vx, vg) = self.apply_inverse(Zl, Zc, Zg, omega=omega)
            Ul, _, Ug, _ = self.apply_inverse(vl, vx, vg)
            with self._phase("k_trace"):
                _lib.check(lib.hdfe_trace_moments(
                    self.starts.data_ptr(), G, self.rows.codes.data_ptr(), len(self.nlev),
                    self.nlev.ctypes.data, psi_column, self._ptr(self.w), Zl.data_ptr(),
                    Zg.data_ptr(), Ul.data_ptr(), Ug.data_ptr(), size, mom.data_ptr(),
                    ws.data_ptr(), ws.numel(), self._status().data_ptr(), sh))
            totals += mom[:size].sum(dim=0)
            drawn += size
            blocks += 1
        return totals, blocks

    def hutchinson_trace(self, sigma2, n_draws=250, block=None, seed=0, covariates=None,
                         psi=None, person_years=None) -> TraceEstimate:
        """leaveout.py:321-391 `hutchinson_trace` and :393-448 `_trace_block`:
        the bias terms of var(psi), var(alpha) and cov(psi, alpha) from
        n_draws Rademacher vectors in coefficient space, two applications of
        the inverse per block; sigma2 (N) per-row variances (w Var(e)).
        Draws are keyed on (seed, position, draw), so the answer does not
        depend on blocking.  person_years: the divisor's count when the rows
        are matches (leaveout_se.py:216-220)."""
        return self._hutchinson(sigma2, n_draws, block, seed, covariates, psi, person_years)

    def _hutchinson(self, sigma2, n_draws, block, seed, covariates, psi, person_years,
                    draws=None, reduce=None):
        self._check_covariates(covariates)
        psi_column = self._psi_column(psi)
        if n_draws < 1:
            raise ValueError("n_draws must be at least 1")
        first, last = (0, int(n_draws)) if draws is None else draws
        totals, blocks = self.trace_totals(sigma2, first, last, block, seed, psi_column)
        if reduce is not None:
            reduce(totals)
        bias = trace_components(totals.cpu().numpy() / n_draws,
                                self.N if person_years is None else person_years)
        self.trace_info = {"blocks": blocks, "n_obs": float(totals[0].item() / n_draws)}
        return TraceEstimate(var_psi=float(bias[0]), var_alpha=float(bias[1]),
                             cov=float(bias[2]), n_draws=int(n_draws),
                             diagnostics={"blocks": blocks,
                                          "block": MAX_BLOCK if block is None else int(block),
                                          "psi": self.o_fe[psi_column], "covariates": self.c,
                                          "draws": (first, last)})

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

    def movers(self, psi=None):
        """(movers (N) bool, psi codes (N) int64) on the device
        (leaveout.py:928-947 `_mover_mask`): a row is a mover's when its
        group is seen at more than one level of psi."""
        torch = _torch()
        col = self._psi_column(psi)
        code = self.rows.codes[:, col].to(torch.int64)
        g = self.rows.gcode.to(torch.int64)
        n_g = int(g.max().item()) + 1 if self.N else 0
        lo = torch.full((n_g,), 2 ** 62, dtype=torch.int64, device=self.dev)
        hi = torch.full((n_g,), -1, dtype=torch.int64, device=self.dev)
        lo.scatter_reduce_(0, g, code, "amin")
        hi.scatter_reduce_(0, g, code, "amax")
        return (lo != hi)[g], code

    def leave_out_sigma2(self, y, residual, leverages: JLALeverages, movers, psi_code,
                         stayers="own", centering="weighted", stayer_sigma2=None, ybar=None):
        """leaveout.py:949-1016 `_leave_one_out_sigma2` on the device:
        sigma2_i = w_i (y_i - ybar) e_i / M_ii times the JLA factor (the
        weighted centring's fused kernel `hdfe_kss_sigma2`), or
        (sqrt(w) y - its mean) sqrt(w) e / M times the factor with
        centering "reference"; stayers "own" keep theirs, "drop" get zero,
        "firm_mean" the w-weighted mean of sigma2 / w over the movers at
        their psi level (times w), "within_match" the caller's
        `stayer_sigma2` (N).  ybar: the weighted mean of y when known."""
        torch = _torch()
        f64 = dict(dtype=torch.float64, device=self.dev)
        w = self.w if self.w is not None else torch.ones(self.N, **f64)
        comp, factor = leverages.complement, leverages.factor
        if centering == "weighted":
            sigma2 = torch.empty(self.N, **f64)
            if ybar is None:
                ybar = float((w @ y).item() / w.sum().item())
            y, residual = y.contiguous(), residual.contiguous()
            _lib.check(_lib.lib().hdfe_kss_sigma2(
                y.data_ptr(), self._ptr(self.w), residual.data_ptr(), comp.data_ptr(),
                factor.data_ptr(), ybar, self.N, sigma2.data_ptr(), _lib.stream_handle()))
        elif centering == "reference":
            root = torch.sqrt(w)
            yt = root * y
            sigma2 = (yt - yt.mean()) * root * residual / comp * factor
        else:
            raise ValueError("centering must be 'weighted' or 'reference'")
        if stayers == "own":
            return sigma2
        stay = ~movers
        if stayers == "drop":
            return torch.where(stay, torch.zeros_like(sigma2), sigma2)
        if stayers == "within_match":
            return torch.where(stay, torch.as_tensor(stayer_sigma2).to(**f64), sigma2)
        n_lev = int(psi_code.max().item()) + 1 if self.N else 0
        tot = torch.zeros(n_lev, **f64).index_add_(0, psi_code[movers], (sigma2 * w)[movers])
        cnt = torch.zeros(n_lev, **f64).index_add_(0, psi_code[movers], (w * w)[movers])
        mean = torch.where(cnt > 0, tot / torch.where(cnt > 0, cnt, 1.0),
                           torch.full_like(cnt, float("nan")))
        sigma2 = torch.where(stay, mean[psi_code] * w, sigma2)
        orphaned = int((~torch.isfinite(sigma2)).sum().item())
        if orphaned:
            raise ValueError(f"{orphaned:,} observations sit at a level of the chosen dimension "
                             "with no movers, so there is nothing to impute their variance "
                             "from; prune to the leave-one-out connected set first")
        return sigma2

    def plug_in_moments(self, gamma, psi=None):
        """(plug-in dict, beta, residuals (N), sums (7)): beta from the
        residual moments (steps 3-4), the rows' residuals and the weighted
        plug-in var(psi), var(alpha), cov(psi, alpha) with the n - 1 divisor
        (leaveout.py:807-833 `_plug_in_moments`)."""
        A = self.residual_moments(gamma).cpu().numpy()
        m = A.shape[0]
        beta = np.linalg.solve(A[1:, 1:], A[1:, 0]) if m > 1 else np.zeros(0)
        resid, _, _, sums = self.row_effects(gamma, beta, self._psi_column(psi))
        s = sums.cpu().numpy()
        if int(self._status().item()) != _lib.HDFE_OK:
            raise _lib.HDFEError(int(self._status().item()), "a level code is out of range")
        T = s[0]
        R = float(self.N)
        scale = T / (T * (R - 1.0) / R) if R > 1 else 1.0
        ma, mb = s[2] / T, s[3] / T
        plug_in = {COMPONENTS[0]: float(scale * (s[4] / T - ma * ma)),
                   COMPONENTS[1]: float(scale * (s[5] / T - mb * mb)),
                   COMPONENTS[2]: float(scale * (s[6] / T - ma * mb))}
        return plug_in, beta, resid, s

    def leave_out_components(self, result, n_draws=250, block=None, seed=0, psi=None,
                             covariates=None, stayers="own", se=False, se_draws=None,
                             se_trace=True, smooth_bins=None, diagnose=None, diagnose_draws=64,
                             weak_interval=True, confidence=0.95, stayer_sigma2=None,
                             centering="weighted", timer=None, split=None) -> LeaveOutComponents:
        """leaveout.py:634-805 `leave_out_components`, on the device:
        `result` the fit (a `fit.FitResult`, or its normalised effects
        Gamma (L, m) for V's variables, outcome first).  JLA leverages for
        n_draws probes (seed), the maximum-leverage check, the weighted
        plug-in components, beta and the residuals (steps 3-4), sigma2 by
        the `stayers` and `centering` rules, the Hutchinson bias
        (seed + 1_000_003) and leave_out = plug_in - bias; with `diagnose`
        (default: `se`) the weak-identification diagnostic (diagnose_draws,
        seed + 9_900_019); with `se` the standard errors
        (`component_variances`, se_draws, seed + 5_500_011) and, for the
        components the diagnostic flags, the q = 1 intervals at
        `confidence`.  `timer`: a `fit.PhaseTimer` for the phases
        "steps34", "leverages", "sigma2" and "trace".  `split`: a
        `shard.DrawSplit` when the job's probes and draws are shared among
        ranks (each rank runs this call on its own replica of the design)."""
        import contextlib
        torch = _torch()
        if stayers not in ("own", "firm_mean", "drop", "within_match"):
            raise ValueError("stayers must be 'own', 'firm_mean', 'drop' or 'within_match'")
        if (stayers == "within_match") != (stayer_sigma2 is not None):
            raise ValueError("stayers='within_match' needs stayer_sigma2, the per-match values "
                             "from leave_out_match")
        self._check_covariates(covariates)
        col = self._psi_column(psi)
        psi_name = self.o_fe[col]
        gamma = result.gamma if hasattr(result, "gamma") else result
        phase = timer or (lambda name: contextlib.nullcontext())
        with phase("leverages"):
            if split is None:
                lev = self.jla_leverages(n_draws, block, seed)
            else:
                lev = self._jla(n_draws, block, seed, None, split.draws(n_draws), split.sum)
        movers, psi_code = self.movers(col)
        match_level = stayers == "within_match"
        checked = movers if match_level else torch.ones_like(movers)
        worst = float(lev.leverage[checked].max().item()) if bool(checked.any()) else 0.0
        if worst >= 1.0 - 1e-9:
            unit = "match" if match_level else "observation"
            raise ValueError(
                f"maximum leverage is {worst:.6f}: the panel is not leave-one-out connected "
                f"(leaving out one {unit} at a time), so the leave-out residual is undefined "
                f"for at least one {unit}; restrict the rows to the leave-one-out connected "
                "set first (connected.leave_one_out)")
        with phase("steps34"):
            plug_in, beta, resid, sums = self.plug_in_moments(gamma, col)
        with phase("sigma2"):
            sigma2 = self.leave_out_sigma2(self.rows.V[0], resid, lev, movers, psi_code,
                                           stayers, centering, stayer_sigma2,
                                           ybar=float(sums[1] / sums[0]))
        with phase("trace"):
            if split is None:
                trace = self.hutchinson_trace(sigma2, n_draws, block, seed + TRACE_SEED_OFFSET,
                                              psi=col)
            else:
                trace = self._hutchinson(sigma2, n_draws, block, seed + TRACE_SEED_OFFSET, None,
                                         col, None, split.draws(n_draws), split.sum)
        bias = trace.as_dict()
        leave_out = {k: plug_in[k] - bias[k] for k in plug_in}
        if diagnose is None:
            diagnose = bool(se)
        weak_id = None
        errors = None
        if (diagnose or se) and split is not None:
            raise ValueError("the standard errors and the diagnostic run on one rank: "
                             "call without split for se=True or diagnose=True")
        if diagnose or se:
            from .leaveout_se import StandardErrors
            ses = StandardErrors(self, col)
        if diagnose:
            from .weakid import weak_id_diagnostics
            weak_id = weak_id_diagnostics(ses, sigma2, lev.leverage, n_draws=int(diagnose_draws),
                                          block=MAX_BLOCK if block is None else int(block),
                                          seed=seed + WEAK_ID_SEED_OFFSET)
        if se:
            from .leaveout_se import ComponentSE, weak_intervals
            draws = n_draws if se_draws is None else int(se_draws)
            raw = ses.component_variances(
                sigma2, lev.leverage, lev.complement, lev.factor, None, draws,
                8 if block is None else int(block), seed + SE_SEED_OFFSET, se_trace,
                smooth_bins, weak_id=weak_id if weak_interval else None)
            if raw["weak"]:
                weak_intervals(leave_out, raw["weak"], confidence)
            errors = ComponentSE.from_dict(raw, trace=se_trace)
        w = self.w
        s2_mean = float((sigma2 / w).mean().item()) if w is not None else \
            float(sigma2.mean().item())
        return LeaveOutComponents(
            plug_in=plug_in, bias=bias, leave_out=leave_out, n_obs=self.N,
            n_movers=int(movers.sum().item()), leverages=lev, trace=trace, se=errors,
            weak_id=weak_id, fit=result if hasattr(result, "gamma") else None,
            diagnostics={"psi": psi_name, "alpha": self.g_fe, "stayers": stayers,
                         "confidence": confidence, "max_leverage": worst,
                         "leave_out": "match" if match_level else "observation",
                         "sigma2_mean": s2_mean, "covariates": self.c, "beta": beta,
                         "sigma2": sigma2, "centering": centering,
                         "n_levels": {psi_name: int(self.nlev[col]), self.g_fe: self.G}})

    def jla_moments(self, first, last, block=None, seed=0, moments=None):
        """The JLA sink's five running sums per row (leaveout.py:181-190:
        P, M, P^2, M^2, P M over the draws) for the draws [first, last),
        added into `moments` (5, N) (zeros when None); returns (moments,
        blocks, the last block's solve info)."""
        torch = _torch()
        block = MAX_BLOCK if block is None else int(block)
        if block < 1:
            raise ValueError("block must be at least 1")
        block = min(block, MAX_BLOCK)
        if moments is None:
            moments = torch.zeros((5, self.N), dtype=torch.float64, device=self.dev)
        drawn, blocks, info = int(first), 0, {}
        while drawn < last:
            size = min(block, last - drawn)
            _, info = self.project(size, seed, drawn, sqrt_weights=self.w is not None,
                                   out=False, moments=moments)
            drawn += size
            blocks += 1
        return moments, blocks, info

    def combine_moments(self, moments, n_draws):
        """leaveout.py:210-282 `_combine_moments` in place (`hdfe_jla_combine`):
        slot 0 <- the leverage, 1 <- its complement, 2 <- the factor."""
        _lib.check(_lib.lib().hdfe_jla_combine(moments.data_ptr(), self.N, n_draws,
                                               _lib.stream_handle()))
        return moments

    def jla_leverages(self, n_draws=250, block=None, seed=0, covariates=None) -> JLALeverages:
        """leaveout.py:130-198 `jla_leverages`: every row's leverage, its
        complement and the correction factor (device tensors), in the
        square-root weight metric when the fit is weighted; `block` draws
        per projection pass (at most 32; None: 32)."""
        return self._jla(n_draws, block, seed, covariates)

    def _jla(self, n_draws, block, seed, covariates, draws=None, reduce=None):
        self._check_covariates(covariates)
        if n_draws < 1:
            raise ValueError("n_draws must be at least 1")
        first, last = (0, int(n_draws)) if draws is None else draws
        moments, blocks, info = self.jla_moments(first, last, block, seed)
        if reduce is not None:
            reduce(moments)
        self.combine_moments(moments, n_draws)
        self.jla_info = {**info, "blocks": blocks}
        return JLALeverages(leverage=moments[0], complement=moments[1], factor=moments[2],
                            n_draws=int(n_draws),
                            diagnostics={"blocks": blocks,
                                         "block": MAX_BLOCK if block is None else int(block),
                                         "covariates": self.c, "draws": (first, last),
                                         "iterations": info.get("iterations")})

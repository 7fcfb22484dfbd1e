"""KSS standard errors on the device: leaveout_se.py's `bii_rows` and
`component_variances` (trace term included), leaving out an observation or
a match.

In the square-root-weight metric the leave-out estimate of each component is
theta = y~' C y~ with the zero-diagonal kernel

    C = B - (diag(b) M + M diag(b)) / 2,   b_i = B_ii / M_ii (with the JLA
                                           correction factor),

B = X S^- Q S^- X', M = I - X S^- X', Q the component's quadratic form, and

    V = 4 sum_i s~_i (C y~)_i^2 - 2 tr(C Om~ C Om~),

s~ the leave-out sigma2 smoothed on (P_ii, B_ii), the trace by Hutchinson
draws.  Every application of C is three row passes around two applications
of the inverse (`InverseOperator.apply_inverse`): A'W^(1/2)[v | b .* v]
(`hdfe_rows_reduce`), S^-, Q in coefficient space (`hdfe_cov_cross` for the
covariance), S^- again, then the readouts (`hdfe_rows_readout`) assembled into
C v and summed (`hdfe_c_sums`).  The smoother's knots come from the
reference's own quantile rule on a sample gathered to the host; the cell sums
and the evaluation run on the device (`hdfe_smooth_cells`, `hdfe_smooth_eval`).

Leaving out a match (leaveout_se.py:616-636), the rows are matches: b is zero
on the stayers' matches, the divisor counts person-years, and the
reference-centred estimator is the uncentred sqrt(w) y through
K = C + (1 u' + u 1') / (2 R), u = M b (`m_times`, one more solve), whose
two scalars per column ride into `hdfe_c_sums_ext`.
"""

from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

from . import _lib
from .leaveout import COMPONENTS, MAX_BLOCK, InverseOperator
QUANTILE_SAMPLE = 2_000_000         # rows sampled for the smoother's knots
TRACE_SEED_OFFSET = 7_700_017       # leaveout_se.py:731
WEAK_SEED_OFFSET = 8_800_021        # leaveout_se.py:757


def _torch():
    import torch
    return torch


def smoother_bins(n: int, dims: int) -> int:
    """Bins per axis (leaveout_se.py:955-964 `_auto_bins`): cells holding
    n^(2/3) rows, the reference's lowess span n^(-1/3)."""
    power = 1.0 / 6.0 if dims == 2 else 1.0 / 3.0
    return int(np.clip(round(n ** power), 2, 500))


def smoother_knots(values: np.ndarray, n_bins: int) -> np.ndarray:
    """Strictly increasing quantile knots (leaveout_se.py:967-973)."""
    q = np.quantile(np.asarray(values, dtype=np.float64), np.linspace(0.0, 1.0, n_bins + 1))
    q = np.maximum.accumulate(q)
    span = max(float(q[-1] - q[0]), 1e-300)
    return q + np.arange(len(q)) * span * 1e-12


@dataclass
class ComponentSE:
    """Standard errors of the three components and the parts they came from
    (leaveout_se.py:74-111 `ComponentSE`), each a dict keyed "var(psi)",
    "var(alpha)", "cov(psi, alpha)": se (NaN where none is reported), the
    estimator's variance, its first term 4 sum_i sigma2_i (C mu)_i^2, the
    trace term 2 tr(C Omega C Omega), the conservative se from the first
    term alone, and theta = y'Cy (the estimand recomputed); n_draws the
    trace's draws; weak, per weakly identified component, the q = 1
    interval ("interval") and its pieces."""

    se: dict
    variance: dict
    first_term: dict
    trace_term: dict
    se_conservative: dict
    theta: dict
    n_draws: int
    diagnostics: dict = field(default_factory=dict)
    weak: dict = None

    @classmethod
    def from_dict(cls, raw: dict, trace: bool = True) -> "ComponentSE":
        """From `StandardErrors.component_variances`' dict."""
        return cls(se=raw["se"], variance=raw["variance"], first_term=raw["first_term"],
                   trace_term=raw["trace_term"], se_conservative=raw["se_conservative"],
                   theta=raw["theta"], n_draws=int(raw["n_draws"]),
                   diagnostics={"trace_included": bool(trace), "blocks": raw.get("blocks")},
                   weak=raw.get("weak"))

    def summary(self) -> str:
        lines = [f"leave-out standard errors ({self.n_draws} draws)",
                 f"{'component':<20}{'estimate':>12}{'se':>11}{'se (cons.)':>12}"
                 f"{'trace share':>13}", "-" * 68]
        for key in COMPONENTS:
            share = (self.trace_term[key] / self.first_term[key]
                     if self.first_term[key] else float("nan"))
            lines.append(f"{key:<20}{self.theta[key]:>12.6f}{self.se[key]:>11.6f}"
                         f"{self.se_conservative[key]:>12.6f}{share:>12.2%}")
        return "\n".join(lines)


class StandardErrors:
    """The KSS standard errors of one design (`InverseOperator`): psi is the
    non-streamed dimension `psi_column`, alpha the streamed one;
    `person_years` the observations behind the rows when they are matches
    (leaveout_se.py:216-220 `_person_years`; None: the rows)."""

    def __init__(self, op: InverseOperator, psi_column: int = 0, person_years=None):
        torch = _torch()
        self.op = op
        self.psi_column = int(psi_column)
        self.dev = op.dev
        self.N, self.L, self.G, self.c = op.N, op.L, op.G, op.c
        offs = np.concatenate(([0], np.cumsum(op.nlev)[:-1])).astype(np.int64)
        p0 = int(offs[self.psi_column])
        self.psi = slice(p0, p0 + int(op.nlev[self.psi_column]))
        self.f64 = dict(dtype=torch.float64, device=self.dev)
        w = op.w
        self.root = None if w is None else torch.sqrt(w)
        self.inv_root = None if w is None else torch.where(
            self.root > 0, 1.0 / torch.where(self.root > 0, self.root, torch.ones_like(w)),
            torch.zeros_like(w))
        # leaveout_se.py:135-162 `_level_weight_totals`
        lw, _, gw = self._to_coef(torch.ones((self.N, 1), **self.f64))
        self.level_w, self.group_w = lw[:, 0], gw[:, 0]
        self.total = float(self.group_w.sum().item())
        R = float(self.N if person_years is None else person_years)
        # leaveout_se.py:202-214 `_moment_divisor`
        self.norm = self.total * (R - 1.0) / R if R > 1 else self.total
        self._ws = torch.empty(int(_lib.lib().hdfe_c_sums_workspace_bytes()), dtype=torch.uint8,
                               device=self.dev)

    # ---- building blocks

    def _base(self):
        op = self.op
        return (op.starts.data_ptr(), op.G, op.rows.codes.data_ptr(), len(op.nlev),
                op.nlev.ctypes.data)

    def _to_coef(self, R):
        """A' W R for rows R (N, B) as (levels (L, B), covariates (c, B),
        groups (G, B)): `_nb_reduce_rows` and `_nb_group_sums`."""
        torch = _torch()
        op = self.op
        B = int(R.shape[1])
        lv, cv, gv = [], [], []
        for j0 in range(0, B, MAX_BLOCK):
            j1 = min(B, j0 + MAX_BLOCK)
            Rc = R[:, j0:j1].contiguous()
            acc = torch.zeros((self.L, j1 - j0), **self.f64)
            acc_x = torch.zeros((max(self.c, 1), j1 - j0), **self.f64)
            gs = torch.empty((self.G, j1 - j0), **self.f64)
            _lib.check(_lib.lib().hdfe_rows_reduce(
                *self._base(), op._ptr(op.w), op._ptr(op.X), self.c, None, Rc.data_ptr(),
                j1 - j0, acc.data_ptr(), acc_x.data_ptr(), gs.data_ptr(),
                op._status().data_ptr(), _lib.stream_handle()))
            lv.append(acc)
            cv.append(acc_x[:self.c])
            gv.append(gs)
        return torch.cat(lv, 1), torch.cat(cv, 1), torch.cat(gv, 1)

    def _apply_inverse(self, levels, cov, groups):
        """`apply_inverse` on any number of columns, in blocks of 32."""
        torch = _torch()
        B = int(levels.shape[1])
        U, C, Ug = [], [], []
        for j0 in range(0, B, MAX_BLOCK):
            j1 = min(B, j0 + MAX_BLOCK)
            u, cc, ug, _ = self.op.apply_inverse(levels[:, j0:j1].contiguous(),
                                                 cov[:, j0:j1].contiguous(),
                                                 groups[:, j0:j1].contiguous())
            U.append(u)
            C.append(cc if cc is not None else torch.zeros((0, j1 - j0), **self.f64))
            Ug.append(ug)
        return torch.cat(U, 1).contiguous(), torch.cat(C, 1).contiguous(), \
            torch.cat(Ug, 1).contiguous()

    def _readout(self, U_l, U_c, U_g, root):
        """(A u)_i for each column (N, B), times sqrt(w_i) when `root`."""
        torch = _torch()
        op = self.op
        B = int(U_l.shape[1])
        out = torch.empty((self.N, B), **self.f64)
        # contiguous copies held in locals: a pointer must not outlive its tensor
        U_l, U_c, U_g = U_l.contiguous(), U_c.contiguous(), U_g.contiguous()
        _lib.check(_lib.lib().hdfe_rows_readout(
            *self._base(), op._ptr(op.X), self.c, U_l.data_ptr(),
            U_c.data_ptr() if self.c else None, U_g.data_ptr(), B,
            op._ptr(op.w) if root else None, out.data_ptr(), op._status().data_ptr(),
            _lib.stream_handle()))
        return out

    def _draws(self, size, seed, first_draw):
        return self._draws_at(self.N, 0, size, seed, first_draw)

    def _draws_at(self, n, ordinal0, size, seed, first_draw):
        """Rademacher draws (n, size) for the ordinals ordinal0 .. ordinal0 + n
        (core/kernels_groups.py:53-76 `_nb_rademacher`)."""
        torch = _torch()
        z = torch.empty((n, size), **self.f64)
        if n:
            _lib.check(_lib.lib().hdfe_rademacher(z.data_ptr(), n, int(ordinal0), size,
                                                  int(seed) & (2**64 - 1), int(first_draw),
                                                  _lib.stream_handle()))
        return z

    # ---- B_ii

    def bii_rows(self, n_draws=250, block=16, seed=0):
        """leaveout_se.py:228-327 `bii_rows`: (3, N) per-row B_ii of
        var(psi), var(alpha), cov(psi, alpha); one pair of solves per draw."""
        torch = _torch()
        block = int(min(max(int(block), 1), MAX_BLOCK // 2))
        if n_draws < 1:
            raise ValueError("n_draws must be at least 1")
        psi, L, G = self.psi, self.L, self.G
        root_total = float(np.sqrt(self.norm))
        out = torch.zeros((3, self.N), **self.f64)
        drawn = 0
        while drawn < n_draws:
            size = min(block, n_draws - drawn)
            q = self._draws(size, seed, drawn)
            if self.inv_root is not None:
                q = q * self.inv_root[:, None]
            levels, _, gsum = self._to_coef(q)
            grand = levels[psi].sum(dim=0) / self.total
            rhs_l = torch.zeros((L, 2 * size), **self.f64)
            rhs_l[psi, :size] = (levels[psi] - torch.outer(self.level_w[psi], grand)) / root_total
            rhs_g = torch.zeros((G, 2 * size), **self.f64)
            rhs_g[:, size:] = (gsum - torch.outer(self.group_w, grand)) / root_total
            U_l, U_c, U_g = self._apply_inverse(rhs_l, torch.zeros((self.c, 2 * size),
                                                                   **self.f64), rhs_g)
            rows = self._readout(U_l, U_c, U_g, root=False)
            _lib.check(_lib.lib().hdfe_bii_moments(rows.data_ptr(), size, self.op._ptr(self.op.w),
                                                   self.N, out.data_ptr(),
                                                   _lib.stream_handle()))
            drawn += size
        return out / n_draws

    # ---- Q and C

    def apply_q(self, k, U_l, U_g):
        """leaveout_se.py:339-385 `_apply_q`: Q_k u as (levels, groups)."""
        torch = _torch()
        psi, norm, total = self.psi, self.norm, self.total
        m = int(U_l.shape[1])
        out_l = torch.zeros((self.L, m), **self.f64)
        out_g = torch.zeros((self.G, m), **self.f64)
        level_w = self.level_w[psi]
        base = U_l[psi]
        psi_mean = (level_w @ base) / total
        alpha_mean = (self.group_w @ U_g) / total
        if k == 0:
            out_l[psi] = level_w[:, None] * (base - psi_mean) / norm
        elif k == 1:
            out_g[:] = self.group_w[:, None] * (U_g - alpha_mean) / norm
        else:
            op = self.op
            cross_l = torch.zeros((self.L, m), **self.f64)
            cross_g = torch.empty((self.G, m), **self.f64)
            for j0 in range(0, m, MAX_BLOCK):
                j1 = min(m, j0 + MAX_BLOCK)
                cl = torch.zeros((self.L, j1 - j0), **self.f64)
                cg = torch.empty((self.G, j1 - j0), **self.f64)
                ul = U_l[:, j0:j1].contiguous()
                ug = U_g[:, j0:j1].contiguous()
                _lib.check(_lib.lib().hdfe_cov_cross(
                    *self._base(), self.psi_column, op._ptr(op.w), ul.data_ptr(), ug.data_ptr(),
                    j1 - j0, cl.data_ptr(), cg.data_ptr(), op._status().data_ptr(),
                    _lib.stream_handle()))
                cross_l[:, j0:j1] = cl
                cross_g[:, j0:j1] = cg
            out_l[psi] = (cross_l[psi] - level_w[:, None] * alpha_mean) / (2 * norm)
            out_g[:] = (cross_g - self.group_w[:, None] * psi_mean) / (2 * norm)
        return out_l, out_g

    def m_times(self, b):
        """leaveout_se.py:387-424 `_m_times`: u_k = M b_k for the three rows
        of b (3, N), one solve for all three."""
        rhs = b.t().contiguous()
        if self.inv_root is not None:
            rhs = rhs * self.inv_root[:, None]
        levels, cov, gsum = self._to_coef(rhs)
        U_l, U_c, U_g = self._apply_inverse(levels, cov, gsum)
        return (b - self._readout(U_l, U_c, U_g, root=True).t()).contiguous()

    def c_sums(self, v, b, s, per_component, y=None, u=None, deflate=None, g=None):
        """leaveout_se.py:426-597 `_apply_c` with its sinks: C v for the three
        components (v (N, size) shared, or the draws z scaled per component by
        sqrt(max(s_k, 0)) when per_component), returned as sums[6]: per k the
        sum of s_k (C v)_k^2 over rows and draws, then of y (C v)_k.  With
        u = M b (3, N), the kernel is the reference-centred K = C +
        (1 u' + u 1') / (2 N) (:536-543, :591-595); with deflate = (lambda (3,),
        x1 (3, N)) B loses lambda_k x1_k x1_k' (:580-582); with g (3, N) sums
        has 9 entries, the last three sum_i g_ki (C v)_ki0."""
        torch = _torch()
        size = int(v.shape[1])
        n_in = 3 if per_component else 1
        if per_component:
            scale = torch.sqrt(torch.clamp(s, min=0.0))
            ins = [v * scale[k][:, None] for k in range(3)]
        else:
            ins = [v]
        # the low-rank terms: per component a constant row and one row per vector
        vecs, rows_c = [], [[torch.zeros(size, **self.f64)] for _ in range(3)]
        if u is not None:
            half = 0.5 / self.N
            vecs.append(u)
            for k in range(3):
                vk = ins[k if per_component else 0]
                rows_c[k][0] = (u[k] @ vk) * half
                rows_c[k].append(vk.sum(0) * half)
        if deflate is not None:
            lams, x1 = deflate
            vecs.append(x1)
            for k in range(3):
                vk = ins[k if per_component else 0]
                rows_c[k].append(-float(lams[k]) * (x1[k] @ vk))
        coef = None
        if vecs:
            coef = torch.stack([torch.stack(r) for r in rows_c]).contiguous()
        stack = torch.cat(ins + [ins[k if per_component else 0] * b[k][:, None]
                                 for k in range(3)], 1)
        if self.inv_root is not None:
            stack = stack * self.inv_root[:, None]
        levels, cov, gsum = self._to_coef(stack)
        del stack
        U0_l, U0_c, U0_g = self._apply_inverse(levels, cov, gsum)
        q_l = torch.zeros((self.L, 3 * size), **self.f64)
        q_g = torch.zeros((self.G, 3 * size), **self.f64)
        for k in range(3):
            j = (k if per_component else 0) * size
            cols = slice(k * size, (k + 1) * size)
            q_l[:, cols], q_g[:, cols] = self.apply_q(k, U0_l[:, j:j + size],
                                                      U0_g[:, j:j + size])
        U1_l, U1_c, U1_g = self._apply_inverse(q_l, torch.zeros((self.c, 3 * size), **self.f64),
                                               q_g)
        base = self._readout(U0_l, U0_c, U0_g, root=True)
        thq = self._readout(U1_l, U1_c, U1_g, root=True)
        sums = torch.empty(9 if g is not None else 6, **self.f64)
        assert n_in * size + 3 * size == base.shape[1]
        v, b, s = v.contiguous(), b.contiguous(), s.contiguous()
        y = None if y is None else y.contiguous()
        g = None if g is None else g.contiguous()
        uv = torch.stack(vecs).contiguous() if vecs else None
        _lib.check(_lib.lib().hdfe_c_sums_ext(
            v.data_ptr(), size, int(bool(per_component)), b.data_ptr(), s.data_ptr(),
            base.data_ptr(), thq.data_ptr(), None if y is None else y.data_ptr(), len(vecs),
            None if uv is None else uv.data_ptr(), None if coef is None else coef.data_ptr(),
            None if g is None else g.data_ptr(), self.N, sums.data_ptr(), self._ws.data_ptr(),
            self._ws.numel(), _lib.stream_handle()))
        return sums

    # ---- the smoother of sigma2 (leaveout_se.py:982-1054)

    def smooth(self, sigma2, leverage, b_ii, n_bins=None):
        """sigma2 smoothed on (P_ii, B_ii), or on P_ii alone when b_ii is
        None, one value per row (device)."""
        torch = _torch()
        lib = _lib.lib()
        N = self.N
        dims = 1 if b_ii is None else 2
        n_bins = smoother_bins(N, dims) if n_bins is None else int(n_bins)
        if n_bins < 1:
            return sigma2
        if N <= QUANTILE_SAMPLE:
            take = None
        else:
            rng = np.random.default_rng(0)
            take = torch.as_tensor(np.sort(rng.choice(N, QUANTILE_SAMPLE, replace=False)),
                                   device=self.dev)

        def sample(x):
            return (x if take is None else x[take]).cpu().numpy()
        k0 = torch.as_tensor(smoother_knots(sample(leverage), n_bins), **self.f64)
        k1 = None if b_ii is None else \
            torch.as_tensor(smoother_knots(sample(b_ii), n_bins), **self.f64)
        fp = torch.as_tensor(np.linspace(0.0, 1.0, n_bins + 1), **self.f64)
        totals = torch.zeros(n_bins ** dims, **self.f64)
        counts = torch.zeros(n_bins ** dims, **self.f64)
        sh = _lib.stream_handle()
        leverage, sigma2 = leverage.contiguous(), sigma2.contiguous()
        b_ii = None if b_ii is None else b_ii.contiguous()
        k1_ptr = None if k1 is None else k1.data_ptr()
        b_ptr = None if b_ii is None else b_ii.data_ptr()
        _lib.check(lib.hdfe_smooth_cells(k0.data_ptr(), k1_ptr, fp.data_ptr(), n_bins,
                                         leverage.data_ptr(), b_ptr, sigma2.data_ptr(), N,
                                         totals.data_ptr(), counts.data_ptr(), sh))
        overall = totals.sum() / torch.clamp(counts.sum(), min=1.0)
        means = torch.where(counts > 0, totals / torch.clamp(counts, min=1.0), overall)
        out = torch.empty(N, **self.f64)
        _lib.check(lib.hdfe_smooth_eval(k0.data_ptr(), k1_ptr, fp.data_ptr(), n_bins,
                                        means.data_ptr(), leverage.data_ptr(), b_ptr, N,
                                        out.data_ptr(), sh))
        return out

    # ---- V

    def component_variances(self, sigma2, leverage, complement, factor, b_ii=None,
                            n_draws=250, block=8, seed=0, trace=True, smooth_bins=None,
                            stayer_rows=None, centering="weighted", reported=(0, 1, 2),
                            weak_id=None, weak_components=None, sigma2_point=None):
        """leaveout_se.py:599-784 `component_variances`: {"se", "variance",
        "first_term", "trace_term", "theta", "se_conservative", "weak"} per
        component.  sigma2, leverage, complement and factor come from
        `leave_out_components` / `jla_leverages`; b_ii from `bii_rows`
        (computed here with the same draws when None).  Leaving out a match:
        `stayer_rows` (bool, N) zeroes b on the stayers' matches,
        centering "reference" applies the rank-two kernel to the uncentred
        outcome, and components outside `reported` are NaN.  With `weak_id`
        (`weakid.weak_id_diagnostics`), "weak" holds the q = 1 moments
        (`weak_moments`, seed + 8_800_021) of the flagged components (by
        default those with q >= 1; at match level var(psi) alone), sigma2_point
        the point estimate's sigma2 when `sigma2` is another (:737-759)."""
        torch = _torch()
        f64 = self.f64
        sigma2 = torch.as_tensor(sigma2).to(**f64)
        leverage = torch.as_tensor(leverage).to(**f64)
        complement = torch.as_tensor(complement).to(**f64)
        factor = torch.as_tensor(factor).to(**f64)
        if b_ii is None:
            b_ii = self.bii_rows(n_draws, min(int(block), MAX_BLOCK // 2), seed)
        b_ii = torch.as_tensor(b_ii).to(**f64)
        if centering not in ("weighted", "reference"):
            raise ValueError("centering must be 'reference' or 'weighted'")
        b = b_ii * (factor / complement)[None, :]
        if stayer_rows is not None:
            keep = ~torch.as_tensor(stayer_rows, device=self.dev).to(torch.bool)
            b = torch.where(keep[None, :], b, torch.zeros_like(b))
        b = b.contiguous()
        u = self.m_times(b) if centering == "reference" else None
        s = torch.stack([self.smooth(sigma2, leverage, b_ii[k], smooth_bins)
                         for k in range(3)]).contiguous()
        op = self.op
        y = op.rows.V[0]
        w = op.w if op.w is not None else torch.ones(self.N, **f64)
        y_bar = float((w @ y).item() / w.sum().item()) if centering == "weighted" else 0.0
        shifted = (torch.sqrt(w) * (y - y_bar)).contiguous()
        sums = self.c_sums(shifted[:, None].contiguous(), b, s, False, y=shifted,
                           u=u).cpu().numpy()
        first = 4.0 * sums[:3]
        theta = sums[3:]
        tr = np.zeros(3)
        blocks = 0
        if trace:
            block = int(min(max(int(block), 1), MAX_BLOCK))
            drawn = 0
            while drawn < n_draws:
                size = min(block, n_draws - drawn)
                z = self._draws(size, int(seed) + TRACE_SEED_OFFSET, drawn)
                tr += self.c_sums(z, b, s, True, u=u).cpu().numpy()[:3]
                drawn += size
                blocks += 1
            tr /= n_draws
        names = list(COMPONENTS)
        weak = None
        if weak_id is not None:
            if weak_components is None:
                weak_components = [k for k in range(3) if weak_id["q"][k] >= 1]
            weak_components = [k for k in weak_components
                               if k in reported and (stayer_rows is None or k == 0)]
            if weak_components:
                point = sigma2 if sigma2_point is None else \
                    torch.as_tensor(sigma2_point).to(**f64)
                weak = self.weak_moments(point, s, b_ii, complement, factor, weak_id,
                                         weak_components, n_draws, block,
                                         int(seed) + WEAK_SEED_OFFSET, stayer_rows, centering)
                weak = {names[k]: v for k, v in weak.items()}
        variance = first - 2.0 * tr
        for k in range(3):
            if k not in reported:
                variance[k] = first[k] = tr[k] = theta[k] = np.nan
        return {"se": {n: float(np.sqrt(v)) if v > 0 else float("nan")
                       for n, v in zip(names, variance)},
                "variance": dict(zip(names, variance.tolist())),
                "first_term": dict(zip(names, first.tolist())),
                "trace_term": dict(zip(names, (2.0 * tr).tolist())),
                "theta": dict(zip(names, theta.tolist())),
                "se_conservative": {n: float(np.sqrt(f)) if f > 0 else float("nan")
                                    for n, f in zip(names, first)},
                "n_draws": n_draws if trace else 0, "blocks": blocks, "weak": weak}

    def weak_moments(self, sigma2, s, b_ii, complement, factor, weak_id, components, n_draws,
                     block, seed, stayer_rows=None, centering="weighted"):
        """leaveout_se.py:786-888 `_weak_moments`: per flagged component k
        {"lambda_1", "b1", "v_raw", "sigma" (2x2), "conservative", "trace",
        "quadratic"}: b1 = x1' y~ with x1 = sqrt(w) A u1 (u1 the leading
        direction), v_raw = sum x1^2 sigma2, and the covariance of (b1,
        theta1) from the deflated kernel C2 (B2 = B - lambda_1 x1 x1', b2 from
        diag(B2), the low-rank terms of `c_sums`), s the smoothed sigma2
        floored at zero; the first term alone where subtracting the trace
        leaves the matrix indefinite."""
        torch = _torch()
        f64 = self.f64
        lams = np.array([float(e[0]) if len(e) else 0.0 for e in weak_id["eigenvalues"]])
        U = weak_id["lead_vectors"]
        x1 = self._readout(U[0], U[1], U[2], root=True).t().contiguous()       # (3, N)
        op = self.op
        y = op.rows.V[0]
        w = op.w if op.w is not None else torch.ones(self.N, **f64)
        root = torch.sqrt(w)
        y_bar = float((w @ y).item() / w.sum().item())
        yt = root * (y - y_bar)
        flo = torch.clamp(s, min=0.0).contiguous()
        b1 = (x1 @ yt).cpu().numpy()
        v_raw = ((x1 * x1) @ sigma2).cpu().numpy()
        s11 = (x1 * x1 * flo).sum(dim=1).cpu().numpy()
        lam_d = torch.as_tensor(lams, **f64)
        b2 = (b_ii - lam_d[:, None] * x1 * x1) * (factor / complement)[None, :]
        if stayer_rows is not None:
            keep = ~torch.as_tensor(stayer_rows, device=self.dev).to(torch.bool)
            b2 = torch.where(keep[None, :], b2, torch.zeros_like(b2))
        b2 = b2.contiguous()
        u2 = self.m_times(b2) if centering == "reference" else None
        shift = y_bar if centering == "weighted" else 0.0
        y_c = (root * (y - shift)).contiguous()
        deflate = (lams, x1)
        sums = self.c_sums(y_c[:, None].contiguous(), b2, flo, False, y=y_c, u=u2,
                           deflate=deflate, g=(x1 * flo)).cpu().numpy()
        first, quad, s12 = 4.0 * sums[:3], sums[3:6], 2.0 * sums[6:9]
        # the trace with only the flagged components drawn (leaveout_se.py:890-930
        # `_cc_trace`, clamp=True): the others get a zero input and weight
        mask = torch.zeros(3, **f64)
        mask[list(components)] = 1.0
        flo_m = (flo * mask[:, None]).contiguous()
        trace = np.zeros(3)
        block = int(min(max(int(block), 1), MAX_BLOCK))
        drawn = 0
        while drawn < n_draws:
            size = min(block, n_draws - drawn)
            z = self._draws(size, int(seed), drawn)
            trace += self.c_sums(z, b2, flo_m, True, u=u2, deflate=deflate).cpu().numpy()[:3]
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


def weak_intervals(leave_out, weak, confidence=0.95):
    """leaveout.py:774-791: for each flagged component, theta1 = the
    leave-out estimate less lambda_1 (b1^2 - v_raw), and the q = 1 interval
    (`am_interval.am_interval`) around it; `leave_out` maps the component
    names (or indexes 0..2) to the estimates.  Adds "theta1", "interval",
    "confidence", "kappa", "z", "rho" to each piece of `weak` and returns it."""
    from .am_interval import am_interval
    for name, piece in (weak or {}).items():
        k = COMPONENTS.index(name)
        est = leave_out[name] if isinstance(leave_out, dict) else leave_out[k]
        theta1 = float(est) - piece["lambda_1"] * (piece["b1"] ** 2 - piece["v_raw"])
        lo, hi, info = am_interval(piece["lambda_1"], piece["b1"], theta1, piece["sigma"],
                                   1.0 - confidence)
        piece.update(theta1=theta1, interval=(lo, hi), confidence=confidence, **info)
    return weak

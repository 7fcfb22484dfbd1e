"""The weak-identification diagnostic of the leave-out components on the
device (leaveout_weakid.py:565-713 `weak_id_diagnostics`).

KSS Theorem 2 (ii) wants lambda_1^2 / sum lambda^2 small for the
eigenvalues of S^- Q; q counts the leading ratios at or above 1/10.  The
eigenvalues come from Lanczos on Q S^-, self-adjoint in <x, y> = x' S^- y, for
the three components in lockstep: a step is one application of Q per
component (coefficient space, `hdfe_cov_cross` for the covariance) and one
solve of three columns (`InverseOperator.apply_inverse`, the library's PCG).
The recurrence keeps three vectors per component; where a component's basis
fits the scratch budget (the reference's `_krylov_plan` rule, :185-215) it is
kept and every new vector reorthogonalized against it twice.  Ghost copies are
merged and spurious singletons dropped on the host (Cullum-Willoughby,
`ritz_top`, :386-434).  The leading Ritz vectors are rebuilt by retracing the
deterministic recurrence; sum lambda^2 is their exact part plus deflated
Hutchinson draws (:467-555); the first-stage F reads the leading direction back
per row against sigma2 smoothed on the leverage (:715-744).  Every vector lives
in HBM as a device tensor; only the tridiagonals travel to the host.
"""

from __future__ import annotations

import numpy as np

from .leaveout_se import StandardErrors

WEAK_ID_THRESHOLD = 0.1             # leaveout_weakid.py:64 (KSS Section 6.2)
SUM_SQ_SEED_OFFSET = 3_300_007      # leaveout_weakid.py:663
MIN_DRAWS = 16                      # leaveout_weakid.py:468


def _torch():
    import torch
    return torch


GHOST_TOL = 1e-8        # leaveout_weakid.py:403: copies of one converged eigenvalue
SPURIOUS_TOL = 1e-11    # leaveout_weakid.py:422: the Cullum-Willoughby match


def ritz_top(alpha, beta, top):
    """The `top` leading genuine Ritz values of the Lanczos tridiagonal
    T = tridiag(beta[:-1], alpha, beta[:-1]), with their error bounds
    |beta[-1] s_m| (s_m the eigenvector's last entry) and eigenvectors, as
    the reference's `_ritz_top` (leaveout_weakid.py:386-434) selects them:

    * ghosts -- in floating point a converged eigenvalue reappears as
      further Ritz values that agree with it to the convergence level, far
      closer than two genuine eigenvalues: sorted Ritz values chained by gaps
      of at most 1e-8 max|theta| are one eigenvalue, represented by the
      member with the smallest error bound;
    * spurious values (Cullum and Willoughby, 1985) -- a value seen once
      that is also an eigenvalue of T without its first row and column (to
      1e-11 max|theta|) is not an eigenvalue of the operator.

    The survivors are ranked by |theta|."""
    from scipy.linalg import eigh_tridiagonal, eigvalsh_tridiagonal
    diag = np.asarray(alpha, float)
    m = len(diag)
    if m == 0:
        return np.array([]), np.array([]), np.zeros((0, 0))
    sub = np.asarray(beta, float)[:m - 1]
    theta, vecs = eigh_tridiagonal(diag, sub)          # ascending
    err = np.abs(float(beta[m - 1]) * vecs[m - 1])
    scale = max(float(np.max(np.abs(theta))), 1e-300)
    # runs of the sorted values: a new run starts where the gap to the run's
    # current representative exceeds the ghost tolerance
    run_of = np.empty(m, np.int64)
    reps, sizes = [], []
    for i in np.argsort(theta):
        if reps and theta[i] - theta[reps[-1]] <= GHOST_TOL * scale:
            sizes[-1] += 1
            if err[i] < err[reps[-1]]:
                reps[-1] = i
        else:
            reps.append(i)
            sizes.append(1)
        run_of[i] = len(reps) - 1
    reps, sizes = np.array(reps, np.int64), np.array(sizes, np.int64)
    if m > 1:
        deleted = eigvalsh_tridiagonal(diag[1:], sub[1:]) if m > 2 else diag[1:]
        near = np.min(np.abs(deleted[None, :] - theta[reps][:, None]), axis=1)
        genuine = (sizes > 1) | (near > SPURIOUS_TOL * scale)
        reps = reps[genuine]
    ranked = reps[np.argsort(-np.abs(theta[reps]), kind="stable")][:top]
    return theta[ranked], err[ranked], vecs[:, ranked]


class _Lanczos:
    """Coefficient triples [levels (L, m), covariates (c, m), groups (G, m)]
    and the operations the recurrence needs, on the device."""

    def __init__(self, se: StandardErrors, seed: int, caps, reorth):
        torch = _torch()
        self.se, self.seed = se, int(seed)
        self.caps, self.reorth = list(caps), list(reorth)
        self.L, self.c, self.G = se.L, se.c, se.G
        self.psi = se.psi
        self.n_psi = se.psi.stop - se.psi.start
        self.f64 = se.f64
        self.torch = torch

    def zeros(self, m):
        t = self.torch
        return [t.zeros((self.L, m), **self.f64), t.zeros((self.c, m), **self.f64),
                t.zeros((self.G, m), **self.f64)]

    def q_block(self, comps, U_l, U_g):
        """Q applied column by column, column j with component comps[j]
        (leaveout_weakid.py:163-179)."""
        torch = self.torch
        out_l, out_g = torch.zeros_like(U_l), torch.zeros_like(U_g)
        comps = np.asarray(comps)
        for k in range(3):
            cols = np.flatnonzero(comps == k)
            if len(cols) == 0:
                continue
            idx = torch.as_tensor(cols, device=U_l.device)
            ql, qg = self.se.apply_q(k, U_l[:, idx].contiguous(), U_g[:, idx].contiguous())
            out_l[:, idx], out_g[:, idx] = ql, qg
        return out_l, out_g

    def solve(self, t):
        U_l, U_c, U_g = self.se._apply_inverse(t[0], t[1], t[2])
        return [U_l, U_c, U_g]

    @staticmethod
    def dot(a, b):
        return sum((x * y).sum(dim=0) for x, y in zip(a, b))

    def support(self, k, t):
        parts = []
        if k in (0, 2):
            parts.append(t[0][self.psi, k])
        if k in (1, 2):
            parts.append(t[2][:, k])
        return self.torch.cat(parts) if len(parts) > 1 else parts[0].clone()

    def scatter(self, k, flat, t):
        at = 0
        if k in (0, 2):
            t[0][self.psi, k] -= flat[:self.n_psi]
            at = self.n_psi
        if k in (1, 2):
            t[2][:, k] -= flat[at:]

    def project(self, t):
        """Back onto range(Q_k): zero mean on the blocks each column touches
        (leaveout_weakid.py:252-270)."""
        for k in (0, 2):
            t[0][self.psi, k] -= t[0][self.psi, k].mean()
        for k in (1, 2):
            t[2][:, k] -= t[2][:, k].mean()

    def run(self, n_iter, ritz=None, check=None, every=20):
        """leaveout_weakid.py:217-383 `_lanczos`: (alphas, betas, lengths,
        steps), or with `ritz` the accumulated Ritz combinations (X, Y)."""
        torch = self.torch
        se = self.se
        # x0 = Q r, r Rademacher over the levels, covariates and groups
        r = []
        for pos, n in ((0, self.L), (self.L, self.c), (self.L + self.c, self.G)):
            r.append(se._draws_at(n, pos, 3, self.seed, 0))
        ql, qg = self.q_block([0, 1, 2], r[0], r[2])
        x = [ql, torch.zeros((self.c, 3), **self.f64), qg]
        self.project(x)
        y = self.solve(x)
        nrm = torch.sqrt(torch.clamp(self.dot(x, y), min=0.0)).cpu().numpy()
        live = (nrm > 0) & (np.array(self.caps) > 0)
        self._normalize(x + y, live, nrm)
        x_prev = self.zeros(3)
        beta_prev = np.zeros(3)
        basis = [([], []) for _ in range(3)]
        alphas, betas = [[], [], []], [[], [], []]
        lengths = np.zeros(3, dtype=int)
        acc = None
        if ritz is not None:
            kk = ritz[0].shape[1]
            acc = (self.zeros(3 * kk), self.zeros(3 * kk))
            ritz_d = [torch.as_tensor(rz, **self.f64) for rz in ritz]
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
                            ax[:, cols] += torch.outer(xb[:, k], ritz_d[k][j])
                            ay[:, cols] += torch.outer(yb[:, k], ritz_d[k][j])
            for k in np.flatnonzero(live):
                if self.reorth[k]:
                    basis[k][0].append(self.support(k, x))
                    basis[k][1].append(self.support(k, y))
            ql, qg = self.q_block([0, 1, 2], y[0], y[2])
            w = [ql, torch.zeros((self.c, 3), **self.f64), qg]
            bp = torch.as_tensor(beta_prev, **self.f64)
            for wb, xp in zip(w, x_prev):
                wb -= bp * xp
            alpha = self.dot(w, y)
            for wb, xb in zip(w, x):
                wb -= alpha * xb
            fix = self.dot(w, y)
            for wb, xb in zip(w, x):
                wb -= fix * xb
            alpha = alpha + fix
            self.project(w)
            for k in np.flatnonzero(live):
                if not self.reorth[k] or not basis[k][0]:
                    continue
                Xs = torch.stack(basis[k][0], dim=1)
                Ys = torch.stack(basis[k][1], dim=1)
                for _ in range(2):
                    wk = self.support(k, w)
                    self.scatter(k, Xs @ (Ys.T @ wk), w)
            self.project(w)
            z = self.solve(w)
            beta = torch.sqrt(torch.clamp(self.dot(w, z), min=0.0)).cpu().numpy()
            alpha = alpha.cpu().numpy()
            beta_max = np.maximum(beta_max, beta)
            for k in np.flatnonzero(live):
                alphas[k].append(float(alpha[k]))
                betas[k].append(float(beta[k]))
                lengths[k] = j + 1
            live = (live & (beta > 1e-8 * np.maximum(beta_max, 1e-300))
                    & (lengths < np.array(self.caps)))
            x_prev = x
            x = [wb.clone() for wb in w]
            y = z
            self._normalize(x + y, live, beta)
            beta_prev = np.where(live, beta, 0.0)
        if acc is not None:
            return acc
        return [np.array(a) for a in alphas], [np.array(b) for b in betas], lengths, steps

    def _normalize(self, blocks, live, by):
        """Live columns divided by `by`, the others zeroed."""
        torch = self.torch
        div = torch.as_tensor(np.where(live, by, 1.0), **self.f64)
        keep = torch.as_tensor(live, device=div.device)
        for t in blocks:
            if t.shape[0]:
                t.copy_(torch.where(keep, t / div, torch.zeros_like(t)))


def weak_id_diagnostics(se: StandardErrors, sigma2, leverage, n_draws=64, block=32, seed=0,
                        max_iter=150, tol=1e-4, top=3, smooth_bins=None, scratch_mb=32):
    """leaveout_weakid.py:565-713 `weak_id_diagnostics` for the design of
    `se` (psi its `psi_column`; no covariates): per component the leading
    eigenvalues of S^- Q with their error bounds, sum lambda^2 and its Monte
    Carlo standard error, the ratios lambda_l^2 / sum, q, whether q reached
    the count of eigenvalues found (q_capped), whether a ratio sits within
    two standard errors of the threshold (q_borderline), the first-stage F,
    and whether Lanczos converged; `scratch_mb` the reference's scratch budget
    (its default 32), which decides full reorthogonalization and how many
    Ritz vectors deflate the trace, so the arithmetic follows it."""
    torch = _torch()
    if n_draws < 2:
        raise ValueError("n_draws must be at least 2, so the Monte Carlo error of sum "
                         "lambda^2 can be reported")
    if se.c:
        raise ValueError("weak_id_diagnostics: designs with covariates are not supported")
    f64 = se.f64
    L, c, G = se.L, se.c, se.G
    n_psi = se.psi.stop - se.psi.start
    # leaveout_weakid.py:185-215 `_krylov_plan`
    dims = [max(n_psi - 1, 0), max(L + c + 1, 1), max(2 * (n_psi - 1), 0)]
    rows = [n_psi, G, n_psi + G]
    budget = int(scratch_mb) << 20
    caps = [min(max_iter, d) for d in dims]
    reorth = [cap * 2 * r * 8 <= budget for cap, r in zip(caps, rows)]
    lz = _Lanczos(se, seed, caps, reorth)

    def converged_all(alphas, betas, lengths, steps):
        for k in range(3):
            if lengths[k] < steps:
                continue
            theta, bounds, _ = ritz_top(alphas[k], betas[k], top)
            lead = float(np.abs(theta[0])) if len(theta) else 0.0
            if np.any(bounds[:2] > tol * max(lead, 1e-300)):
                return False
        return True

    alphas, betas, lengths, n_iter = lz.run(max_iter, check=converged_all, every=10)
    checked = [ritz_top(alphas[k], betas[k], top) for k in range(3)]
    kk = top if 2 * 3 * top * (L + c + G) * 8 <= budget else 1
    ritz = []
    for _, _, S in checked:
        coef = np.zeros((S.shape[0], kk))
        coef[:, :min(kk, S.shape[1])] = S[:, :kk]
        ritz.append(coef)
    X, Y = lz.run(n_iter, ritz=ritz)
    # leaveout_weakid.py:436-465: modified Gram-Schmidt in <x, y> = x' S^- y
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
            n2 = float(sum(xb[:, ca] @ yb[:, ca] for xb, yb in zip(X, Y)))
            lead = float(sum(xb[:, base] @ yb[:, base] for xb, yb in zip(X, Y)))
            if n2 <= 1e-20 * max(lead, 1e-300) or n2 <= 0:
                for t in (*X, *Y):
                    t[:, ca] = 0.0
                continue
            for t in (*X, *Y):
                t[:, ca] *= 1.0 / np.sqrt(n2)
    u = [t[:, ::kk].contiguous() for t in Y]
    leading = [theta for theta, _, _ in checked]

    # leaveout_weakid.py:467-555 `_sum_sq_eigenvalues`
    comps = [k for k in range(3) for _ in range(kk)]
    ql, qg = lz.q_block(comps, Y[0], Y[2])
    zq = lz.solve([ql, torch.zeros((c, 3 * kk), **f64), qg])
    exact = ((ql * zq[0]).sum(0) + (qg * zq[2]).sum(0)).reshape(3, kk).sum(dim=1).cpu().numpy()

    def summarize(values):
        n = values.shape[1]
        sd = values.std(axis=1, ddof=1) / np.sqrt(n) if n > 1 else np.full(3, np.nan)
        return exact + values.mean(axis=1), sd

    def settled(est, sd):
        for k in range(3):
            if not est[k] > 0 or not np.isfinite(sd[k]):
                return False
            r = leading[k] ** 2 / est[k]
            if np.any(np.abs(r - WEAK_ID_THRESHOLD) < 2.0 * (sd[k] / est[k]) * r):
                return False
        return True

    draws, drawn = [], 0
    size = max(1, int(block) // 3)
    while drawn < n_draws:
        m = min(size, n_draws - drawn)
        xi = se._draws(m, int(seed) + SUM_SQ_SEED_OFFSET, drawn)
        if se.inv_root is not None:
            xi = xi * se.inv_root[:, None]
        zeta = list(se._to_coef(xi))
        yv = lz.solve(zeta)
        y_def = [torch.empty((t.shape[0], 3 * m), **f64) for t in yv]
        for k in range(3):
            cols = slice(k * kk, (k + 1) * kk)
            proj = sum(zb.T @ Yb[:, cols] for zb, Yb in zip(zeta, Y))
            for yd, yb, Yb in zip(y_def, yv, Y):
                yd[:, k * m:(k + 1) * m] = yb - Yb[:, cols] @ proj.T
        ql, qg = lz.q_block([k for k in range(3) for _ in range(m)], y_def[0], y_def[2])
        bq = lz.solve([ql, torch.zeros((c, 3 * m), **f64), qg])
        draws.append(((ql * bq[0]).sum(dim=0) + (qg * bq[2]).sum(dim=0)).reshape(3, m)
                     .cpu().numpy())
        drawn += m
        if drawn >= MIN_DRAWS and drawn < n_draws and settled(*summarize(np.hstack(draws))):
            break
    sum_sq, sum_sq_se = summarize(np.hstack(draws))

    # leaveout_weakid.py:715-744 `_first_stage_f`
    sigma2 = torch.as_tensor(sigma2).to(**f64)
    leverage = torch.as_tensor(leverage).to(**f64)
    smooth = se.smooth(sigma2, leverage, None, smooth_bins)
    x1 = se._readout(u[0], u[1], u[2], root=True)
    op = se.op
    y = op.rows.V[0]
    w = op.w if op.w is not None else torch.ones(se.N, **f64)
    y_t = torch.sqrt(w) * (y - (w @ y) / w.sum())
    num = (x1.T @ y_t).cpu().numpy()
    den = ((x1 * x1).T @ smooth).cpu().numpy()
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
        out["q_borderline"].append(bool(np.any(np.abs(r - WEAK_ID_THRESHOLD)
                                               < 2.0 * rel_se * r)))
        out["converged"].append(bool(lengths[k] < n_iter or lengths[k] >= caps[k]
                                     or np.all(bnd[:2] <= tol * max(lead, 1e-300))))
    return out

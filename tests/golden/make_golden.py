"""Generate the golden vectors that pin the oracle to the reference.

Run once, in a container where the reference tree is readable:

    python tests/golden/make_golden.py /path/to/hdfe-stream

It imports the reference's own numba kernels and solver mixins (hdfe-stream
v0.13.4) from that tree -- with stand-in `polars` and `stream_limits` modules,
which the code on this path imports but does not call -- writes each panel's
rows in pass 0's Parquet layout (columns __hdfe_gcode, __hdfe_c1, __hdfe_c2,
__hdfe_v0..2, __hdfe_w), and drives the reference's pass 1
(`_PassesMixin._pass1_cells`), components (`_components`), explicit S
(`_build_explicit`), block PCG (`_pcg` through `_make_block_solver`), the full
step-2 solve with normalisation (`_solve`), the inverse operator
(`project_rows`, `apply_inverse`), the JLA leverages (`jla_leverages`) and the
Hutchinson trace (`hutchinson_trace`) on them.  Inputs and outputs go to
tests/golden/<panel>.npz.  Nothing at test time reads the reference.
"""

from __future__ import annotations

import importlib
import logging
import sys
import tempfile
import types
from pathlib import Path

import numpy as np

REPO = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(REPO))

from hdfe_stream_b200.simulate import pass0_layout, simulate_panel  # noqa: E402

NUMBA_THREADS = 4


def import_reference(root: str):
    class _Anything:
        def __getattr__(self, k):
            return _Anything()

        def __call__(self, *a, **k):
            return _Anything()

    for name in ("polars", "stream_limits"):
        stub = types.ModuleType(name)
        stub.__getattr__ = lambda k: _Anything()
        sys.modules[name] = stub
    for name, sub in (("hdfe_stream", "hdfe_stream"), ("hdfe_stream.core", "hdfe_stream/core")):
        mod = types.ModuleType(name)
        mod.__path__ = [str(Path(root) / sub)]
        sys.modules[name] = mod
    import numba
    numba.set_num_threads(NUMBA_THREADS)
    mods = {n: importlib.import_module(f"hdfe_stream.{n}") for n in
            ("core.passes", "core.solve", "inverse", "leaveout", "core.kernels_groups",
             "core.kernels_base", "core.connected", "core.kernels_graph")}
    return mods


def write_rows(rows, path):
    import pyarrow as pa
    import pyarrow.parquet as pq
    cols = {"__hdfe_gcode": pa.array(rows.gcode, pa.uint32()),
            "__hdfe_c1": pa.array(rows.codes[:, 0], pa.uint32()),
            "__hdfe_c2": pa.array(rows.codes[:, 1], pa.uint32())}
    for j in range(rows.V.shape[1]):
        cols[f"__hdfe_v{j}"] = pa.array(rows.V[:, j])
    if rows.w is not None:
        cols["__hdfe_w"] = pa.array(rows.w)
    pq.write_table(pa.table(cols), path)


def make_estimator(mods, rows, workdir: Path):
    passes, solve = mods["core.passes"], mods["core.solve"]
    inverse, leaveout = mods["inverse"], mods["leaveout"]

    class Budget:
        def fits(self, *a, **k):
            return True

        def headroom_gb(self, *a, **k):
            return 64.0

    class Est(passes._PassesMixin, solve._SolveMixin, inverse._InverseMixin,
              leaveout._LeaveOutMixin, leaveout._TraceMixin):
        def _offsets(self):
            off, o = {}, 0
            for f in self.o_fe:
                off[f] = o
                o += self.n_levels[f]
            return off, o

        def _s_limit_gb(self, upcoming_gb=0.0):
            return 64.0

        def _acc_copies(self, levels, width):
            import numba
            return numba.get_num_threads()

        def _log(self, msg):
            pass

        def _debug(self, msg):
            pass

        def _track_disk(self):
            pass

        def _moment_divisor(self, total):
            rows = self.n_obs
            return total * (rows - 1.0) / rows if rows > 1 else total

    est = Est()
    path = workdir / "rows.parquet"
    write_rows(rows, path)
    m = rows.V.shape[1]
    est.__dict__.update(
        collapse=True, combos_ratio=None, m=m, cell_sums=True,
        o_fe=["firm", "year"], g_fe="worker", fe=["worker", "firm", "year"],
        n_levels={"worker": rows.n_groups, "firm": rows.n_levels[0], "year": rows.n_levels[1]},
        rhs_block=8, budget=Budget(), slope_vars=[], p=1, assembly="cells", solver="explicit",
        device="cpu", precond="jacobi", tol=1e-12, maxiter=5000, verbose=False, logger=None,
        log_level=logging.INFO, ccols=["__hdfe_c1", "__hdfe_c2"],
        weights=None if rows.w is None else "w", means=rows.V.mean(axis=0),
        tmeans=np.zeros(0), batch_rows=10**9, cells_in_memory=True,
        var_names=list(rows.names), raw_ss=rows.V.var(axis=0, ddof=1) * (rows.n_rows - 1),
        n_obs=rows.n_rows, models=[{"x": ()}], workdir=workdir,
        paths={"rows": [str(path)], "rhs": str(workdir / "rhs.npy"),
               "gamma": str(workdir / "gamma.npy"),
               "ident": {k: str(workdir / f"ident_{k}.bin") for k in
                         ("codes", "n", "sums", "st", "ainv", "cmat")}
               | {"starts": str(workdir / "ident_starts.npy")}})
    return est


def run_panel(mods, name, rows, out_dir: Path):
    kg = mods["core.kernels_groups"]
    with tempfile.TemporaryDirectory() as tmp:
        est = make_estimator(mods, rows, Path(tmp))
        est._pass1_cells()
        rhs = np.array(est._rhs_pass1)          # consumed by _solve
        est._components()
        out = dict(
            gcode=rows.gcode, codes_rows=rows.codes, V=rows.V,
            w=rows.w if rows.w is not None else np.zeros(0),
            n_levels=np.array(rows.n_levels, np.int64), n_groups=rows.n_groups,
            means=est.means, raw_ss=est.raw_ss,
            starts=np.array(est.starts), codes=np.array(est.codes), n=np.array(est.n),
            sums=np.array(est.sums), obs=est.obs, cnt=est.cnt, diag=est.diag, rhs=rhs,
            comp=np.array(est.comp), n_components=est.n_components, n_cells=est.n_cells,
            fe0_rank=est.fe0_rank,
            pair_components=np.array([est.pair_components[k] for k in sorted(
                est.pair_components)], np.int64))
        S, _ = est._build_explicit()
        out.update(S_indptr=S.indptr.astype(np.int64), S_indices=S.indices.astype(np.int32),
                   S_data=S.data)
        # the block PCG on a right-hand side with a zero column and a warm start
        solve_fn, _ = est._make_block_solver()
        rng = np.random.default_rng(3)
        L = S.shape[0]
        b = S @ rng.standard_normal((L, 4))
        b[:, 1] = 0.0
        zero = np.array([False, True, False, False])
        X, it, ok, rel = solve_fn(b, zero, None)
        x0 = np.zeros_like(b)
        x0[:, 2] = X[:, 2]
        X2, it2, ok2, rel2 = solve_fn(b, zero, x0)
        out.update(pcg_b=b, pcg_zero=zero, pcg_X=X, pcg_it=it, pcg_ok=ok, pcg_rel=rel,
                   pcg_x0=x0, pcg_X2=X2, pcg_it2=it2, pcg_ok2=ok2, pcg_rel2=rel2,
                   tol=est.tol)
        # step 2 in full: blocks, zero detection, normalisation
        est._rhs_pass1 = rhs.copy()
        gamma, info = est._solve(in_memory=True)
        out.update(gamma=np.array(gamma), gamma_iterations=np.atleast_1d(info["iterations"]),
                   gamma_converged=info["converged"])
        # counter-based draws
        out["rademacher"] = np.empty((257, 5))
        kg._nb_rademacher(1000, 257, 5, 12345, 7, out["rademacher"])
        # inverse operator: projection of Rademacher row vectors
        proj = np.zeros((rows.n_rows, 6))

        def sink(ordinal, chunk, projected):
            proj[ordinal:ordinal + len(projected)] = projected
        est.project_rows(est.rademacher(seed=11), 6, sink,
                         sqrt_weights=rows.w is not None)
        out["project_rows_seed11"] = proj
        # S^- for a coefficient-space vector
        rng = np.random.default_rng(5)
        lv = rng.standard_normal((L, 3))
        gv = rng.standard_normal((rows.n_groups, 3))
        rows_out = np.zeros((rows.n_rows, 3))

        def sink2(ordinal, chunk, values):
            rows_out[ordinal:ordinal + len(values)] = values
        U, C, Ug = est.apply_inverse(lv, np.zeros((0, 3)), gv, sink=sink2)
        out.update(ainv_levels=lv, ainv_groups=gv, ainv_U=U, ainv_Ug=Ug, ainv_rows=rows_out)
        # JLA leverages and the Hutchinson trace
        lev = est.jla_leverages(n_draws=24, block=8, seed=2, in_memory=True, covariates=())
        out.update(jla_leverage=np.array(lev.leverage), jla_factor=np.array(lev.factor))
        sigma2 = np.abs(np.random.default_rng(9).standard_normal(rows.n_rows)) + 0.1
        tr = est.hutchinson_trace(sigma2, n_draws=16, block=8, seed=4, covariates=())
        out.update(trace_sigma2=sigma2,
                   trace=np.array([tr.var_psi, tr.var_alpha, tr.cov]))
    out["numba_threads"] = NUMBA_THREADS
    np.savez_compressed(out_dir / f"{name}.npz", **out)
    print(f"{name}: rows {rows.n_rows}, L {L}, nnz {len(S.data)}, cells {est.n_cells}, "
          f"pcg it {it}/{it2}, gamma it {info['iterations']}")


# The golden panels: small enough to commit, shaped like the measured ones.
GOLDEN = {
    # 2,000 workers, 200 firms, 10 years, 8 consecutive years each
    "akm_small": (dict(n_workers=2_000, n_firms=200, n_years=10, spell=(8, 8), p_move=0.1,
                       seed=101), None),
    # weighted (U[0.5, 2]), uneven spells 1-10 years: single-row workers,
    # which pass 1 drops as non-identifying
    "akm_weighted": (dict(n_workers=1_500, n_firms=120, n_years=10, spell=(1, 10),
                          p_move=0.15, weights=True, seed=202), None),
    # few movers and several connected components
    "akm_components": (dict(n_workers=600, n_firms=150, n_years=6, spell=(2, 6),
                            p_move=0.02, seed=303), None),
}


def main(root):
    mods = import_reference(root)
    out_dir = Path(__file__).resolve().parent
    for name, (kw, keep) in GOLDEN.items():
        panel = simulate_panel(**kw)
        rows = pass0_layout(panel, keep)
        run_panel(mods, name, rows, out_dir)


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else "/root/reference")

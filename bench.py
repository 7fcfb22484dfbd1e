"""Benchmark of the fixed-effects solve path on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

One step is one AKM fit's hot path over the 5M-worker panel (5,000,000
workers, 500,000 firms, 15 years, ~8.5 rows per worker, yearly move
probability 0.08; largest connected set after min_degree = 2), model
log_earn ~ age_squared + age_cubed | worker_id + firm_id + year:
pass 1 (cells, identifying cells, obs/cnt, Jacobi diagonal, D_o'M_0V), the
explicit S, the connected components, the FP64 block PCG to tol 1e-10 and the
normalisation of the fixed effects -- on rows already in HBM (`value`), and
through the public call with host rows and the effects copied back (`e2e`).
The panel is built on the host first (generation and pass 0's layout and
restriction are not timed).  Under torchrun each rank fits its own panel
(weak scaling, no collective on the data path); rank 0 prints one JSON line.

`--impl reference` times the reference's CPU implementation of the same path
(the oracle's restatement of its numba kernels, all host threads) on the
same panel, rank 0 only.
"""

from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

REPO = Path(__file__).resolve().parent
sys.path.insert(0, str(REPO))

WORKLOAD = "akm_5m"
METRIC = "AKM fit throughput (pass 1 + S build + FP64 Jacobi PCG to 1e-10 + normalisation)"
UNIT = "fits/s"
PEAKS = REPO / "MEASURED_PEAKS.json"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=30)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", default=WORKLOAD)
    ap.add_argument("--tol", type=float, default=1e-10)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-jla", dest="jla", action="store_false",
                    help="skip the KSS-JLA leverage measurement")
    ap.add_argument("--kss-workload", default="kss_1m",
                    help="panel of the KSS measurement (kss_100k: a small case for profiling)")
    ap.add_argument("--parts", default="all",
                    help="comma list of the measurements besides the fit to run: accuracy, "
                         "kss, adjoint, batched, e2e, streamed (default all; for profiling)")
    return ap.parse_args()


def describe(name):
    """The panel preset in words (simulate.PANELS) and its restriction."""
    from hdfe_stream_b200.simulate import PANELS
    p = PANELS[name]
    lo, hi = p["spell"]
    text = (f"{name}: {p['n_workers']:,} workers, {p['n_firms']:,} firms, {p['n_years']} years, "
            f"spells of {lo}-{hi} years, p_move {p['p_move']}")
    if p.get("weights"):
        text += ", weights U[0.5, 2]"
    restriction = "leave-one-out connected set" if name.startswith("kss_") else \
        {"akm_5m": "largest connected set with min_degree=2",
         "akm_2m": "largest connected set with min_degree=2"}.get(name)
    return text + (f", {restriction}" if restriction else "")


def config(args, n, rows):
    return {"workload": describe(args.workload),
            "rows": rows.n_rows, "workers": rows.n_groups, "levels": int(sum(rows.n_levels)),
            "model": "log_earn ~ age_squared + age_cubed | worker_id + firm_id + year",
            "tol": args.tol, "parallelism": f"replicas{n}" if n > 1 else "single",
            "l2": "inputs (rows, S) larger than the 126 MB L2"}


# ------------------------------------------------------------------ clocks

class ClockSampler:
    """nvidia-smi samples of the SM clock and throttle reasons while running."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []

    def start(self, wait_s=10.0):
        """Start sampling and wait (up to wait_s) for the first sample, so that
        nvidia-smi's own start-up is over before anything is timed."""
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "50"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except FileNotFoundError:
            self.proc = None
            return
        t_end = time.monotonic() + wait_s
        while not self.lines and time.monotonic() < t_end and self.proc.poll() is None:
            time.sleep(0.02)

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append((time.monotonic(), line.strip()))

    def mark(self):
        """Host time stamps bracketing the timed region (samples outside are dropped)."""
        return time.monotonic()

    def stop(self, t_begin=None, t_end=None):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for t, line in self.lines:
            if (t_begin is not None and t < t_begin) or (t_end is not None and t > t_end):
                continue
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax = float(f[2])
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


# ----------------------------------------------------------- algorithmic bytes

def phase_bytes(rows, counts, S, iterations, m=3, small=None):
    """Compulsory DRAM bytes per launch of each phase (written out in the
    design notes): pass 1 reads each row once and writes the identifying
    cells and level arrays; the S build reads the cells and writes S; one
    PCG iteration reads S and streams the L x k vectors: 12 nnz + 4 (L+1) +
    72 L k on the whole S, the algorithm's figure whatever layout solves it
    (the roofline's `achieved`).  small: the fit's info["small_block"] when S
    was built and solved in the split form -- the build writes the big
    block's CSR and the dense cross block (first x 16 doubles); that layout's
    own iteration reads them once and writes and reads back the big rows'
    products with the small levels (16 first m), fewer bytes than the whole
    S's (reported beside, as "pcg_kernel_split")."""
    N, D, L = rows.n_rows, rows.codes.shape[1], int(sum(rows.n_levels))
    M, G = counts["n_ident_cells"], counts["n_ident_groups"]
    w = 0 if rows.w is None else 8
    p1 = N * (4 + 4 * D + 8 * m + w) + M * (4 * D + 8) + G * 16 + L * 8 * (3 + m)
    sb = M * (4 * D + 8) + G * 16 + S.nnz * 12 + (L + 1) * 8
    per_it = 12 * S.nnz + 4 * (L + 1) + 8 * L * m * 9
    out = {"pass1": p1, "sbuild": sb, "pcg_kernel": per_it * max(iterations, 1)}
    if small:
        out["sbuild"] = (M * (4 * D + 8) + G * 16 + small["big_nnz"] * 12 + (L + 1) * 8
                         + 8 * 16 * small["first"])
        out["pcg_kernel_split"] = (12 * small["big_nnz"] + 8 * (L + 1) + 8 * 16 * small["first"]
                                   + 8 * L * m * 9 + 16 * small["first"] * m) * max(iterations, 1)
    return out


# DRAM bytes (read + write) of one PCG iteration on the 5M-worker panel, from
# an ncu capture of pcg_kernel<3, 4> (the split form of S) in this bench's
# own command: 3.22 GB over 19 iterations and the set-up
PCG_DRAM_BYTES_PER_ITER = (3140617472 + 80062976) / 19


def measured_peak():
    try:
        d = json.loads(PEAKS.read_text())
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


# ------------------------------------------------------------- our arm

def run_ours(args, rank, world, local_rank):
    import torch
    from hdfe_stream_b200 import _lib, fit, replicas
    from hdfe_stream_b200.simulate import prepare

    torch.cuda.set_device(local_rank)
    dist = replicas.init(world, "nccl", device=torch.device("cuda", local_rank))
    rows = prepare(args.workload, seed=replicas.rank_seed(rank))
    drows = fit.DeviceRows.from_rows(rows)
    torch.cuda.synchronize()
    sampler = ClockSampler(local_rank)
    sampler.start()                 # before the warm-up: its start-up is not timed
    for _ in range(max(args.warmup, 0)):
        res = fit.fit(drows, tol=args.tol)
    torch.cuda.synchronize()
    lib = _lib.lib()
    timer = fit.PhaseTimer()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    launches0 = lib.hdfe_kernel_launches()
    t0 = torch.cuda.Event(enable_timing=True)
    t1 = torch.cuda.Event(enable_timing=True)
    h0 = sampler.mark()
    t0.record()
    for _ in range(args.steps):
        res = fit.fit(drows, tol=args.tol, timer=timer)
    t1.record()
    torch.cuda.synchronize()
    h1 = sampler.mark()
    if dist:
        dist.barrier()
    launches = lib.hdfe_kernel_launches() - launches0
    clocks = sampler.stop(h0, h1)
    ms = replicas.max_over_ranks(t0.elapsed_time(t1), dist, "cuda")
    phases = timer.totals()
    info = res.info
    its = int(np.max(np.atleast_1d(info["iterations"])))

    # accuracy: FP64 and the mixed-precision solve (FP32 inner CG, FP64
    # refinement) compared at equal error -- for each, the loosest residual
    # tolerance whose fixed effects are within 1e-8 (relative, max norm) of an
    # FP64 solve at 1e-13, and the solve's time at that tolerance (components,
    # PCG, normalisation on the same cells and S)
    parts = set(("accuracy,kss,adjoint,batched,e2e,streamed" if args.parts == "all"
                 else args.parts).split(","))
    accuracy = equal_error_solves(res.cells, res.S, max(args.steps, 3)) \
        if "accuracy" in parts else None
    # KSS-JLA: p = 256 Rademacher probes through A S^- A' on the 1M-worker panel
    jla = run_jla(args, rank, world, dist) if args.jla and "kss" in parts else None
    adjoint = run_adjoint(args, rank) if args.jla and "adjoint" in parts else None
    batched = run_batched(args, rank) if args.jla and "batched" in parts else None

    # e2e through the public call: pinned host rows up, fixed effects back
    e2e = run_e2e(args, rows, dist) if "e2e" in parts else None
    # the same fit with the rows streamed through the device in 4M-row batches
    streamed = run_streamed(args, rows, res.gamma, dist) \
        if args.jla and "streamed" in parts else None

    out = None
    if rank == 0:
        value = replicas.job_rate(args.steps, ms, world)
        by = phase_bytes(rows, res.cells.counts, res.S, its, small=info.get("small_block"))
        peak, peak_kind = measured_peak()
        roof = {}
        for name in ("pass1", "sbuild", "pcg_kernel"):
            tot, cnt = phases.get(name, (0.0, 0))
            if cnt:
                avg_ms = tot / cnt
                gbs = by[name] / (avg_ms / 1e3) / 1e9
                roof[name] = {"ms": round(avg_ms, 4), "bytes": int(by[name]),
                              "achieved_gbs": round(gbs, 1), "frac": round(gbs / peak, 4)}
                if name == "pcg_kernel" and "pcg_kernel_split" in by:
                    # the split form's own (smaller) bytes for the same iterations
                    sg = by["pcg_kernel_split"] / (avg_ms / 1e3) / 1e9
                    roof[name]["split_form_bytes"] = int(by["pcg_kernel_split"])
                    roof[name]["split_form_gbs"] = round(sg, 1)
                    roof[name]["split_form_frac"] = round(sg / peak, 4)
        # the dominant single kernel is the PCG (one launch per fit); the S
        # build and pass 1 are phases of several kernels, reported alongside
        dom = "pcg_kernel"
        traffic = None
        if args.workload == WORKLOAD:
            traffic = int(PCG_DRAM_BYTES_PER_ITER * its)
        out = {
            "metric": METRIC, "value": round(value, 4), "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms / args.steps, 3),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded generator, 5M-worker AKM panel per rank)",
            "config": config(args, world, rows),
            "roofline": {"bound": "hbm", "kernel": dom, "achieved": roof[dom]["achieved_gbs"],
                         "peak": peak, "unit": "GB/s",
                         "frac": roof[dom]["frac"], "traffic": traffic,
                         "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum of "
                                           "one pcg_kernel launch on this panel, per iteration "
                                           "x this run's iterations",
                         "peak_source": f"{peak_kind} hbm_gbs", "phases": roof},
            "e2e": e2e, "gpu_launches": int(launches), "clocks": clocks,
            "equal_error_1e-8": accuracy, "kss_jla": jla, "adjoint": adjoint,
            "batched": batched, "streamed_4m_batches": streamed,
            "solve": {"iterations": info["iterations"], "converged": info["converged"],
                      "max_rel_residual": info["max_rel_residual"], "S_nnz": info["S_nnz"],
                      "n_components": info["n_components"]},
        }
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return out, rows


TOL_LADDER = (1e-7, 3e-8, 1e-8, 3e-9, 1e-9, 3e-10, 1e-10, 3e-11, 1e-11, 3e-12, 1e-12)


def equal_error_solves(cells, S, reps, target=1e-8):
    """For FP64 and mixed precision: the loosest tolerance of TOL_LADDER
    whose fixed effects are within `target` of an FP64 solve at 1e-13, with
    its iterations and its solve time (CUDA events, `reps` solves)."""
    import torch
    from hdfe_stream_b200 import fit
    ref = fit.solve(cells, S, tol=1e-13)
    scale = float(ref.gamma.abs().max())
    out = {"target_rel_fe_err": target, "oracle": "FP64 PCG at 1e-13", "norm": "max |dFE| / max |FE|"}
    for prec in ("fp64", "mixed"):
        chosen = None
        for tol in TOL_LADDER:
            r = fit.solve(cells, S, tol=tol, precision=prec)
            err = float((r.gamma - ref.gamma).abs().max()) / scale
            if err <= target:
                chosen = (tol, err, r)
                break
        if chosen is None:
            out[prec] = {"reached": False}
            continue
        tol, err, r = chosen
        fit.solve(cells, S, tol=tol, precision=prec)
        torch.cuda.synchronize()
        a0, a1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a0.record()
        for _ in range(reps):
            fit.solve(cells, S, tol=tol, precision=prec)
        a1.record()
        torch.cuda.synchronize()
        out[prec] = {"tol": tol, "rel_fe_err": err, "iterations": r.info["iterations"],
                     "solve_ms": round(a0.elapsed_time(a1) / reps, 3)}
    if out["fp64"].get("solve_ms") and out["mixed"].get("solve_ms"):
        out["mixed_speedup"] = round(out["fp64"]["solve_ms"] / out["mixed"]["solve_ms"], 3)
    return out


def run_jla(args, rank, world, dist):
    """KSS `leave_out_components` on the 1M-worker panel with the model's
    covariates, from the device fit's Gamma: beta and the residuals (steps
    3-4), JLA leverages for p = 256 probes, sigma2, and the Hutchinson bias
    term for 256 draws (two applications of the inverse per draw), blocks of
    32.  RHS solves per second = p (1 + 2) / device time of the whole call."""
    import torch
    from hdfe_stream_b200 import fit, leaveout, replicas, shard
    from hdfe_stream_b200.simulate import prepare

    # under torchrun the ranks share ONE job: the same panel, the probes and
    # draws split over the ranks (one all-reduce of the moment sums each)
    rows = prepare(args.kss_workload, seed=100)
    drows = fit.DeviceRows.from_rows(rows)
    res = fit.fit(drows, tol=args.tol)
    S = res.S
    X = drows.V[1:].T.contiguous()
    op = leaveout.InverseOperator(drows, res.cells, S, X, tol=args.tol)
    p = 256
    split = shard.DrawSplit(rank, world, None) if dist else None

    def kss_call(operator, timer=None):
        if split is None:
            return operator.leave_out_components(res, p, block=32, seed=1, timer=timer)
        return shard.leave_out_components(operator, res, p, block=32, seed=1, timer=timer,
                                          split=split)
    op.leave_out_components(res, 32, block=32, seed=1)   # warm-up (border, null space)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    timer = fit.PhaseTimer()
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
    ev[0].record()
    kss = kss_call(op, timer)
    ev[1].record()
    torch.cuda.synchronize()
    phases = {k: v[0] for k, v in timer.totals().items()}
    ms = ev[0].elapsed_time(ev[1])
    # the kernels one by one: the same call again with an event pair around
    # every launch (kept apart from the timed call above, whose events are
    # per phase only)
    ktimer = fit.PhaseTimer()
    op.timer = ktimer
    it0 = dict(op.solver.stats)
    kss_call(op)
    op.timer = None
    op.solver.timer = None
    kern = {k: v for k, v in ktimer.totals().items()}
    pcg_its = op.solver.stats["iterations"] - it0["iterations"]
    roofline = kss_roofline(rows, S, kern, pcg_its, c=X.shape[1], B=32)
    # the same call with the block solves in mixed precision (FP32 inner CG on
    # 32 columns, FP64 refinement to the same residual tolerance)
    op_m = leaveout.InverseOperator(drows, res.cells, S, X, tol=args.tol, precision="mixed")
    kss_call(op_m)
    torch.cuda.synchronize()
    evm = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
    evm[0].record()
    kss_m = kss_call(op_m)
    evm[1].record()
    torch.cuda.synchronize()
    ms_m = replicas.max_over_ranks(evm[0].elapsed_time(evm[1]), dist, "cuda")
    comp = np.array([*kss.leave_out.values()])
    comp_m = np.array([*kss_m.leave_out.values()])
    mixed_block = {"ms": round(ms_m, 3), "value": round(3 * p / (ms_m / 1e3), 2),
                   "unit": "RHS solves/s", "speedup_vs_fp64": round(ms / ms_m, 3),
                   "max_rel_diff_leave_out": float(np.max(np.abs(comp_m - comp) / np.abs(comp)))}
    block_cmp = equal_error_block(op, S, res.cells, max(args.steps, 3))
    ms_jla, ms_tr = phases["leverages"], phases["trace"]
    if dist:
        t = torch.tensor([ms, ms_jla, ms_tr], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms, ms_jla, ms_tr = (float(x) for x in t.tolist())
    sigma2 = kss.diagnostics["sigma2"]
    bad = int((~torch.isfinite(sigma2)).sum().item())
    # KSS standard errors (leaveout_se.py `component_variances`): B_ii by p
    # draws, C y, and the trace term by p draws
    from hdfe_stream_b200.leaveout_se import StandardErrors
    se_op = StandardErrors(op)
    se_ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
    se_ev[0].record()
    lev = kss.leverages
    ses = se_op.component_variances(sigma2, lev.leverage, lev.complement, lev.factor,
                                    None, n_draws=p, block=8, seed=1)
    se_ev[1].record()
    torch.cuda.synchronize()
    ms_se = se_ev[0].elapsed_time(se_ev[1])

    def finite(x):
        return [float(v) if np.isfinite(v) else None for v in x]
    out = {"workload": describe(args.kss_workload) + "; log_earn ~ age_squared + age_cubed | "
                       "worker_id + firm_id",
           "rows": rows.n_rows, "levels": int(sum(rows.n_levels)), "S_nnz": S.nnz, "draws": p,
           "block": 32, "ms": round(ms, 3), "ms_leverages": round(ms_jla, 3),
           "ms_trace": round(ms_tr, 3), "ms_steps34": round(phases["steps34"], 3),
           "ms_sigma2": round(phases["sigma2"], 3),
           "value": round(3 * p / (ms / 1e3), 2), "unit": "RHS solves/s",
           "note": "p (1 + 2 Hutchinson) RHS solves: the leverages' one application of "
                   "the inverse per probe and the bias term's two per draw; the timed call "
                   "is the whole leave_out_components (steps 3-4, leverages, sigma2, trace)",
           "max_leverage": kss.diagnostics["max_leverage"],
           "plug_in": finite(kss.plug_in.values()), "bias_terms": finite(kss.bias.values()),
           "leave_out": finite(kss.leave_out.values()),
           "rows_without_sigma2": bad,
           "standard_errors": {"se": dict(zip(ses["se"], finite(ses["se"].values()))),
                               "se_conservative": dict(zip(ses["se_conservative"], finite(
                                   ses["se_conservative"].values()))),
                               "ms": round(ms_se, 3), "draws": p,
                               "rhs_solves": 2 * p + 7 + 9 * p,
                               "note": "B_ii: 2 solves per draw; C y: 7; trace term: 9 "
                                       "per draw (6 then 3)"},
           "iterations_last_block": op.jla_info["iterations"], "roofline": roofline,
           "mixed": mixed_block, "equal_error_1e-8_block": block_cmp,
           "scaling": "strong (one job: probes and draws split over the ranks)" if dist
                      else "single"}
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        sys.path.insert(0, str(REPO / "oracle"))
        import oracle as orc
        orc.set_threads(os.cpu_count() or 1)
        c = orc.pass1(rows)
        des = orc.Design(rows, c, orc.build_explicit(c), X=rows.V[:, 1:], tol=args.tol)
        des.border()
        des.null_space()
        t0 = time.perf_counter()
        des.jla_leverages(32, 32, 1)
        t1 = time.perf_counter()
        des.hutchinson_trace(np.nan_to_num(sigma2.cpu().numpy()), 32, 32, 2)
        t2 = time.perf_counter()
        out["cpu_baseline"] = {"value": round(3 * 32 / (t2 - t0), 3), "unit": "RHS solves/s",
                               "cores": orc.num_threads(), "kind": "port",
                               "sample": "one block of 32 probes and one of 32 Hutchinson draws "
                                         "on the same panel"}
    return out


def equal_error_block(op, S, cells, reps, target=1e-8):
    """One JLA block of 32 probes (the KSS path's solve): for FP64 and for
    mixed precision, the loosest tolerance of TOL_LADDER whose projected rows
    A S^- A' r are within `target` (relative, max norm) of an FP64 solve at
    1e-13, and the block solve's time at that tolerance (CUDA events), with
    its roofline: per iteration 12 nnz + 8 (L + 1) + 72 L k bytes in FP64,
    8 nnz + 4 (L + 1) + 36 L k in the FP32 inner iterations."""
    import torch
    from hdfe_stream_b200 import fit
    from hdfe_stream_b200.gpu import BlockSolver
    dinv = fit.jacobi(cells.diag)
    keep = op.solver
    op.solver = BlockSolver(S, dinv, 1e-13, 5000)
    ref, _ = op.project(32, seed=1)
    rhs, _, sq = op.center(32, seed=1)
    zero = (torch.linalg.vector_norm(rhs, dim=0) <= 1e-11 * torch.sqrt(sq)).cpu().numpy()
    scale = float(ref.abs().max())
    peak, _ = measured_peak()
    L, k = S.L, 32
    out = {"target_rel_err": target, "quantity": "projected rows of one 32-probe block",
           "oracle": "FP64 PCG at 1e-13"}
    for prec in ("fp64", "mixed"):
        chosen = None
        for tol in TOL_LADDER:
            op.solver = BlockSolver(S, dinv, tol, 5000, precision=prec)
            got, _ = op.project(32, seed=1)
            err = float((got - ref).abs().max()) / scale
            if err <= target:
                chosen = (tol, err)
                break
        if chosen is None:
            out[prec] = {"reached": False}
            continue
        tol, err = chosen
        solver = op.solver
        solver.solve_device(rhs, zero)
        torch.cuda.synchronize()
        its0 = solver.stats["iterations"]
        a0, a1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a0.record()
        for _ in range(reps):
            solver.solve_device(rhs, zero)
        a1.record()
        torch.cuda.synchronize()
        its = (solver.stats["iterations"] - its0) / reps
        ms = a0.elapsed_time(a1) / reps
        per_it = (12 * S.nnz + 8 * (L + 1) + 72 * L * k) if prec == "fp64" else \
            (8 * S.nnz + 4 * (L + 1) + 36 * L * k)
        gbs = per_it * its / (ms / 1e3) / 1e9
        out[prec] = {"tol": tol, "rel_err": err, "iterations": its, "solve_ms": round(ms, 3),
                     "achieved_gbs": round(gbs, 1), "frac": round(gbs / peak, 4)}
    op.solver = keep
    if out["fp64"].get("solve_ms") and out["mixed"].get("solve_ms"):
        out["mixed_speedup"] = round(out["fp64"]["solve_ms"] / out["mixed"]["solve_ms"], 3)
    return out


def kss_roofline(rows, S, kern, pcg_its, c, B):
    """Per-kernel roofline of one leave_out_components call: each kernel's
    compulsory DRAM bytes (N rows, D non-streamed codes, c covariates, L
    levels, G groups, B vectors per launch; written out in the design
    notes) over its CUDA-event time, against the measured HBM peak."""
    N, D, L, G = rows.n_rows, rows.codes.shape[1], int(sum(rows.n_levels)), rows.n_groups
    w = 0 if rows.w is None else 8
    row = N * (4 * D + 8 * c + w)              # codes, covariates, weights: one read
    per_launch = {
        "k_center": row + L * B * 8,
        "k_project": row + L * B * 8 + 80 * N,            # U gathers, the 5 JLA sums r/w
        "k_reduce": row + G * B * 8 + L * B * 8,
        "k_project_coef": row + L * B * 8 + 2 * G * B * 8,
        "k_trace": N * 4 * D + 2 * (L + G) * B * 8,
    }
    peak, kind = measured_peak()
    out = {"bound": "hbm", "peak": peak, "peak_source": f"{kind} hbm_gbs", "unit": "GB/s",
           "kernels": {}}
    for name, (tot_ms, launches) in kern.items():
        if name == "pcg_kernel":
            nbytes = pcg_its * (12 * S.nnz + 8 * (L + 1) + 72 * L * B)
        elif name in per_launch:
            nbytes = launches * per_launch[name]
        else:
            continue
        gbs = nbytes / (tot_ms / 1e3) / 1e9
        out["kernels"][name] = {"launches": launches, "ms": round(tot_ms, 3),
                                "bytes": int(nbytes), "achieved_gbs": round(gbs, 1),
                                "frac": round(gbs / peak, 4)}
    if "pcg_kernel" in out["kernels"]:
        out["kernels"]["pcg_kernel"]["iterations"] = int(pcg_its)
    dom = max(out["kernels"], key=lambda k: out["kernels"][k]["ms"])
    out.update(kernel=dom, achieved=out["kernels"][dom]["achieved_gbs"],
               frac=out["kernels"][dom]["frac"])
    return out


def run_adjoint(args, rank):
    """Gradients through the fit on the weighted 400k-worker panel (3.4M
    rows, weights U[0.5, 2]): the plug-in var(psi) and the age_squared
    coefficient with respect to y and the weights; forward = the fit with
    steps 3-4, backward = one inverse application and the row scatter per
    objective."""
    import torch
    from hdfe_stream_b200.adjoint import FixedEffectsSolve, plug_in_components
    from hdfe_stream_b200.simulate import prepare

    rows = prepare("akm_400k_w", seed=300 + rank)
    dev = torch.device("cuda", torch.cuda.current_device())
    t = lambda a, dt: torch.as_tensor(np.ascontiguousarray(a), device=dev).to(dt)
    gcode, codes = t(rows.gcode.view(np.int32), torch.int32), t(rows.codes.view(np.int32),
                                                                  torch.int32)
    X = t(rows.V[:, 1:], torch.float64)

    def once():
        y = t(rows.V[:, 0], torch.float64).requires_grad_(True)
        w = t(rows.w, torch.float64).requires_grad_(True)
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
        ev[0].record()
        beta, gam, alpha, _ = FixedEffectsSolve.apply(y, w, gcode, codes, X, rows.n_levels,
                                                      args.tol)
        comp = plug_in_components(gam, alpha, w, gcode, codes, rows.n_levels)
        ev[1].record()
        g1 = torch.autograd.grad(comp[0], (y, w), retain_graph=True)
        g2 = torch.autograd.grad(beta[0], (y, w))
        ev[2].record()
        torch.cuda.synchronize()
        return ev[0].elapsed_time(ev[1]), ev[1].elapsed_time(ev[2]), comp, beta, g1, g2
    once()
    ms_f, ms_b, comp, beta, g1, g2 = once()
    return {"workload": "akm_400k_w: 400k workers, 40k firms, 10 years, weights U[0.5, 2]",
            "rows": rows.n_rows, "ms_forward": round(ms_f, 3), "ms_backward": round(ms_b, 3),
            "objectives": ["plug-in var(psi)", "age_squared coefficient"],
            "values": [float(comp[0].detach()), float(beta[0].detach())],
            "grad_norms": [float(torch.linalg.vector_norm(g).item()) for g in (*g1, *g2)],
            "note": "backward: two objectives x (one inverse application + row scatter); "
                    "gradients checked against dense autograd and finite differences in "
                    "tests/test_gpu_adjoint.py"}


def run_batched(args, rank):
    """64 independent AKM regressions (the 20k-worker panel's generator:
    workers log-uniform on 5,000-400,000, firms = workers / 10, 10 years,
    8 consecutive years each, move probability 0.1, largest connected set):
    all fitted by one pass 1, one S build and one batched PCG launch, against
    64 sequential single fits; rows resident on the device for both."""
    import torch
    from hdfe_stream_b200 import batch, fit
    from hdfe_stream_b200.simulate import pass0_layout, restrict_connected, simulate_panel

    rng = np.random.default_rng(500 + rank)
    sizes = np.exp(rng.uniform(np.log(5_000), np.log(400_000), 64)).astype(np.int64)
    systems = []
    for i, n in enumerate(sizes):
        p = simulate_panel(int(n), int(n) // 10, 10, spell=(8, 8), p_move=0.1,
                           seed=1_000 + 64 * rank + i)
        systems.append(pass0_layout(p, restrict_connected(p, (1, 1))))
    b = batch.concat(systems)
    drows = fit.DeviceRows.from_rows(b.rows)
    singles = [fit.DeviceRows.from_rows(r) for r in systems]

    def batched_fit():
        solver = batch.BatchSolver(b, tol=args.tol, drows=drows, lanes=lanes)
        solver.shape = dict(shape)
        X, info = solver.solve()
        return solver, solver.gammas(solver.normalize(X)), info
    tuner = batch.BatchSolver(b, tol=args.tol, drows=drows)
    lanes = tuner.tune()
    shape = dict(tuner.shape)
    del tuner
    batched_fit()                                   # warm-up
    torch.cuda.synchronize()
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
    ev[0].record()
    solver, gammas, info = batched_fit()
    ev[1].record()
    torch.cuda.synchronize()
    for r in singles:                               # warm-up (allocator, occupancy)
        fit.fit(r, tol=args.tol)
    torch.cuda.synchronize()
    ev[2].record()
    ref = [fit.fit(r, tol=args.tol).gamma for r in singles]
    ev[3].record()
    torch.cuda.synchronize()
    ms_b, ms_s = ev[0].elapsed_time(ev[1]), ev[2].elapsed_time(ev[3])
    diff = max(float((g - h).abs().max() / h.abs().max()) for g, h in zip(gammas, ref))
    return {"workload": "64 AKM regressions, workers log-uniform 5k-400k, firms = workers/10, "
                        "10 years, 8-year spells, largest connected sets",
            "rows": b.rows.n_rows, "workers": int(sizes.sum()), "systems": 64,
            "ms_batched": round(ms_b, 3), "ms_sequential": round(ms_s, 3),
            "fits_per_s_batched": round(64 / (ms_b / 1e3), 2),
            "fits_per_s_sequential": round(64 / (ms_s / 1e3), 2),
            "launch_shape": {"lanes_per_row": lanes, **shape},
            "max_iterations": int(info["iterations"].max()),
            "all_converged": bool(info["converged"].all()), "tol": args.tol,
            "max_rel_diff_vs_sequential": diff,
            "note": "FP64 batched PCG (per-system scalars, one cooperative launch); the "
                    "batched time includes pass 1, the S build, the renumbering and the "
                    "normalisation; the sequential arm is 64 plain FP64 device fits"}


def run_e2e(args, rows, dist):
    """Same metric through the public host-input call with pinned host
    buffers: every step copies its rows host->device and its fixed effects
    back, inside the timed region.  A stream of fits runs as a pipeline
    (`fit.upload_host` for step i+1 is issued before `fit.fit_uploaded` of
    step i, so the next rows cross the bus while this fit computes, into
    the device buffers of step i - 1; within a step the structure goes first
    and the outcome's chunks are passed through pass 1 as they land);
    `serial` is the same with one `fit.fit_host` at a time."""
    import torch
    from hdfe_stream_b200 import fit, replicas

    pinned = {
        "gcode": torch.from_numpy(rows.gcode.view(np.int32)).pin_memory(),
        "codes": torch.from_numpy(np.ascontiguousarray(rows.codes).view(np.int32)).pin_memory(),
        "V": torch.from_numpy(np.ascontiguousarray(rows.V.T)).pin_memory(),
    }
    if rows.w is not None:
        pinned["w"] = torch.from_numpy(np.ascontiguousarray(rows.w, dtype=np.float64)).pin_memory()
    h2d = sum(t.numel() * t.element_size() for t in pinned.values())
    out_host = None
    d2h = 0

    def upload(reuse=None):
        return fit.upload_host(pinned["gcode"], pinned["codes"], pinned["V"], w=pinned.get("w"),
                               reuse=reuse)

    def finish(res):
        nonlocal out_host, d2h
        if out_host is None:
            out_host = torch.empty(res.gamma.shape, dtype=res.gamma.dtype, pin_memory=True)
        out_host.copy_(res.gamma, non_blocking=True)
        d2h = res.gamma.numel() * res.gamma.element_size()

    def timed(run):
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record()
        # the uploads (on the copy stream) start after the timed region does
        fit._copy_stream(torch.device("cuda", torch.cuda.current_device())).wait_stream(
            torch.cuda.current_stream())
        run()
        b.record()
        torch.cuda.synchronize()
        return replicas.max_over_ranks(a.elapsed_time(b), dist, "cuda")

    def pipeline():
        # two sets of device buffers in turn: step i + 1's rows go into the
        # buffers of step i - 1, whose fit has returned
        up, prev = upload(), None
        for i in range(args.steps):
            nxt = upload(reuse=prev) if i + 1 < args.steps else None
            finish(fit.fit_uploaded(up, rows.n_levels, tol=args.tol))
            prev, up = up, nxt

    def serial():
        for _ in range(args.steps):
            finish(fit.fit_host(pinned["gcode"], pinned["codes"], pinned["V"], rows.n_levels,
                                w=pinned.get("w"), tol=args.tol))

    finish(fit.fit_host(pinned["gcode"], pinned["codes"], pinned["V"], rows.n_levels,
                        w=pinned.get("w"), tol=args.tol))                 # warm-up
    ms = timed(pipeline)
    ms_serial = timed(serial)
    world = dist.get_world_size() if dist else 1
    return {"value": round(replicas.job_rate(args.steps, ms, world), 4), "unit": UNIT,
            "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h),
            "serial": {"value": round(replicas.job_rate(args.steps, ms_serial, world), 4),
                       "note": "one fit_host at a time: the next upload starts after this "
                               "fit's solve"}}


def run_streamed(args, rows, gamma_resident, dist):
    """The fit with the rows streamed through the device in batches of 4M
    rows (`fit.fit_stream`: pinned host batches, each uploaded on a copy
    stream while pass 1 runs on the one before), timed per step with the
    copies inside, against the resident one-pass fit's fixed effects."""
    import torch
    from hdfe_stream_b200 import fit, replicas
    batches = fit.group_batches(rows, fit.BATCH_ROWS)
    h2d = sum(t.numel() * t.element_size() for b in batches for t in b if t is not None)
    res = fit.fit_stream(batches, rows.n_levels, tol=args.tol, names=rows.names)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    a = torch.cuda.Event(enable_timing=True)
    b = torch.cuda.Event(enable_timing=True)
    a.record()
    for _ in range(args.steps):
        res = fit.fit_stream(batches, rows.n_levels, tol=args.tol, names=rows.names)
    b.record()
    torch.cuda.synchronize()
    ms = replicas.max_over_ranks(a.elapsed_time(b), dist, "cuda")
    world = dist.get_world_size() if dist else 1
    diff = float((res.gamma - gamma_resident).abs().max() / gamma_resident.abs().max())
    return {"batches": len(batches), "batch_rows": fit.BATCH_ROWS,
            "ms_per_fit": round(ms / args.steps, 3),
            "value": round(replicas.job_rate(args.steps, ms, world), 4), "unit": UNIT,
            "h2d_bytes_per_step": int(h2d), "max_rel_diff_vs_resident": diff,
            "note": "host batches -> device (copy stream, one ahead) -> pass 1 per batch; "
                    "the S build and the PCG on the appended cells"}


# ------------------------------------------------------- the CPU baseline

def oracle_fit(rows, tol):
    sys.path.insert(0, str(REPO / "oracle"))
    import oracle as orc
    cells = orc.pass1(rows)
    S = orc.build_explicit(cells)
    gamma, info = orc.solve(cells, S, tol=tol)
    return gamma, info


def cpu_baseline(rows, tol, steps=1):
    sys.path.insert(0, str(REPO / "oracle"))
    import oracle as orc
    orc.set_threads(os.cpu_count() or 1)
    t = time.perf_counter()
    for _ in range(steps):
        oracle_fit(rows, tol)
    dt = time.perf_counter() - t
    return {"value": round(steps / dt, 5), "unit": UNIT, "cores": orc.num_threads(),
            "kind": "port", "seconds_per_fit": round(dt / steps, 3),
            "sample": f"{steps} full fit(s) of the same panel on the host cores (the oracle: "
                      "the reference's numba kernels restated in C, OpenMP over all threads)"}


def run_reference(args, rank):
    if rank != 0:
        return None
    from hdfe_stream_b200.simulate import prepare
    sys.path.insert(0, str(REPO / "oracle"))
    import oracle as orc
    orc.set_threads(os.cpu_count() or 1)
    rows = prepare(args.workload, seed=0)
    # a bounded sample of the workload: one full CPU fit takes seconds, so at
    # most one warm-up fit and three timed fits, whatever --steps asks
    warm, steps = min(max(args.warmup, 0), 1), max(1, min(args.steps, 3))
    for _ in range(warm):
        oracle_fit(rows, args.tol)
    t = time.perf_counter()
    for _ in range(steps):
        _, info = oracle_fit(rows, args.tol)
    dt = time.perf_counter() - t
    value = steps / dt
    return {"metric": METRIC, "value": round(value, 5), "unit": UNIT, "impl": "reference",
            "n_gpus": args.gpus, "steps": steps, "warmup": warm,
            "ms_per_step": round(dt / steps * 1e3, 1), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded generator, 5M-worker AKM panel)",
            "config": config(args, 1, rows),
            "cpu_baseline": {"value": round(value, 5), "unit": UNIT, "cores": orc.num_threads(),
                             "kind": "port",
                             "sample": f"{steps} full fits of the panel (each step one fit), "
                                       f"after {warm} warm-up fit"},
            "e2e": {"value": round(value, 5), "unit": UNIT, "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0},
            "solve": {"iterations": info["iterations"], "converged": info["converged"]}}


def main():
    args = parse()
    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", 1))
    local_rank = int(os.environ.get("LOCAL_RANK", 0))
    if args.impl == "reference":
        out = run_reference(args, rank)
        if out is not None:
            print(json.dumps(out), flush=True)
        return
    out, rows = run_ours(args, rank, world, local_rank)
    if rank == 0 and out is not None:
        if world == 1 and not args.no_cpu_baseline:
            out["cpu_baseline"] = cpu_baseline(rows, args.tol)
        print(json.dumps(out), flush=True)


if __name__ == "__main__":
    main()

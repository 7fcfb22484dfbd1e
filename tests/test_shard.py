"""One KSS job split over ranks (hdfe_stream_b200.shard) on the CPU: two gloo
ranks share the JLA probes and the Hutchinson draws of the same design and
sum their moments with one all-reduce each.  The per-rank block sums come
from the oracle here (the device kernels need a GPU); what is tested is the
split itself -- the draw ranges, the reduction, and that the union of the
ranks' draws gives the single-rank answer and the reference's own numbers
(tests/golden, made by the reference's `jla_leverages` / `hutchinson_trace`)."""

import json
import os
import socket
import sys
from pathlib import Path

import numpy as np
import pytest
import torch
import torch.multiprocessing as mp

REPO = Path(__file__).resolve().parents[1]
TESTS = Path(__file__).resolve().parent


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def host_operator(rows):
    """An InverseOperator whose per-block sums are the oracle's (CPU)."""
    import oracle as orc
    from hdfe_stream_b200 import leaveout

    class HostOperator(leaveout.InverseOperator):
        def __init__(self, rows):               # no device state: the oracle does the work
            c = orc.pass1(rows)
            self.des = orc.Design(rows, c, orc.build_explicit(c), tol=1e-12)
            self.N, self.c, self.dev = rows.n_rows, 0, torch.device("cpu")
            self.w = None if rows.w is None else torch.as_tensor(rows.w)
            self.o_fe = [f"fe{d + 1}" for d in range(len(rows.n_levels))]
            self.g_fe = "fe0"

        def jla_moments(self, first, last, block=None, seed=0, moments=None):
            moments = torch.zeros((5, self.N), dtype=torch.float64) if moments is None \
                else moments
            drawn, blocks = int(first), 0
            while drawn < last:
                size = min(block, last - drawn)
                proj = self.des.project_rows(size, seed, drawn, sqrt_weights=self.w is not None)
                r = orc.rademacher(0, self.N, size, seed, drawn)
                P, M = proj ** 2, (r - proj) ** 2
                moments += torch.as_tensor(np.stack([P.sum(1), M.sum(1), (P * P).sum(1),
                                                     (M * M).sum(1), (P * M).sum(1)]))
                drawn += size
                blocks += 1
            return moments, blocks, {"iterations": None}

        def combine_moments(self, moments, n_draws):
            P, M, mPP, mMM, mPM = (m.numpy() / n_draws for m in moments)
            tot = P + M
            Pb = np.divide(P, tot, out=np.zeros_like(P), where=tot > 0)
            Mb = 1.0 - Pb
            V = (Mb ** 2 * mPP + Pb ** 2 * mMM - 2 * Pb * Mb * mPM) / n_draws
            B = (Mb * mPP - Pb * mMM + (Mb - Pb) * mPM) / n_draws
            ok = Mb > 0
            f = np.where(ok, 1.0 - np.divide(V, Mb ** 2, out=np.zeros_like(V), where=ok)
                         + np.divide(B, Mb, out=np.zeros_like(B), where=ok), 1.0)
            moments[0], moments[1], moments[2] = (torch.as_tensor(x) for x in (Pb, Mb, f))
            return moments

        def trace_totals(self, sigma2, first, last, block=None, seed=0, psi=None):
            des, col = self.des, self._psi_column(psi)
            L, G = des.cells.L, len(des.starts) - 1
            totals = np.zeros(8)
            drawn, blocks = int(first), 0
            while drawn < last:
                size = min(block, last - drawn)
                Z = orc.rademacher(0, L + G, size, seed, drawn)
                Zl, Zg = Z[:L], Z[L:]
                *_, (vl, vx, vg) = des.apply_inverse(Zl, np.zeros((0, size)), Zg,
                                                     row_weights=np.asarray(sigma2))
                Ul, _, Ug, _ = des.apply_inverse(vl, vx, vg)
                totals += orc.trace_moments(des.starts, des.codes, col,
                                            int(des.cells.offs[col]), des.w, Zl, Zg, Ul,
                                            Ug).sum(axis=(0, 1))
                drawn += size
                blocks += 1
            return torch.as_tensor(totals), blocks

    return HostOperator(rows)


def _rank(rank, world, port, out):
    for p in (str(REPO), str(REPO / "oracle"), str(TESTS)):
        sys.path.insert(0, p)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world))
    from conftest import golden_rows, load_golden
    from hdfe_stream_b200 import replicas, shard
    dist = replicas.init(world, backend="gloo", timeout_s=60)
    g = load_golden("akm_small")
    op = host_operator(golden_rows(g))
    split = shard.DrawSplit.current()
    lev = shard.jla_leverages(op, 24, block=5, seed=2, split=split)
    tr = shard.hutchinson_trace(op, g["trace_sigma2"], 16, block=3, seed=4, split=split)
    np.savez(Path(out, f"rank{rank}.npz"), leverage=lev.leverage.numpy(),
             factor=lev.factor.numpy(), trace=tr.as_array(),
             draws=np.array([*lev.diagnostics["draws"], *tr.diagnostics["draws"]]))
    dist.barrier()
    dist.destroy_process_group()


def test_draw_ranges_partition():
    from hdfe_stream_b200.shard import draw_range
    for n in (1, 7, 24, 256):
        for world in (1, 2, 3, 8):
            ranges = [draw_range(n, r, world) for r in range(world)]
            assert ranges[0][0] == 0 and ranges[-1][1] == n
            assert all(a[1] == b[0] for a, b in zip(ranges, ranges[1:]))
            sizes = [hi - lo for lo, hi in ranges]
            assert max(sizes) - min(sizes) <= 1


def test_two_ranks_share_one_kss_job(tmp_path):
    from conftest import golden_rows, load_golden
    world = 2
    mp.spawn(_rank, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True)
    got = [dict(np.load(Path(tmp_path, f"rank{r}.npz"))) for r in range(world)]
    # every rank ends with the same answer, from its own half of the draws
    assert np.array_equal(got[0]["leverage"], got[1]["leverage"])
    assert np.array_equal(got[0]["trace"], got[1]["trace"])
    assert list(got[0]["draws"]) == [0, 12, 0, 8] and list(got[1]["draws"]) == [12, 24, 8, 16]
    # the single-rank job
    g = load_golden("akm_small")
    one = host_operator(golden_rows(g))
    lev1 = one.jla_leverages(24, block=5, seed=2)
    tr1 = one.hutchinson_trace(g["trace_sigma2"], 16, block=3, seed=4)

    def rel(a, b):
        a, b = np.asarray(a, float), np.asarray(b, float)
        return float(np.max(np.abs(a - b)) / np.max(np.abs(b)))
    assert rel(got[0]["leverage"], lev1.leverage.numpy()) < 1e-13
    assert rel(got[0]["factor"], lev1.factor.numpy()) < 1e-12
    assert rel(got[0]["trace"], tr1.as_array()) < 1e-12
    # and the reference's own numbers for the same draws
    assert rel(got[0]["leverage"], g["jla_leverage"]) < 1e-8
    assert rel(got[0]["factor"], g["jla_factor"]) < 1e-8
    assert rel(got[0]["trace"], g["trace"]) < 1e-8

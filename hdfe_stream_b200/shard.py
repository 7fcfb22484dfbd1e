"""One KSS job over several GPUs, one process each: the probes and draws split.

The leave-out estimator's cost is its random projections: p JLA probes
(leaveout.py:130-198, one application of A S^- A' each) and p Hutchinson
draws (:321-448, two applications of S^- each), every one an independent
block solve on the same design.  Draw j is generated from (seed, row or
coefficient position, j) alone (core/kernels_groups.py:53-76), so any rank
can produce any draw.  Each rank therefore holds a full replica of the
design (rows, cells, S; about 1.5 GB for 8.5M rows) and runs the draws
[r p / N, (r + 1) p / N); the only exchange is one all-reduce of what the
draws accumulate:

* the JLA sink's five running sums per row (5 x N doubles), summed over the
  ranks before they are combined into leverages (leaveout.py:210-282);
* the trace's eight moment sums, summed before the bias terms are formed.

Everything between (the leverages' maximum check, beta and the residuals,
sigma2) is computed identically on every rank from the reduced sums.  The
union of the ranks' draws is exactly the single-GPU job's; the results
differ from one GPU's only by the order of the cross-rank sums (last bits).
On GPUs the all-reduce is NCCL's (NVLink); the same logic runs with gloo on
the CPU for the tests.
"""

from __future__ import annotations

from dataclasses import dataclass


def draw_range(n_draws: int, rank: int, world: int):
    """(first, last): rank's share of draws 0 .. n_draws - 1, contiguous and
    within one of equal."""
    n, r, w = int(n_draws), int(rank), int(world)
    return n * r // w, n * (r + 1) // w


@dataclass
class DrawSplit:
    """This rank's place in the job and the group its sums are reduced over."""

    rank: int
    world: int
    group: object = None

    @classmethod
    def current(cls, group=None):
        import torch.distributed as dist
        return cls(dist.get_rank(group), dist.get_world_size(group), group)

    def draws(self, n_draws: int):
        return draw_range(n_draws, self.rank, self.world)

    def sum(self, t):
        """t summed over the ranks, in place."""
        if self.world > 1:
            import torch.distributed as dist
            dist.all_reduce(t, op=dist.ReduceOp.SUM, group=self.group)
        return t


def jla_leverages(op, n_draws=250, block=None, seed=0, split: DrawSplit | None = None):
    """`InverseOperator.jla_leverages` with the probes shared among the
    ranks of `split` (default: the current process group)."""
    split = split or DrawSplit.current()
    return op._jla(n_draws, block, seed, None, split.draws(n_draws), split.sum)


def hutchinson_trace(op, sigma2, n_draws=250, block=None, seed=0, psi=None,
                     person_years=None, split: DrawSplit | None = None):
    """`InverseOperator.hutchinson_trace` with the draws shared among the
    ranks of `split`."""
    split = split or DrawSplit.current()
    return op._hutchinson(sigma2, n_draws, block, seed, None, psi, person_years,
                          split.draws(n_draws), split.sum)


def leave_out_components(op, result, n_draws=250, block=None, seed=0, psi=None,
                         stayers="own", centering="weighted", timer=None,
                         split: DrawSplit | None = None):
    """`InverseOperator.leave_out_components` (point estimates) with the JLA
    probes and the Hutchinson draws shared among the ranks of `split`; every
    rank returns the same components."""
    split = split or DrawSplit.current()
    return op.leave_out_components(result, n_draws, block, seed, psi, stayers=stayers,
                                   centering=centering, timer=timer, split=split)

"""The multi-rank path on the CPU: two gloo ranks (127.0.0.1), each fitting
its own seeded panel with the oracle, then the timing collectives
`bench.py --gpus N` uses -- the max over ranks and the whole job's rate."""

import json
import os
import socket
import sys
from pathlib import Path

import numpy as np
import torch.multiprocessing as mp

REPO = Path(__file__).resolve().parents[1]


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    sys.path.insert(0, str(REPO))
    sys.path.insert(0, str(REPO / "oracle"))
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world))
    import oracle as orc
    from hdfe_stream_b200 import replicas
    from hdfe_stream_b200.simulate import pass0_layout, simulate_panel
    dist = replicas.init(world, backend="gloo", timeout_s=60)
    rows = pass0_layout(simulate_panel(400, 40, 6, spell=(6, 6), p_move=0.2,
                                       seed=replicas.rank_seed(rank, 7)))
    c = orc.pass1(rows)
    gamma, info = orc.solve(c, orc.build_explicit(c), tol=1e-10)
    dist.barrier()
    ms_local = 10.0 * (rank + 1)             # a stand-in device time per rank
    ms = replicas.max_over_ranks(ms_local, dist)
    rate = replicas.job_rate(1, ms, world)
    Path(out, f"rank{rank}.json").write_text(json.dumps(
        {"ms": ms, "rate": rate, "gamma0": float(gamma[0, 0]), "rows": rows.n_rows,
         "converged": bool(info["converged"])}))
    dist.barrier()
    dist.destroy_process_group()


def test_two_gloo_ranks(tmp_path):
    world = 2
    mp.spawn(_rank, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True)
    res = [json.loads(Path(tmp_path, f"rank{r}.json").read_text()) for r in range(world)]
    assert all(r["ms"] == 20.0 for r in res)                  # the slowest rank's
    assert all(abs(r["rate"] - world / 0.02) < 1e-9 for r in res)
    assert all(r["converged"] for r in res)
    assert res[0]["gamma0"] != res[1]["gamma0"]               # replicas fit their own panels

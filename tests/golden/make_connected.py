"""Golden vectors for the connected set (pass 0's side), made by the
reference's own kernels.

Run once, in a container where the reference tree is readable:

    python tests/golden/make_connected.py /path/to/hdfe-stream

On seeded panels it forms the distinct (worker, firm) pairs as
core/connected.py:656-687 `_DistinctPairs` does (sorted keys a * n1 + b and
their row counts), then runs the reference's core/kernels_graph.py kernels
the way `_find_components` (core/connected.py:378-493) does for
`connected="largest"`: `_nb_peel` for min_degree, `_nb_union_keys`,
`_nb_dense_labels`, `_nb_pair_rows`, and the stable ranking by rows; and
the leave-one-out connected set, core/connected.py:503-557 `_leave_one_out`
(after `_nb_peel` for min_degree (2, 2), as `_find_components` does).
Inputs and outputs go to tests/golden/connected.npz.  Nothing at test time
reads the reference.
"""

from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

REPO = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(REPO))
sys.path.insert(0, str(Path(__file__).resolve().parent))

from hdfe_stream_b200.simulate import pass0_layout, simulate_panel  # noqa: E402
from make_golden import import_reference  # noqa: E402

PANELS = {
    # many small components (few moves), pruning bites at (2, 2)
    "sparse": dict(n_workers=3_000, n_firms=900, n_years=6, spell=(1, 6), p_move=0.03, seed=21),
    # several components left after pruning
    "middle": dict(n_workers=3_000, n_firms=600, n_years=8, spell=(2, 8), p_move=0.04, seed=23),
    # one large component with a fringe
    "dense": dict(n_workers=4_000, n_firms=300, n_years=10, spell=(2, 10), p_move=0.1, seed=22),
    # one large component of small firms: single observations and many
    # articulation-point movers, removed over several rounds
    "fringe": dict(n_workers=5_000, n_firms=1_500, n_years=8, spell=(1, 8), p_move=0.15,
                   seed=24),
}


def main(root):
    mods = import_reference(root)
    kg, cn = mods["core.kernels_graph"], mods["core.connected"]
    out = {}
    for name, spec in PANELS.items():
        rows = pass0_layout(simulate_panel(**spec))
        a = rows.gcode.astype(np.uint32)
        b = rows.codes[:, 0].astype(np.uint32)
        n0, n1 = int(rows.n_groups), int(rows.n_levels[0])
        key = a.astype(np.uint64) * np.uint64(n1) + b.astype(np.uint64)
        keys, counts = np.unique(key, return_counts=True)
        counts = counts.astype(np.uint32)
        n1u = np.uint64(n1)
        out[f"{name}_a"], out[f"{name}_b"] = a, b
        out[f"{name}_n"] = np.array([n0, n1])
        for k in (1, 2):
            alive = np.ones(n0 + n1, bool)
            rounds = 0
            if k > 1:
                rounds = kg._nb_peel(keys, n1u, k, k, alive[:n0], alive[n0:])
            parent = np.arange(n0 + n1, dtype=np.int32)
            kg._nb_union_keys(parent, keys, n1u, alive[:n0], alive[n0:])
            nc = kg._nb_dense_labels(parent, alive)
            comp_rows = np.zeros(nc, np.int64)
            kg._nb_pair_rows(keys, counts, n1u, parent, comp_rows)
            order = np.argsort(-comp_rows, kind="stable")
            rank = np.empty(nc, parent.dtype)
            rank[order] = np.arange(nc, dtype=parent.dtype)
            kg._nb_relabel(parent, rank)
            out[f"{name}_k{k}_alive"] = alive
            out[f"{name}_k{k}_labels"] = parent
            out[f"{name}_k{k}_rows"] = comp_rows[order]
            out[f"{name}_k{k}_rounds"] = np.array([rounds])
            print(name, k, "components", nc, "largest rows", comp_rows[order][:3], "rounds", rounds)
            # the leave-one-out connected set, after the (k, k) core
            alive = np.ones(n0 + n1, bool)
            if k > 1:
                kg._nb_peel(keys, n1u, k, k, alive[:n0], alive[n0:])
            lo = cn._leave_one_out(keys, counts, n1u, n0, n1, alive, None)
            kept = cn._rows_alive(keys, counts, n1u, n0, alive)
            out[f"{name}_k{k}_loo_alive"] = alive
            out[f"{name}_k{k}_loo_counts"] = np.array([lo["components_before"],
                                                       lo["single_observation"], lo["cut"],
                                                       lo["rounds"], kept])
            print("  leave-one-out", lo, "rows", kept)
    np.savez_compressed(Path(__file__).resolve().parent / "connected.npz", **out)


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else "/root/reference")

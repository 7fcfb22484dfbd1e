"""The connected set on the device (pass 0's side).

`pair_components` is core/connected.py:378-493 `_find_components` for two
fixed effects (the workers and the firms) on coded rows already in HBM, in
pass 0's order (sorted by the first dimension, then the second): distinct
pairs, the min_degree core (`_nb_peel`), union-find over the pairs left,
labels ranked by rows (a stable sort, ties to the component with the smaller
first vertex, as the reference's), rows per component.  The kernels are
`hdfe_pair_components` (csrc/pairs.cu); only the ranking of the components'
sizes runs on the host.

`leave_one_out` is core/connected.py:503-557 `_leave_one_out`: the
leave-one-out connected set the KSS estimator needs (`hdfe_leave_one_out`).
"""

from __future__ import annotations

import numpy as np

from . import _lib


def pair_components(a, b, n0: int, n1: int, min_degree=(1, 1), stream=None):
    """(labels (n0 + n1) int64 device tensor -- rank of each level's
    component by rows, -1 where pruned --, rows per rank (host int64 array),
    info).  The largest connected set is labels == 0; a's levels come first,
    then b's."""
    import torch
    lib = _lib.lib()
    dev = a.device
    n = int(n0) + int(n1)
    N = int(a.shape[0])
    alive = torch.empty(n, dtype=torch.uint8, device=dev)
    labels = torch.empty(n, dtype=torch.int32, device=dev)
    rows = torch.empty(n, dtype=torch.int64, device=dev)
    counts = torch.zeros(4, dtype=torch.int64, device=dev)
    ws = torch.empty(int(lib.hdfe_pair_components_workspace_bytes(N, n0, n1)), dtype=torch.uint8,
                     device=dev)
    k0, k1 = (int(x) for x in min_degree)
    _lib.check(lib.hdfe_pair_components(a.data_ptr(), b.data_ptr(), N, int(n0), int(n1), k0, k1,
                                        alive.data_ptr(), labels.data_ptr(), rows.data_ptr(),
                                        counts.data_ptr(), ws.data_ptr(), ws.numel(),
                                        _lib.stream_handle(stream)))
    n_pairs, nc, status, rounds = (int(x) for x in counts.cpu())
    if status != _lib.HDFE_OK:
        why = {_lib.HDFE_ERR_ARG: "rows are not sorted by the first dimension, then the second",
               _lib.HDFE_ERR_BAD_CODE: "a code is out of range"}
        raise _lib.HDFEError(status, "pair_components: " + why.get(status, "device error"))
    comp_rows = rows[:nc].cpu().numpy()
    order = np.argsort(-comp_rows, kind="stable")
    rank = np.empty(nc, np.int64)
    rank[order] = np.arange(nc)
    rank_t = torch.as_tensor(rank, device=dev)
    lab = labels.to(torch.int64)
    ranked = torch.where(lab >= 0, rank_t[lab.clamp(min=0)] if nc else lab, lab)
    info = {"distinct_pairs": n_pairs, "components": nc, "pruning_rounds": rounds}
    return ranked, comp_rows[order], info


def leave_one_out(a, b, n0: int, n1: int, min_degree=(1, 1), stream=None):
    """(alive (n0 + n1) bool device tensor, info): the levels of the
    leave-one-out connected set, a's levels first; info holds the counts of
    `_leave_one_out`'s diagnostics (components before, single observations,
    workers cut, rounds) and the rows kept."""
    import torch
    lib = _lib.lib()
    dev = a.device
    n = int(n0) + int(n1)
    N = int(a.shape[0])
    alive = torch.empty(n, dtype=torch.uint8, device=dev)
    counts = torch.zeros(8, dtype=torch.int64, device=dev)
    ws = torch.empty(int(lib.hdfe_leave_one_out_workspace_bytes(N, n0, n1)), dtype=torch.uint8,
                     device=dev)
    k0, k1 = (int(x) for x in min_degree)
    _lib.check(lib.hdfe_leave_one_out(a.data_ptr(), b.data_ptr(), N, int(n0), int(n1), k0, k1,
                                      alive.data_ptr(), counts.data_ptr(), ws.data_ptr(),
                                      ws.numel(), _lib.stream_handle(stream)))
    c = [int(x) for x in counts.cpu()]
    if c[6] != _lib.HDFE_OK:
        why = {_lib.HDFE_ERR_ARG: "rows are not sorted by the first dimension, then the second",
               _lib.HDFE_ERR_BAD_CODE: "a code is out of range",
               _lib.HDFE_ERR_SPIN_LIMIT: "a union-find walk did not end"}
        raise _lib.HDFEError(c[6], "leave_one_out: " + why.get(c[6], "device error"))
    info = {"distinct_pairs": c[0], "components_before": c[1], "single_observation": c[2],
            "cut": c[3], "rounds": c[4], "rows": c[5], "bfs_depth": c[7]}
    return alive.bool(), info

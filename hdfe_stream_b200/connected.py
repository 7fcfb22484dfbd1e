"""The connected set on the device (pass 0's side).

`pair_components` is core/connected.py:378-493 `_find_components` for two
fixed effects (the workers and the firms) on coded rows already in HBM, in
pass 0's order (sorted by the first dimension, then the second): distinct
pairs, the min_degree core (`_nb_peel`), union-find over the pairs left,
labels ranked by rows (a stable sort, ties to the component with the smaller
first vertex, as the reference's), rows per component.  The kernels are
`hdfe_pair_components` (csrc/pairs.cu); only the ranking of the components'
sizes runs on the host.
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

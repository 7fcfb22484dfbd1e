"""Pass 0 on the device: factorize the fixed-effect ids and sort the rows.

core/passes.py:285-294 codes every fixed effect by the rank of its level
among the sorted distinct levels, and :359-373 sorts the rows by the
streamed dimension's code, the other codes and then the variables (when the
fit keeps its intermediates; n_buckets = 1), the streamed code becoming the
dense group code.  Here the raw columns are already on the device: each id
column is factorized by a sorted unique (its inverse is the rank code), and
the rows are ordered by a stable sort on the packed key (streamed code,
fixed-effect codes, any further sort codes), falling back to a lexicographic
sort with the variables as the last keys when two rows share a key -- the
same order as the host reference of this layout (`simulate.pass0_layout`).
The sorts and uniques are torch's (CUB radix sorts).
"""

from __future__ import annotations

import numpy as np

from .fit import DeviceRows


def _torch():
    import torch
    return torch


def factorize(ids):
    """(codes int64, levels): the rank of each id among the sorted distinct ids."""
    torch = _torch()
    levels, codes = torch.unique(ids, sorted=True, return_inverse=True)
    return codes.to(torch.int64), levels


def pass0(streamed, fixed_effects, V, w=None, sort_only=()):
    """DeviceRows in pass 0's layout from raw device columns: `streamed` (N,)
    the streamed dimension's ids (the groups), `fixed_effects` a list of (N,)
    id columns (the codes, in order), V (N, m) float64 (outcome first), w (N,)
    or None, `sort_only` id columns that order the rows without being fixed
    effects.  Returns (rows, levels): levels per column, streamed first."""
    torch = _torch()
    g, glev = factorize(streamed)
    fe = [factorize(c) for c in fixed_effects]
    extra = [factorize(c) for c in sort_only]
    cols = [g] + [c for c, _ in fe] + [c for c, _ in extra]
    sizes = [len(glev)] + [len(l) for _, l in fe] + [len(l) for _, l in extra]
    if np.prod([float(max(n, 1)) for n in sizes]) < 2.0 ** 62:
        key = torch.zeros_like(g)
        for c, n in zip(cols, sizes):
            key = key * n + c
        order = torch.argsort(key, stable=True)
        sk = key[order]
        tie = sk.numel() > 1 and bool((sk[1:] == sk[:-1]).any())
    else:
        # the packed key would overflow int64: sort column by column instead
        # (least significant first, each sort stable) and find ties by
        # comparing every column of neighbouring rows
        order = torch.arange(g.numel(), device=g.device)
        for c in cols[::-1]:
            order = order[torch.argsort(c[order], stable=True)]
        same = torch.ones(max(g.numel() - 1, 0), dtype=torch.bool, device=g.device)
        for c in cols:
            sc = c[order]
            same &= sc[1:] == sc[:-1]
        tie = bool(same.any())
    if tie:
        # rows sharing every code: the variables break the tie (least
        # significant key sorted first, each sort stable)
        order = torch.arange(key.numel(), device=key.device)
        for k in [V[:, j] for j in reversed(range(V.shape[1]))] + cols[::-1]:
            order = order[torch.argsort(k[order], stable=True)]
    codes = torch.stack([c[order] for c, _ in fe], 1).to(torch.int32).contiguous()
    rows = DeviceRows(g[order].to(torch.int32).contiguous(), codes,
                      V[order].T.contiguous().to(torch.float64),
                      None if w is None else w[order].to(torch.float64).contiguous(),
                      [len(l) for _, l in fe])
    return rows, [glev] + [l for _, l in fe]

"""Pass 0 on the device: factorize the fixed-effect ids and sort the rows.

core/passes.py:285-294 codes every fixed effect by the rank of its level
among the sorted distinct levels, and :359-373 sorts the rows by the
streamed dimension's code, the other codes and then the variables (when the
fit keeps its intermediates; n_buckets = 1), the streamed code becoming the
dense group code.  Here the raw columns are already on the device and both
steps run on this library's own radix sort (csrc/sort.cu):

* each id column is factorized by `hdfe_factorize` (a stable radix sort of
  the ids' order-preserving unsigned keys with their positions, run heads,
  a scan of the heads, the ranks scattered back); integer ids are shifted by
  their minimum first, so only the bits their range needs are sorted;
* the codes are packed, most significant first, into one 64-bit key of
  ceil(log2(levels)) bits each (columns that do not fit go in further keys)
  and the rows ordered by a stable `hdfe_sort_pairs` of the keys with the
  row positions;
* when two rows share every code, the variables break the tie: the order
  is rebuilt least significant key first (the last variable ... the first,
  then the code keys), each pass stable -- the same order as the host
  layout of these rows (`simulate.pass0_layout`, numpy's lexsort).
"""

from __future__ import annotations

from . import _lib
from .fit import DeviceRows

SIGN = -(2 ** 63)           # the int64 with only the top bit set


def _torch():
    import torch
    return torch


def _bits(n: int) -> int:
    """Bits that codes 0 .. n - 1 need (at least one)."""
    return max((int(n) - 1).bit_length(), 1)


def order_key(t):
    """int64 tensor whose bits, read as unsigned, order like t's values:
    integers by value; floats by value with -0.0 = 0.0 and NaN last."""
    torch = _torch()
    if t.dtype.is_floating_point:
        x = t.to(torch.float64) + 0.0                      # -0.0 -> +0.0
        b = x.view(torch.int64)
        k = torch.where(b < 0, ~b, b ^ SIGN)
        return torch.where(torch.isnan(x), torch.full_like(k, -1), k)
    return t.to(torch.int64) ^ SIGN


def _from_key(k, dtype):
    torch = _torch()
    if dtype.is_floating_point:
        b = torch.where(k < 0, k ^ SIGN, ~k)
        return b.view(torch.float64).to(dtype)
    return (k ^ SIGN).to(dtype)


def _workspace(n: int, device):
    torch = _torch()
    size = int(_lib.lib().hdfe_sort_workspace_bytes(int(n)))
    return torch.empty(size, dtype=torch.uint8, device=device), size


def sort_pairs(keys, vals=None, key_bits: int = 64):
    """(sorted keys, values) of a stable ascending sort of the int64 `keys`
    read as unsigned, by their low `key_bits` bits; vals int32 (None: the
    positions 0 .. n-1)."""
    torch = _torch()
    keys = keys.contiguous()
    n = keys.numel()
    if n > 2 ** 31 - 1:
        raise ValueError("sort_pairs: at most 2^31 - 1 items")
    if vals is not None:
        vals = vals.to(torch.int32).contiguous()
        if vals.numel() != n:
            raise ValueError("sort_pairs: keys and vals differ in length")
    k_out = torch.empty_like(keys)
    v_out = torch.empty(n, dtype=torch.int32, device=keys.device)
    if n == 0:
        return k_out, v_out
    ws, size = _workspace(n, keys.device)
    _lib.check(_lib.lib().hdfe_sort_pairs(keys.data_ptr(), _lib.ptr(vals), n, int(key_bits),
                                          k_out.data_ptr(), v_out.data_ptr(), ws.data_ptr(),
                                          size, _lib.stream_handle()))
    return k_out, v_out


def factorize(ids):
    """(codes int64, levels): the rank of each id among the sorted distinct
    ids, and those ids in order (ids' dtype)."""
    torch = _torch()
    n = ids.numel()
    if n == 0:
        return torch.zeros(0, dtype=torch.int64, device=ids.device), ids.clone()
    if n > 2 ** 31 - 1:
        raise ValueError("factorize: at most 2^31 - 1 ids")
    if ids.dtype.is_floating_point:
        keys, base, bits = order_key(ids), None, 64
    else:
        x = ids.to(torch.int64)
        lo, hi = (int(v) for v in torch.aminmax(x))
        if hi - lo < 2 ** 63:
            keys, base, bits = x - lo, lo, max((hi - lo).bit_length(), 1)
        else:                                   # the range needs the sign bit
            keys, base, bits = x ^ SIGN, None, 64
    keys = keys.contiguous()
    codes = torch.empty(n, dtype=torch.int32, device=ids.device)
    levels = torch.empty(n, dtype=torch.int64, device=ids.device)
    count = torch.zeros(1, dtype=torch.int64, device=ids.device)
    ws, size = _workspace(n, ids.device)
    _lib.check(_lib.lib().hdfe_factorize(keys.data_ptr(), n, bits, codes.data_ptr(),
                                         levels.data_ptr(), count.data_ptr(), ws.data_ptr(),
                                         size, _lib.stream_handle()))
    levels = levels[:int(count.item())]
    levels = (levels + base).to(ids.dtype) if base is not None else _from_key(levels, ids.dtype)
    return codes.to(torch.int64), levels


def _packed_keys(cols, sizes):
    """[(key, bits)] most significant first: consecutive code columns packed
    into 64-bit keys, each column `_bits(size)` wide."""
    torch = _torch()
    keys, cur, used = [], None, 0
    for c, n in zip(cols, sizes):
        b, c = _bits(n), c.to(torch.int64)
        if cur is None:
            cur, used = c, b
        elif used + b > 64:
            keys.append((cur, used))
            cur, used = c, b
        else:
            cur, used = (cur << b) | c, used + b
    keys.append((cur, used))
    return keys


def _chain(keys, n, device):
    """The stable order of n rows by keys [(key, bits)], most significant
    first: one sort per key, least significant first."""
    torch = _torch()
    order = None
    for k, b in reversed(keys):
        k = k if order is None else k[order.to(torch.int64)]
        _, order = sort_pairs(k, order, b)
    return order.to(torch.int64) if order is not None else torch.arange(n, device=device)


def pass0(streamed, fixed_effects, V, w=None, sort_only=()):
    """DeviceRows in pass 0's layout from raw device columns: `streamed` (N,)
    the streamed dimension's ids (the groups), `fixed_effects` a list of (N,)
    id columns (the codes, in order), V (N, m) float64 (outcome first), w (N,)
    or None, `sort_only` id columns that order the rows without being fixed
    effects.  Returns (rows, levels): levels per column, streamed first."""
    torch = _torch()
    N = streamed.numel()
    g, glev = factorize(streamed)
    fe = [factorize(c) for c in fixed_effects]
    extra = [factorize(c) for c in sort_only]
    cols = [g] + [c for c, _ in fe] + [c for c, _ in extra]
    sizes = [len(glev)] + [len(l) for _, l in fe] + [len(l) for _, l in extra]
    code_keys = _packed_keys(cols, sizes)
    order = _chain(code_keys, N, g.device)
    # rows sharing every code: neighbours equal in every key after the sort
    same = torch.ones(max(N - 1, 0), dtype=torch.bool, device=g.device)
    for k, _ in code_keys:
        sk = k[order]
        same &= sk[1:] == sk[:-1]
    if bool(same.any()):
        var_keys = [(order_key(V[:, j]), 64) for j in range(V.shape[1])]
        order = _chain(code_keys + var_keys, N, g.device)
    codes = torch.stack([c[order] for c, _ in fe], 1).to(torch.int32).contiguous()
    rows = DeviceRows(g[order].to(torch.int32).contiguous(), codes,
                      V[order].T.contiguous().to(torch.float64),
                      None if w is None else w[order].to(torch.float64).contiguous(),
                      [len(l) for _, l in fe])
    return rows, [glev] + [l for _, l in fe]

"""X' W X of a wide design on the tensor cores (`hdfe_gram_bf16x3`).

The reference forms the design's cross-products with an FP64 BLAS product
(core/inference.py:109-137 `_assemble`).  For designs with many covariates
this product is the one GEMM-shaped piece of the path: `xtx` runs it as
split-BF16 products on the 5th-generation tensor cores (tcgen05.mma, FP32
accumulators in tensor memory per CTA, FP64 across CTAs), about 1e-5
relative per entry.  The FP64 path (`inference`, `leaveout`) stays the
default; this is for designs wide enough that the product matters.
"""

from __future__ import annotations

from . import _lib


def xtx(X, w=None):
    """X' diag(w) X for X (N, c) float64 on the device (c <= 128), w (N) or
    None: a (c, c) float64 device tensor."""
    import torch
    if X.dim() != 2 or X.dtype != torch.float64 or not X.is_cuda:
        raise ValueError("xtx: X must be an (N, c) float64 CUDA tensor")
    N, c = (int(x) for x in X.shape)
    if not 1 <= c <= _lib.GRAM_MAX_COLS:
        raise ValueError(f"xtx: 1 <= c <= {_lib.GRAM_MAX_COLS} columns")
    lib = _lib.lib()
    X = X.contiguous()
    wt = None if w is None else w.to(X.device, torch.float64).contiguous()
    out = torch.empty((c, c), dtype=torch.float64, device=X.device)
    ws = torch.zeros(int(lib.hdfe_gram_workspace_bytes(N, c)), dtype=torch.uint8, device=X.device)
    _lib.check(lib.hdfe_gram_bf16x3(X.data_ptr(), N, c, None if wt is None else wt.data_ptr(),
                                    out.data_ptr(), ws.data_ptr(), ws.numel(),
                                    _lib.stream_handle()))
    status = int(ws[:4].view(torch.int32).item())
    if status != _lib.HDFE_OK:
        raise _lib.HDFEError(status, "xtx: a wait on the tensor core timed out")
    return out

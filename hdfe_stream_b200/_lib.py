"""ctypes binding of libhdfe_b200.so (the C ABI declared in include/hdfe_b200.h).

There is no fallback: if the library is missing this raises, and every
device entry point of the package goes through it.
"""

from __future__ import annotations

import ctypes
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "libhdfe_b200.so"

HDFE_OK = 0
HDFE_ERR_ARG = 1
HDFE_ERR_CUDA = 2
HDFE_ERR_SPIN_LIMIT = 3
HDFE_ERR_WORKSPACE = 4
HDFE_ERR_BAD_CODE = 5
HDFE_ERR_CAPACITY = 6
PCG_MAX_K = 32          # HDFE_PCG_MAX_K
PCG_MIXED_MAX_K = 32    # HDFE_PCG_MIXED_MAX_K
GRAM_MAX_COLS = 128     # HDFE_GRAM_MAX_COLS
SMALL_MAX_LEVELS = 16   # HDFE_SMALL_MAX_LEVELS
PCG_SMALL_MAX_K = 4     # HDFE_PCG_SMALL_MAX_K

_c = ctypes
_vp = _c.c_void_p
_i64 = _c.c_int64
_i32 = _c.c_int32
_f64 = _c.c_double

# name -> (restype, argtypes); mirrors include/hdfe_b200.h
SIGNATURES = {
    "hdfe_error_string": (_c.c_char_p, []),
    "hdfe_version": (_c.c_char_p, []),
    "hdfe_kernel_launches": (_i64, []),
    "hdfe_pass1_workspace_bytes": (_i64, [_i64, _i32, _i32]),
    "hdfe_pass1": (_c.c_int, [_vp, _vp, _i32, _vp, _i32, _vp, _i64, _vp, _vp, _vp, _vp, _vp,
                              _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _i64,
                              _vp]),
    "hdfe_sbuild_workspace_bytes": (_i64, [_i64, _i64, _i32]),
    "hdfe_sbuild_wide_workspace_bytes": (_i64, [_i64, _i64, _i32, _i64]),
    "hdfe_sbuild_analyze": (_c.c_int, [_vp, _i64, _vp, _i32, _vp, _vp, _i64, _vp, _vp, _vp,
                                       _vp, _i64, _vp, _vp]),
    "hdfe_sbuild_count": (_c.c_int, [_vp, _i64, _vp, _i32, _vp, _vp, _i64, _vp, _vp, _vp,
                                     _i64, _i64, _vp, _vp, _i64, _vp, _i64, _vp, _i64, _vp,
                                     _vp]),
    "hdfe_sbuild_fill": (_c.c_int, [_vp, _i64, _vp, _i32, _vp, _vp, _i64, _vp, _vp, _vp, _i64,
                                    _i64, _vp, _vp, _vp, _vp, _i64, _vp, _i64, _vp, _i64, _vp,
                                    _vp]),
    "hdfe_sbuild_analyze_split": (_c.c_int, [_vp, _i64, _vp, _i32, _vp, _vp, _i64, _vp, _vp,
                                             _vp, _i64, _i32, _vp, _i64, _vp, _vp]),
    "hdfe_sbuild_count_split": (_c.c_int, [_vp, _i64, _vp, _i32, _vp, _vp, _i64, _vp, _vp, _vp,
                                           _i64, _i64, _i64, _i32, _vp, _vp, _vp, _vp, _i64,
                                           _vp, _i64, _vp, _i64, _vp, _vp]),
    "hdfe_sbuild_fill_split": (_c.c_int, [_vp, _i64, _vp, _i32, _vp, _vp, _i64, _vp, _vp, _vp,
                                          _i64, _i64, _vp, _vp, _vp, _vp, _i64, _vp, _i64, _vp,
                                          _i64, _vp, _vp]),
    "hdfe_components_workspace_bytes": (_i64, []),
    "hdfe_components": (_c.c_int, [_vp, _i64, _vp, _i32, _i32, _i64, _vp, _vp, _vp, _i64, _vp]),
    "hdfe_normalize_workspace_bytes": (_i64, [_i64, _i32]),
    "hdfe_normalize": (_c.c_int, [_vp, _i32, _i32, _vp, _vp, _vp, _vp, _i64, _vp]),
    "hdfe_row_groups_workspace_bytes": (_i64, [_i64]),
    "hdfe_row_groups": (_c.c_int, [_vp, _i64, _vp, _vp, _vp, _i64, _vp]),
    "hdfe_rows_center": (_c.c_int, [_vp, _i64, _vp, _i32, _vp, _vp, _vp, _i32, _vp, _i32,
                                    _c.c_uint64, _i64, _i64, _i32, _vp, _vp, _vp, _vp, _i64,
                                    _vp]),
    "hdfe_rows_project": (_c.c_int, [_vp, _i64, _vp, _i32, _vp, _vp, _vp, _i32, _vp, _vp, _vp,
                                     _i32, _c.c_uint64, _i64, _i64, _i32, _i64, _vp, _vp, _vp]),
    "hdfe_jla_combine": (_c.c_int, [_vp, _i64, _i64, _vp]),
    "hdfe_rows_reduce": (_c.c_int, [_vp, _i64, _vp, _i32, _vp, _vp, _vp, _i32, _vp, _vp, _i32,
                                    _vp, _vp, _vp, _vp, _vp]),
    "hdfe_rows_project_coef": (_c.c_int, [_vp, _i64, _vp, _i32, _vp, _vp, _vp, _i32, _vp, _vp,
                                          _vp, _i32, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp]),
    "hdfe_trace_moments_workspace_bytes": (_i64, [_i32]),
    "hdfe_trace_moments": (_c.c_int, [_vp, _i64, _vp, _i32, _vp, _i32, _vp, _vp, _vp, _vp,
                                      _vp, _i32, _vp, _vp, _i64, _vp, _vp]),
    "hdfe_rademacher": (_c.c_int, [_vp, _i64, _i64, _i32, _c.c_uint64, _i64, _vp]),
    "hdfe_stream_matvec": (_c.c_int, [_vp, _i64, _vp, _i32, _vp, _vp, _vp, _i32, _vp, _vp,
                                      _vp]),
    "hdfe_pair_components_workspace_bytes": (_i64, [_i64, _i64, _i64]),
    "hdfe_pair_components": (_c.c_int, [_vp, _vp, _i64, _i64, _i64, _i64, _i64, _vp, _vp, _vp,
                                        _vp, _vp, _i64, _vp]),
    "hdfe_assemble_workspace_bytes": (_i64, [_i32]),
    "hdfe_resid_moments": (_c.c_int, [_vp, _i64, _vp, _i32, _vp, _vp, _vp, _i32, _i64, _vp,
                                      _vp, _vp, _i64, _vp, _vp]),
    "hdfe_row_effects": (_c.c_int, [_vp, _i64, _vp, _i32, _vp, _i32, _vp, _vp, _i32, _i64, _vp,
                                    _vp, _vp, _vp, _vp, _vp, _i64, _vp, _vp]),
    "hdfe_kss_sigma2": (_c.c_int, [_vp, _vp, _vp, _vp, _vp, _f64, _i64, _vp, _vp]),
    "hdfe_small_split_workspace_bytes": (_i64, [_i64]),
    "hdfe_small_split": (_c.c_int, [_vp, _vp, _vp, _i64, _i64, _i32, _vp, _vp, _vp, _vp, _vp,
                                    _vp, _vp, _vp, _i64, _vp]),
    "hdfe_pcg_solve_small": (_c.c_int, [_vp, _vp, _vp, _i64, _i64, _i64, _i32, _vp, _vp, _vp,
                                        _vp, _i32, _vp, _vp, _f64, _i64, _vp, _vp, _i64, _vp,
                                        _vp]),
    "hdfe_sort_workspace_bytes": (_i64, [_i64]),
    "hdfe_sort_pairs": (_c.c_int, [_vp, _vp, _i64, _i32, _vp, _vp, _vp, _i64, _vp]),
    "hdfe_factorize": (_c.c_int, [_vp, _i64, _i32, _vp, _vp, _vp, _vp, _i64, _vp]),
    "hdfe_gram_workspace_bytes": (_i64, [_i64, _i32]),
    "hdfe_gram_bf16x3": (_c.c_int, [_vp, _i64, _i32, _vp, _vp, _vp, _i64, _vp]),
    "hdfe_solver_create": (_c.c_int, [_vp, _vp, _vp, _i64, _i64, _vp, _f64, _i64, _i32, _vp]),
    "hdfe_solver_solve": (_c.c_int, [_vp, _vp, _i32, _vp, _vp, _vp, _vp, _vp]),
    "hdfe_solver_destroy": (_c.c_int, [_vp]),
    "hdfe_row_scores": (_c.c_int, [_vp, _i64, _vp, _i32, _vp, _vp, _vp, _i32, _i64, _vp, _vp,
                                   _vp, _vp, _vp, _vp]),
    "hdfe_variance_sums_workspace_bytes": (_i64, [_i32]),
    "hdfe_variance_sums": (_c.c_int, [_vp, _i64, _vp, _i32, _vp, _vp, _vp, _i32, _i64, _vp,
                                      _vp, _vp, _vp, _i64, _vp, _vp]),
    "hdfe_leave_one_out_workspace_bytes": (_i64, [_i64, _i64, _i64]),
    "hdfe_leave_one_out": (_c.c_int, [_vp, _vp, _i64, _i64, _i64, _i64, _i64, _vp, _vp, _vp,
                                      _i64, _vp]),
    "hdfe_rows_readout": (_c.c_int, [_vp, _i64, _vp, _i32, _vp, _vp, _i32, _vp, _vp, _vp,
                                     _i32, _vp, _vp, _vp, _vp]),
    "hdfe_cov_cross": (_c.c_int, [_vp, _i64, _vp, _i32, _vp, _i32, _vp, _vp, _vp, _i32, _vp,
                                  _vp, _vp, _vp]),
    "hdfe_bii_moments": (_c.c_int, [_vp, _i32, _vp, _i64, _vp, _vp]),
    "hdfe_c_sums_workspace_bytes": (_i64, []),
    "hdfe_c_sums": (_c.c_int, [_vp, _i32, _i32, _vp, _vp, _vp, _vp, _vp, _i64, _vp, _vp, _i64,
                               _vp]),
    "hdfe_c_sums_ext": (_c.c_int, [_vp, _i32, _i32, _vp, _vp, _vp, _vp, _vp, _i32, _vp, _vp,
                                   _vp, _i64, _vp, _vp, _i64, _vp]),
    "hdfe_smooth_cells": (_c.c_int, [_vp, _vp, _vp, _i32, _vp, _vp, _vp, _i64, _vp, _vp, _vp]),
    "hdfe_smooth_eval": (_c.c_int, [_vp, _vp, _vp, _i32, _vp, _vp, _vp, _i64, _vp, _vp]),
    "hdfe_batch_pcg_grid": (_c.c_int, [_i32, _i32, _vp, _vp]),
    "hdfe_batch_pcg_workspace_bytes": (_i64, [_i64, _i32, _i64, _i64]),
    "hdfe_batch_pcg_solve": (_c.c_int, [_vp, _vp, _vp, _i64, _vp, _vp, _i32, _vp, _i64, _vp,
                                        _vp, _vp, _vp, _vp, _vp, _vp, _vp, _i64, _i32, _i32,
                                        _f64, _i64, _vp, _vp, _vp, _vp, _vp, _vp, _i64, _vp]),
    "hdfe_pcg_workspace_bytes": (_i64, [_i64, _i64, _i32]),
    "hdfe_pcg_solve": (_c.c_int, [_vp, _vp, _vp, _i64, _i64, _vp, _vp, _i32, _vp, _vp, _f64,
                                  _i64, _vp, _vp, _i64, _vp, _vp]),
    "hdfe_pcg_mixed_workspace_bytes": (_i64, [_i64, _i64, _i32]),
    "hdfe_pcg_solve_mixed": (_c.c_int, [_vp, _vp, _vp, _vp, _i64, _i64, _vp, _vp, _i32, _vp,
                                        _vp, _f64, _f64, _i64, _vp, _vp, _i64, _vp, _vp]),
    "hdfe_pcg_solve_noalloc": (_c.c_int, [_vp, _vp, _vp, _i64, _i64, _vp, _vp, _i32, _vp, _vp,
                                          _f64, _i64, _vp, _vp, _vp]),
}


class Pass1Counts(ctypes.Structure):
    """struct hdfe_pass1_counts."""
    _fields_ = [(n, _i64) for n in ("n_rows", "n_groups", "n_cells", "n_ident_groups",
                                    "n_ident_cells", "status")]


class SbuildInfo(ctypes.Structure):
    """struct hdfe_sbuild_info."""
    _fields_ = [(n, _i64) for n in ("L", "nnz", "n_wide", "n_warp_rows", "n_block_rows",
                                    "lgrp_len", "temp_len", "status")]


def read_struct(cls, t):
    """A ctypes struct from a device tensor holding it (synchronises)."""
    return cls.from_buffer_copy(t.cpu().numpy().tobytes()[:ctypes.sizeof(cls)])


class PcgInfo(ctypes.Structure):
    """struct hdfe_pcg_info."""
    _fields_ = [("iterations", _i64), ("converged", _i32), ("status", _i32),
                ("max_rel", _f64)]


_lib = None


def lib():
    """The loaded library; raises ImportError when it has not been built."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise ImportError(f"{LIB_PATH.name} is not built; run "
                              "`python -m hdfe_stream_b200.build` (needs nvcc)")
        handle = ctypes.CDLL(str(LIB_PATH))
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(handle, name)
            fn.restype = res
            fn.argtypes = args
        _lib = handle
    return _lib


class HDFEError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"hdfe_b200 error {code}: {msg}")
        self.code = code


def check(status: int) -> None:
    if status != HDFE_OK:
        raise HDFEError(status, lib().hdfe_error_string().decode())


def ptr(t) -> int | None:
    """Device pointer of a torch tensor (None for None)."""
    return None if t is None else t.data_ptr()


def stream_handle(stream=None) -> int:
    import torch
    s = torch.cuda.current_stream() if stream is None else stream
    return s.cuda_stream

"""The C ABI: the library builds, loads without a GPU, and exports every
entry point include/hdfe_b200.h declares (no device calls here)."""

import re
from pathlib import Path

import pytest

REPO = Path(__file__).resolve().parents[1]


def declared_functions():
    names = set()
    for h in (REPO / "include").glob("*.h"):
        text = re.sub(r"/\*.*?\*/", "", h.read_text(), flags=re.S)
        names |= set(re.findall(r"\b(hdfe_\w+)\s*\(", text))
    return sorted(names)


def test_header_declares_entry_points():
    names = declared_functions()
    assert "hdfe_pcg_solve" in names and "hdfe_error_string" in names


def test_library_exports_every_declared_symbol():
    from hdfe_stream_b200 import _lib
    handle = _lib.lib()
    missing = [n for n in declared_functions() if not hasattr(handle, n)]
    assert not missing, missing
    assert b"sm_100a" in handle.hdfe_version()


def test_binding_covers_every_declared_symbol():
    from hdfe_stream_b200 import _lib
    assert set(declared_functions()) == set(_lib.SIGNATURES)


def test_bad_arguments_are_rejected_without_a_device():
    from hdfe_stream_b200 import _lib
    # k out of range: rejected before any CUDA call
    assert _lib.lib().hdfe_pcg_workspace_bytes(10, 10, 0) == -1
    assert _lib.lib().hdfe_pcg_workspace_bytes(10, 10, _lib.PCG_MAX_K + 1) == -1
    assert _lib.lib().hdfe_pcg_mixed_workspace_bytes(10, 10, _lib.PCG_MIXED_MAX_K + 1) == -1
    st = _lib.lib().hdfe_pcg_solve(None, None, None, 0, 0, None, None, 3, None, None, 1e-10,
                                   10, None, None, 0, None, None)
    assert st == _lib.HDFE_ERR_ARG
    assert b"bad argument" in _lib.lib().hdfe_error_string()


def test_backend_without_library_says_what_to_build(monkeypatch, tmp_path):
    from hdfe_stream_b200 import _lib, gpu
    monkeypatch.setattr(_lib, "_lib", None)
    monkeypatch.setattr(_lib, "LIB_PATH", tmp_path / "missing.so")
    with pytest.raises(ImportError, match="hdfe_stream_b200.build"):
        gpu.cuda_backend()

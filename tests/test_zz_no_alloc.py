"""hdfe_pcg_solve_noalloc: the PCG for callers that cannot allocate device
memory (a host binding without a CUDA allocator of its own, or code that
must not call cudaMalloc because it synchronises the device).  Its scratch
lives in a device array inside the library; here it is checked, through the
C ABI, against hdfe_pcg_solve with a caller-provided workspace, on two calls
in a row with different right-hand sides (the second call reuses the array
the first one left behind).  This file sorts last so a run that stops at the
first failure has run every other test before it."""

import ctypes

import numpy as np
import pytest

import oracle as orc

pytestmark = pytest.mark.gpu


def _system(seed=31):
    from hdfe_stream_b200.simulate import pass0_layout, simulate_panel
    rows = pass0_layout(simulate_panel(20_000, 2_000, 10, spell=(8, 8), p_move=0.1, seed=seed))
    cells = orc.pass1(rows)
    return orc.build_explicit(cells), orc.jacobi(cells.diag)


def _solve(lib, S, dinv, B, zero, noalloc):
    import torch
    from hdfe_stream_b200 import _lib
    dev = torch.device("cuda", 0)
    indptr, indices, data = (torch.as_tensor(np.ascontiguousarray(a)).to(dev) for a in S)
    d = torch.as_tensor(dinv).to(dev)
    Bd = torch.as_tensor(np.ascontiguousarray(B)).to(dev)
    zd = torch.as_tensor(zero.astype(np.uint8)).to(dev)
    X = torch.empty_like(Bd)
    info = torch.zeros(3, dtype=torch.float64, device=dev)
    L, k = B.shape
    nnz = len(S[2])
    stream = torch.cuda.current_stream().cuda_stream
    if noalloc:
        st = lib.hdfe_pcg_solve_noalloc(indptr.data_ptr(), indices.data_ptr(), data.data_ptr(), L,
                                        nnz, d.data_ptr(), Bd.data_ptr(), k, zd.data_ptr(), None,
                                        1e-11, 5000, X.data_ptr(), info.data_ptr(), stream)
    else:
        nbytes = lib.hdfe_pcg_workspace_bytes(L, nnz, k)
        ws = torch.empty(int(nbytes), dtype=torch.uint8, device=dev)
        st = lib.hdfe_pcg_solve(indptr.data_ptr(), indices.data_ptr(), data.data_ptr(), L, nnz,
                                d.data_ptr(), Bd.data_ptr(), k, zd.data_ptr(), None, 1e-11, 5000,
                                X.data_ptr(), ws.data_ptr(), ws.numel(), info.data_ptr(), stream)
    assert st == _lib.HDFE_OK, lib.hdfe_error_string()
    torch.cuda.synchronize()
    inf = _lib.PcgInfo.from_buffer_copy(info.cpu().numpy().tobytes())
    assert inf.status == _lib.HDFE_OK
    return X.cpu().numpy(), int(inf.iterations), bool(inf.converged)


def test_noalloc_matches_the_workspace_entry_point():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from hdfe_stream_b200 import _lib
    lib = _lib.lib()
    S, dinv = _system()
    L = len(dinv)
    rng = np.random.default_rng(8)
    for call, k in enumerate((3, 5)):            # two calls in a row, different shapes
        B = orc.csr_matmat(S, rng.standard_normal((L, k)))
        zero = np.zeros(k, bool)
        zero[1] = True
        B[:, 1] = 0.0
        X_ws, it_ws, ok_ws = _solve(lib, S, dinv, B, zero, noalloc=False)
        X_na, it_na, ok_na = _solve(lib, S, dinv, B, zero, noalloc=True)
        assert ok_ws and ok_na, call
        assert it_na == it_ws
        assert np.all(X_na[:, 1] == 0.0)
        assert np.max(np.abs(X_na - X_ws)) <= 1e-8 * np.max(np.abs(X_ws))


def test_noalloc_rejects_sizes_beyond_its_scratch():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from hdfe_stream_b200 import _lib
    lib = _lib.lib()
    # rejected on the host, before any pointer is used or any kernel launched
    st = lib.hdfe_pcg_solve_noalloc(None, None, None, 5_000_000, 1, None, None, 8, None, None,
                                    1e-10, 10, None, None, None)
    assert st == _lib.HDFE_ERR_WORKSPACE
    assert b"too large" in lib.hdfe_error_string()

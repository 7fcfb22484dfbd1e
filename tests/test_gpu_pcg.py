"""The device block-PCG against the oracle (the reference's _pcg restated),
on the golden panels' S and on larger panels: zero columns, warm starts,
iteration counts and solutions, with the tolerances of the reference's own
device test (tests/test_gpu.py:56-81 there: |d iterations| <= 1,
max|dX| < 1e-8 max|X|)."""

import numpy as np
import pytest

import oracle as orc
from conftest import golden_rows, load_golden, GOLDEN_PANELS

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def device():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch.device("cuda", 0)


def _solvers(S, diag, tol, maxiter=5000):
    from hdfe_stream_b200 import gpu
    A = gpu.DeviceCSR.from_host(*S)
    return gpu.BlockSolver(A, orc.jacobi(diag), tol, maxiter)


@pytest.mark.parametrize("name", GOLDEN_PANELS)
def test_pcg_matches_oracle_on_golden(device, name):
    g = load_golden(name)
    S = (g["S_indptr"], g["S_indices"], g["S_data"])
    tol = float(g["tol"])
    solve = _solvers(S, g["diag"], tol)
    for x0 in (None, g["pcg_x0"]):
        X_ref, it_ref, ok_ref, _ = orc.pcg(S, orc.jacobi(g["diag"]), g["pcg_b"], g["pcg_zero"],
                                           x0, tol)
        X, it, ok, rel = solve(g["pcg_b"], g["pcg_zero"], x0)
        assert ok and ok_ref
        assert abs(it - it_ref) <= 1
        assert np.all(X[:, 1] == 0.0)
        assert np.max(np.abs(X - X_ref)) < 1e-8 * np.max(np.abs(X_ref))
        assert rel <= tol


@pytest.mark.parametrize("k", [1, 3, 4, 5, 8, 11, 16, 23, 32])
def test_pcg_widths(device, k):
    from hdfe_stream_b200.simulate import pass0_layout, simulate_panel
    rows = pass0_layout(simulate_panel(20_000, 2_000, 10, spell=(8, 8), p_move=0.1, seed=7))
    c = orc.pass1(rows)
    S = orc.build_explicit(c)
    rng = np.random.default_rng(k)
    b = orc.csr_matmat(S, rng.standard_normal((c.L, k)))
    X_ref, it_ref, ok_ref, _ = orc.pcg(S, orc.jacobi(c.diag), b, None, None, 1e-10)
    X, it, ok, rel = _solvers(S, c.diag, 1e-10)(b)
    assert ok and ok_ref and abs(it - it_ref) <= 1
    assert np.max(np.abs(X - X_ref)) < 1e-8 * np.max(np.abs(X_ref))


@pytest.mark.parametrize("k", [7, 13, 32])
def test_pcg_wide_zero_columns_and_warm_start(device, k):
    """Blocks solved one column per lane: zero columns stay 0, a warm start
    is honoured, and every column matches the oracle's CG."""
    from hdfe_stream_b200.simulate import pass0_layout, simulate_panel
    rows = pass0_layout(simulate_panel(20_000, 2_000, 10, spell=(8, 8), p_move=0.1, seed=11))
    c = orc.pass1(rows)
    S = orc.build_explicit(c)
    rng = np.random.default_rng(100 + k)
    b = orc.csr_matmat(S, rng.standard_normal((c.L, k)))
    zero = np.zeros(k, bool)
    zero[[1, k - 1]] = True
    x0 = 0.5 * rng.standard_normal((c.L, k))
    solve = _solvers(S, c.diag, 1e-10)
    for guess in (None, x0):
        X_ref, it_ref, ok_ref, _ = orc.pcg(S, orc.jacobi(c.diag), b, zero, guess, 1e-10)
        X, it, ok, rel = solve(b, zero, guess)
        assert ok and ok_ref and abs(it - it_ref) <= 1 and rel <= 1e-10
        assert np.all(X[:, zero] == 0.0)
        assert np.max(np.abs(X - X_ref)) < 1e-8 * np.max(np.abs(X_ref))


def test_pcg_wide_golden_and_deterministic(device):
    """The golden right-hand sides repeated to 32 columns: each copy solves
    like the narrow kernel's, and two solves give identical bits."""
    g = load_golden("akm_small")
    S = (g["S_indptr"], g["S_indices"], g["S_data"])
    reps = -(-32 // g["pcg_b"].shape[1])
    b = np.tile(g["pcg_b"], (1, reps))[:, :32]
    zero = np.tile(g["pcg_zero"], reps)[:32]
    solve = _solvers(S, g["diag"], 1e-12)
    X_ref, it_ref, ok_ref, _ = orc.pcg(S, orc.jacobi(g["diag"]), b, zero, None, 1e-12)
    X1, it, ok, rel = solve(b, zero)
    X2, *_ = solve(b, zero)
    assert ok and abs(it - it_ref) <= 1
    assert np.array_equal(X1, X2)
    assert np.max(np.abs(X1 - X_ref)) < 1e-8 * np.max(np.abs(X_ref))


def test_pcg_wide_maxiter(device):
    g = load_golden("akm_small")
    S = (g["S_indptr"], g["S_indices"], g["S_data"])
    b = np.tile(g["pcg_b"], (1, 8))[:, :20]
    X, it, ok, rel = _solvers(S, g["diag"], 1e-12, maxiter=3)(b)
    X_ref, it_ref, ok_ref, rel_ref = orc.pcg(S, orc.jacobi(g["diag"]), b, None, None, 1e-12,
                                             maxiter=3)
    assert it == it_ref == 3 and not ok and not ok_ref
    assert rel == pytest.approx(rel_ref, rel=1e-6)
    assert np.max(np.abs(X - X_ref)) < 1e-8 * np.max(np.abs(X_ref))


def test_pcg_is_deterministic(device):
    g = load_golden("akm_small")
    S = (g["S_indptr"], g["S_indices"], g["S_data"])
    solve = _solvers(S, g["diag"], 1e-12)
    X1, *_ = solve(g["pcg_b"])
    X2, *_ = solve(g["pcg_b"])
    assert np.array_equal(X1, X2)


def test_pcg_maxiter_reports_not_converged(device):
    g = load_golden("akm_small")
    S = (g["S_indptr"], g["S_indices"], g["S_data"])
    X, it, ok, rel = _solvers(S, g["diag"], 1e-12, maxiter=3)(g["pcg_b"])
    X_ref, it_ref, ok_ref, rel_ref = orc.pcg(S, orc.jacobi(g["diag"]), g["pcg_b"], None, None,
                                             1e-12, maxiter=3)
    assert it == it_ref == 3 and not ok and not ok_ref
    assert rel == pytest.approx(rel_ref, rel=1e-6)


def test_pcg_all_zero_columns(device):
    g = load_golden("akm_small")
    S = (g["S_indptr"], g["S_indices"], g["S_data"])
    b = np.zeros((len(g["diag"]), 2))
    X, it, ok, rel = _solvers(S, g["diag"], 1e-10)(b, np.array([True, True]))
    assert it == 0 and ok and rel == 0.0 and np.all(X == 0)


def test_explicit_solver_seam(device):
    import scipy.sparse as sp
    from hdfe_stream_b200 import gpu
    g = load_golden("akm_weighted")
    L = len(g["diag"])
    S = sp.csr_matrix((g["S_data"], g["S_indices"], g["S_indptr"]), shape=(L, L))
    solve, name = gpu.explicit_solver(S, orc.jacobi(g["diag"]), 1e-11, 5000)
    assert "B200" in name or "NVIDIA" in name
    X, it, ok, rel = solve(g["pcg_b"], g["pcg_zero"], None)
    assert ok
    assert np.max(np.abs(X - g["pcg_X"])) < 1e-8 * np.max(np.abs(g["pcg_X"]))


@pytest.mark.parametrize("name", GOLDEN_PANELS)
def test_mixed_precision_matches_fp64(device, name):
    """FP32 inner CG with FP64 refinement: the same FP64 residual tolerance,
    solutions within 1e-8 relative of the FP64 oracle's."""
    from hdfe_stream_b200 import gpu
    g = load_golden(name)
    S = (g["S_indptr"], g["S_indices"], g["S_data"])
    A = gpu.DeviceCSR.from_host(*S)
    solve = gpu.BlockSolver(A, orc.jacobi(g["diag"]), 1e-11, 5000, precision="mixed")
    for x0 in (None, g["pcg_x0"]):
        X_ref, *_ = orc.pcg(S, orc.jacobi(g["diag"]), g["pcg_b"], g["pcg_zero"], x0, 1e-13)
        X, it, ok, rel = solve(g["pcg_b"], g["pcg_zero"], x0)
        assert ok and rel <= 1e-11
        assert np.all(X[:, 1] == 0.0)
        # S is singular (shifts between effects within a component); the FP32
        # inner solves may move X along that null space, which no fitted value
        # sees, so the identified part S X is what is compared
        dSX = orc.csr_matmat(S, X - X_ref)
        assert np.max(np.abs(dSX)) < 1e-8 * np.max(np.abs(g["pcg_b"]))


@pytest.mark.parametrize("k", [1, 3, 8, 13, 32])
def test_mixed_precision_widths(device, k):
    """The refined solve at register widths (1, 3) and one column per lane
    (8, 13 padded to 16, 32), with a zero column and a warm start for the
    wide ones, against the FP64 oracle at 1e-13."""
    from hdfe_stream_b200 import gpu
    from hdfe_stream_b200.simulate import pass0_layout, simulate_panel
    rows = pass0_layout(simulate_panel(20_000, 2_000, 10, spell=(8, 8), p_move=0.1, seed=9))
    c = orc.pass1(rows)
    S = orc.build_explicit(c)
    rng = np.random.default_rng(k)
    b = orc.csr_matmat(S, rng.standard_normal((c.L, k)))
    zero = np.zeros(k, bool)
    if k > 4:
        b[:, 2] = 0.0
        zero[2] = True
    dinv = orc.jacobi(c.diag)
    X_ref, *_ = orc.pcg(S, dinv, b, zero, None, 1e-13)
    solve = gpu.BlockSolver(gpu.DeviceCSR.from_host(*S), dinv, 1e-10, 5000, precision="mixed")
    X, it, ok, rel = solve(b, zero)
    assert ok and rel <= 1e-10
    assert np.max(np.abs(orc.csr_matmat(S, X - X_ref))) < 1e-8 * np.max(np.abs(b))
    if k > 4:
        assert np.all(X[:, 2] == 0.0)
        x0 = X_ref + 1e-3 * rng.standard_normal(X_ref.shape)
        X2, it2, ok2, rel2 = solve(b, zero, x0)
        assert ok2 and rel2 <= 1e-10 and it2 <= it
        assert np.max(np.abs(orc.csr_matmat(S, X2 - X_ref))) < 1e-8 * np.max(np.abs(b))


def test_mixed_precision_maxiter(device):
    from hdfe_stream_b200 import gpu
    g = load_golden("akm_small")
    S = (g["S_indptr"], g["S_indices"], g["S_data"])
    solve = gpu.BlockSolver(gpu.DeviceCSR.from_host(*S), orc.jacobi(g["diag"]), 1e-12, 4,
                            precision="mixed")
    X, it, ok, rel = solve(g["pcg_b"])
    assert it == 4 and not ok and rel > 1e-12


@pytest.mark.parametrize("k", [1, 3, 32])
def test_stream_matvec_matches_explicit_s(device, k):
    """`_nb_stream_matvec`: (D_o' M_0 D_o) P from the cells equals S P with
    the explicit S, on the golden panels and a two-dimension panel."""
    import torch
    from hdfe_stream_b200 import _lib, fit
    from hdfe_stream_b200.simulate import pass0_layout, simulate_panel
    panels = [golden_rows(load_golden(n)) for n in GOLDEN_PANELS]
    panels.append(pass0_layout(simulate_panel(20_000, 2_000, 10, spell=(3, 10), p_move=0.1,
                                              weights=True, seed=13)))
    for rows in panels:
        c = orc.pass1(rows)
        S = orc.build_explicit(c)
        P = np.random.default_rng(k).standard_normal((c.L, k))
        ref = orc.csr_matmat(S, P)
        cells = fit.pass1(fit.DeviceRows.from_rows(rows))
        out = torch.empty((cells.L, k), dtype=torch.float64, device=device)
        nlev = np.asarray(cells.n_levels, dtype=np.int64)
        st = torch.zeros(1, dtype=torch.int32, device=device)
        Pd = torch.as_tensor(P, device=device)
        _lib.check(_lib.lib().hdfe_stream_matvec(
            cells.starts.data_ptr(), int(cells.starts.shape[0]) - 1, cells.codes.data_ptr(),
            len(nlev), nlev.ctypes.data, cells.n.data_ptr(), Pd.data_ptr(), k, out.data_ptr(),
            st.data_ptr(), _lib.stream_handle()))
        got = out.cpu().numpy()
        assert int(st.item()) == 0
        assert np.max(np.abs(got - ref)) < 1e-12 * np.max(np.abs(ref))


@pytest.mark.parametrize("name", list(GOLDEN_PANELS) + ["weighted"])
def test_stream_cg_matches_explicit(device, name):
    """The `stream_cg` solver (S P from the cells every iteration) gives the
    explicit solve's fixed effects (1e-9) with iterations within one, and
    the oracle's PCG on the explicit S."""
    from hdfe_stream_b200 import fit
    from hdfe_stream_b200.simulate import pass0_layout, simulate_panel
    rows = (golden_rows(load_golden(name)) if name != "weighted" else
            pass0_layout(simulate_panel(20_000, 2_000, 10, spell=(3, 10), p_move=0.1,
                                        weights=True, seed=13)))
    drows = fit.DeviceRows.from_rows(rows)
    cells = fit.pass1(drows)
    want = fit.solve(cells, fit.build_s(cells), tol=1e-12)
    got = fit.solve(cells, None, tol=1e-12, solver="stream_cg")
    assert got.info["solver"] == "stream_cg" and got.info["converged"]
    g, w = got.gamma.cpu().numpy(), want.gamma.cpu().numpy()
    assert np.max(np.abs(g - w)) <= 1e-9 * np.max(np.abs(w))
    its = np.atleast_1d(got.info["iterations"]) - np.atleast_1d(want.info["iterations"])
    assert np.all(np.abs(its) <= 1)


def test_solver_handle_matches_block_solver(device):
    """The opaque solver handle of the C ABI (`hdfe_solver_create` /
    `_solve` / `_destroy`, the `explicit_solver` closure for FFI hosts): the
    same X bit for bit as BlockSolver on the same S, host info filled, host
    zero flags honoured, k above max_k refused."""
    import ctypes
    import torch
    from hdfe_stream_b200 import _lib, fit
    rows = golden_rows(load_golden(GOLDEN_PANELS[0]))
    drows = fit.DeviceRows.from_rows(rows)
    cells = fit.pass1(drows)
    S = fit.build_s(cells)
    dinv = fit.jacobi(cells.diag).contiguous()
    lib = _lib.lib()
    handle = ctypes.c_void_p()
    _lib.check(lib.hdfe_solver_create(S.indptr.data_ptr(), S.indices.data_ptr(),
                                      S.data.data_ptr(), S.L, S.nnz, dinv.data_ptr(), 1e-12,
                                      5000, 4, ctypes.byref(handle)))
    try:
        B = cells.rhs.contiguous()
        k = int(B.shape[1])
        X = torch.empty_like(B)
        info = _lib.PcgInfo()
        zero = (ctypes.c_uint8 * k)(*([0] * (k - 1) + [1]))
        _lib.check(lib.hdfe_solver_solve(handle, B.data_ptr(), k, zero, None, X.data_ptr(),
                                         ctypes.byref(info), _lib.stream_handle()))
        from hdfe_stream_b200.gpu import BlockSolver
        want, its, conv, rel = BlockSolver(S, dinv, 1e-12, 5000).solve_device(
            B, np.array([False] * (k - 1) + [True]))
        assert torch.equal(X, want)
        assert (info.iterations, bool(info.converged)) == (its, conv)
        assert abs(info.max_rel - rel) <= 1e-15
        assert float(X[:, -1].abs().max()) == 0.0
        X5 = torch.empty((S.L, 5), dtype=torch.float64, device=device)
        B5 = torch.zeros_like(X5)
        assert lib.hdfe_solver_solve(handle, B5.data_ptr(), 5, None, None, X5.data_ptr(),
                                     ctypes.byref(info), _lib.stream_handle()) != _lib.HDFE_OK
    finally:
        assert lib.hdfe_solver_destroy(handle) == _lib.HDFE_OK


def _small_cases():
    from hdfe_stream_b200.simulate import pass0_layout, simulate_panel
    out = []
    for name in GOLDEN_PANELS:
        g = load_golden(name)
        out.append((name, (g["S_indptr"], g["S_indices"], g["S_data"]), g["diag"],
                    list(g["n_levels"])))
    rows = pass0_layout(simulate_panel(20_000, 2_000, 10, spell=(2, 10), p_move=0.1,
                                       weights=True, seed=9))
    c = orc.pass1(rows)
    out.append(("weighted_20k", orc.build_explicit(c), c.diag, list(c.n_levels)))
    return out


SMALL_CASES = _small_cases()


@pytest.mark.parametrize("case", SMALL_CASES, ids=[c[0] for c in SMALL_CASES])
def test_small_block_split_and_solve(device, case):
    """S with its trailing small dimension (the years) stored densely
    (`hdfe_small_split` + `hdfe_pcg_solve_small`): the split reproduces S's
    entries exactly (big block in CSR with the entries' order kept, cross
    and small dense), and the solve matches the oracle's CG on the whole S
    for 1, 3 and 4 columns, with a zero column and a warm start."""
    import scipy.sparse as sp
    import torch
    from hdfe_stream_b200 import gpu
    _, S, diag, n_levels = case
    small = gpu.small_levels(n_levels)
    assert small is not None
    first, count = small
    A = gpu.DeviceCSR.from_host(*S)
    split = gpu.SmallSplit(A, first, count)
    dense = sp.csr_matrix((S[2], S[1], S[0]), shape=(A.L, A.L))
    big = dense[:first, :first].tocsr()
    big.sort_indices()
    ip = split.S_big.indptr.cpu().numpy()
    assert np.array_equal(ip[:first + 1], big.indptr) and np.all(ip[first:] == big.nnz)
    assert np.array_equal(split.S_big.indices.cpu().numpy(), big.indices)
    assert np.array_equal(split.S_big.data.cpu().numpy(), big.data)
    cross = split.cross.cpu().numpy()
    assert np.array_equal(cross[:, :count], dense[:first, first:].toarray())
    assert np.all(cross[:, count:] == 0.0)
    assert np.array_equal(split.small.cpu().numpy(), dense[first:, first:].toarray())

    dinv = orc.jacobi(diag)
    plain = gpu.BlockSolver(A, dinv, 1e-10, 5000)
    solver = gpu.BlockSolver(A, dinv, 1e-10, 5000, small=small)
    rng = np.random.default_rng(first)
    for k in (1, 3, 4):
        b = orc.csr_matmat(S, rng.standard_normal((A.L, k)))
        zero = np.zeros(k, bool)
        if k > 1:
            zero[1] = True
        x0 = 0.3 * rng.standard_normal((A.L, k))
        for guess in (None, x0):
            X_ref, it_ref, ok_ref, _ = orc.pcg(S, dinv, b, zero, guess, 1e-10)
            X, it, ok, rel = solver(b, zero, guess)
            Xp, itp, _, _ = plain(b, zero, guess)
            assert ok and ok_ref and abs(it - it_ref) <= 1 and rel <= 1e-10, (k, it, it_ref)
            assert np.all(X[:, zero] == 0.0)
            assert np.max(np.abs(X - X_ref)) < 1e-8 * np.max(np.abs(X_ref))
            assert np.max(np.abs(X - Xp)) < 1e-9 * np.max(np.abs(Xp)) and abs(it - itp) <= 1
    # deterministic: the same bits twice
    b = orc.csr_matmat(S, rng.standard_normal((A.L, 3)))
    X1, *_ = solver(b)
    X2, *_ = solver(b)
    assert np.array_equal(X1, X2)

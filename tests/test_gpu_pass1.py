"""Device pass 1 and the device S build against the oracle (the reference's
_pass1_cells and _build_explicit restated): integer outputs identical, FP64
outputs to 1e-12 relative (the device sums in another order)."""

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


def rel(a, b):
    a, b = np.asarray(a, float), np.asarray(b, float)
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300)) if a.size else 0.0


def three_dim_rows(seed=5, regions=7):
    """A panel with a third non-streamed dimension (a region of the firm)."""
    from hdfe_stream_b200.simulate import Rows, pass0_layout, simulate_panel
    r = pass0_layout(simulate_panel(3_000, 300, 8, spell=(2, 8), p_move=0.2, seed=seed))
    region = (r.codes[:, 0] % regions).astype(np.uint32)
    codes = np.column_stack([r.codes, region])
    order = np.lexsort((r.V[:, 2], r.V[:, 1], r.V[:, 0], codes[:, 2], codes[:, 1],
                        codes[:, 0], r.gcode))
    return Rows(gcode=r.gcode[order], codes=np.ascontiguousarray(codes[order]),
                V=r.V[order], w=None, n_levels=r.n_levels + [regions], n_groups=r.n_groups,
                names=r.names)


def years_first_rows(seed=8):
    """The year before the firm (`| worker + year + firm`): pass 0 orders a
    group's rows by year, so the firms' codes within a group are not sorted
    and their level lists take the walk over the group's cells."""
    from hdfe_stream_b200.simulate import Rows, pass0_layout, simulate_panel
    r = pass0_layout(simulate_panel(4_000, 400, 8, spell=(2, 8), p_move=0.25, seed=seed))
    codes = np.ascontiguousarray(r.codes[:, ::-1])
    order = np.lexsort((r.V[:, 2], r.V[:, 1], r.V[:, 0], codes[:, 1], codes[:, 0], r.gcode))
    return Rows(gcode=r.gcode[order], codes=np.ascontiguousarray(codes[order]),
                V=r.V[order], w=None, n_levels=r.n_levels[::-1], n_groups=r.n_groups,
                names=r.names)


def panels():
    from hdfe_stream_b200.simulate import pass0_layout, simulate_panel
    out = [(n, golden_rows(load_golden(n))) for n in GOLDEN_PANELS]
    out.append(("akm_20k", pass0_layout(simulate_panel(20_000, 2_000, 10, spell=(8, 8),
                                                        p_move=0.1, seed=11))))
    out.append(("weighted_uneven", pass0_layout(simulate_panel(
        30_000, 1_500, 12, spell=(1, 12), p_move=0.12, weights=True, seed=12))))
    out.append(("three_dims", three_dim_rows()))
    # more than 16 wide rows: the wide x wide block takes its atomic path
    out.append(("many_wide", three_dim_rows(seed=6, regions=30)))
    out.append(("years_first", years_first_rows()))
    # 20 cells a group: 32 groups' cells exceed what the list pass stages in
    # shared memory, so it reads them in place
    out.append(("long_groups", pass0_layout(simulate_panel(3_000, 300, 20, spell=(20, 20),
                                                            p_move=0.15, seed=13))))
    return out


PANELS = panels()


@pytest.mark.parametrize("name,rows", PANELS, ids=[p[0] for p in PANELS])
def test_pass1_matches_oracle(device, name, rows):
    from hdfe_stream_b200 import fit
    ref = orc.pass1(rows)
    got = fit.pass1(fit.DeviceRows.from_rows(rows), keep_sums=True)
    assert got.counts["n_cells"] == ref.n_cells
    assert got.counts["n_groups"] == ref.fe0_rank
    assert np.array_equal(got.starts.cpu().numpy(), ref.starts)
    assert np.array_equal(got.codes.cpu().numpy().view(np.uint32), ref.codes)
    assert np.array_equal(got.cnt.cpu().numpy(), ref.cnt)
    if rows.w is None:
        assert np.array_equal(got.n.cpu().numpy(), ref.n)
        assert np.array_equal(got.obs.cpu().numpy(), ref.obs)
    else:
        assert rel(got.n.cpu().numpy(), ref.n) < 1e-14
        assert rel(got.obs.cpu().numpy(), ref.obs) < 1e-13
    # numpy sums the column sequentially, the device by blocks: 1e-12 apart
    assert rel(got.means.cpu().numpy(), ref.means) < 1e-12
    assert rel(got.sums.cpu().numpy(), ref.sums) < 1e-12
    assert rel(got.diag.cpu().numpy(), ref.diag) < 1e-12
    assert rel(got.rhs.cpu().numpy(), ref.rhs) < 1e-12
    gn = np.add.reduceat(ref.n, ref.starts[:-1])
    assert rel(got.group_n.cpu().numpy(), gn) < 1e-14


@pytest.mark.parametrize("name,rows", PANELS, ids=[p[0] for p in PANELS])
def test_sbuild_matches_oracle(device, name, rows):
    from hdfe_stream_b200 import fit
    ref_cells = orc.pass1(rows)
    ip, ix, dt = orc.build_explicit(ref_cells)
    cells = fit.pass1(fit.DeviceRows.from_rows(rows))
    S = fit.build_s(cells)
    assert S.nnz == len(dt)
    assert np.array_equal(S.indptr.cpu().numpy(), ip)
    assert np.array_equal(S.indices.cpu().numpy(), ix)
    d = S.data.cpu().numpy()
    assert np.max(np.abs(d - dt)) <= 1e-12 * np.max(np.abs(dt))
    # exact zeros of the reference (stayers' cancellations) stay tiny
    zero = dt == 0.0
    if zero.any():
        assert np.max(np.abs(d[zero])) <= 1e-12 * np.max(np.abs(dt))


def test_sbuild_without_pass1_statistics(device):
    """The S build computes the per-level statistics itself when not given."""
    from hdfe_stream_b200 import fit
    rows = PANELS[3][1]
    ip, ix, dt = orc.build_explicit(orc.pass1(rows))
    cells = fit.pass1(fit.DeviceRows.from_rows(rows))
    cells.lcount = None
    cells.work = None
    S = fit.build_s(cells)
    assert np.array_equal(S.indptr.cpu().numpy(), ip)
    assert np.array_equal(S.indices.cpu().numpy(), ix)
    assert np.max(np.abs(S.data.cpu().numpy() - dt)) <= 1e-12 * np.max(np.abs(dt))


def test_pass1_level_statistics(device):
    """lcount / work: identifying groups per level and their cells
    (`_nb_level_groups` / `_nb_row_work`)."""
    from hdfe_stream_b200 import fit
    rows = PANELS[4][1]
    c = orc.pass1(rows)
    cells = fit.pass1(fit.DeviceRows.from_rows(rows))
    L = c.L
    lcount = np.zeros(L, np.int64)
    work = np.zeros(L, np.int64)
    for g in range(len(c.starts) - 1):
        s, e = c.starts[g], c.starts[g + 1]
        for d in range(c.codes.shape[1]):
            for lv in np.unique(c.codes[s:e, d]):
                lcount[c.offs[d] + lv] += 1
                work[c.offs[d] + lv] += e - s
    assert np.array_equal(cells.lcount.cpu().numpy(), lcount)
    assert np.array_equal(cells.work.cpu().numpy(), work)


def test_sbuild_is_deterministic(device):
    from hdfe_stream_b200 import fit
    rows = PANELS[3][1]
    cells = fit.pass1(fit.DeviceRows.from_rows(rows))
    a = fit.build_s(cells)
    b = fit.build_s(cells)
    assert np.array_equal(a.indices.cpu().numpy(), b.indices.cpu().numpy())
    # narrow rows sum in a fixed order; the wide x wide block sums atomically
    da, db = a.data.cpu().numpy(), b.data.cpu().numpy()
    assert np.max(np.abs(da - db)) <= 1e-13 * np.max(np.abs(da))


def test_pass1_rejects_out_of_range_codes(device):
    from hdfe_stream_b200 import _lib, fit
    rows = golden_rows(load_golden("akm_components"))
    bad = fit.DeviceRows.from_rows(rows)
    bad.n_levels = [rows.n_levels[0] - 1, rows.n_levels[1]]     # the last firm is now out of range
    with pytest.raises(_lib.HDFEError, match="out of range"):
        fit.pass1(bad)

"""The bench's algorithmic-byte accounting (CPU): the PCG iteration's bytes
are the whole S's 12 nnz + 4 (L+1) + 72 L k whatever layout solves it, the
split form's own bytes are reported beside them, and pass 1 and the S build
follow their compulsory-byte formulas."""

import sys
import types
from pathlib import Path

sys.path.insert(0, str(Path(__file__).resolve().parents[1]))

import bench  # noqa: E402


def _rows(N=1000, D=2, n_levels=(90, 10), w=None):
    return types.SimpleNamespace(n_rows=N, codes=types.SimpleNamespace(shape=(N, D)),
                                 n_levels=list(n_levels), w=w)


COUNTS = {"n_ident_cells": 800, "n_ident_groups": 120}


def test_pcg_bytes_are_the_whole_s_figure():
    S = types.SimpleNamespace(nnz=5000)
    L, k, its = 100, 3, 7
    by = bench.phase_bytes(_rows(), COUNTS, S, its)
    assert by["pcg_kernel"] == (12 * 5000 + 4 * (L + 1) + 8 * L * k * 9) * its
    assert "pcg_kernel_split" not in by


def test_split_form_bytes_reported_beside_the_whole_s_figure():
    S = types.SimpleNamespace(nnz=5000)
    L, k, its = 100, 3, 7
    small = {"big_nnz": 2000, "first": 90}
    by = bench.phase_bytes(_rows(), COUNTS, S, its, small=small)
    whole = (12 * 5000 + 4 * (L + 1) + 8 * L * k * 9) * its
    split = (12 * 2000 + 8 * (L + 1) + 8 * 16 * 90 + 8 * L * k * 9 + 16 * 90 * k) * its
    assert by["pcg_kernel"] == whole
    assert by["pcg_kernel_split"] == split
    assert split < whole                # the split form moves fewer bytes


def test_pass1_and_sbuild_bytes():
    S = types.SimpleNamespace(nnz=5000)
    N, D, m, L = 1000, 2, 3, 100
    M, G = COUNTS["n_ident_cells"], COUNTS["n_ident_groups"]
    by = bench.phase_bytes(_rows(), COUNTS, S, 1)
    assert by["pass1"] == N * (4 + 4 * D + 8 * m) + M * (4 * D + 8) + G * 16 + L * 8 * (3 + m)
    assert by["sbuild"] == M * (4 * D + 8) + G * 16 + 5000 * 12 + (L + 1) * 8
    weighted = bench.phase_bytes(_rows(w=object()), COUNTS, S, 1)
    assert weighted["pass1"] == by["pass1"] + 8 * N


def test_zero_iterations_count_one():
    S = types.SimpleNamespace(nnz=10)
    by = bench.phase_bytes(_rows(), COUNTS, S, 0)
    assert by["pcg_kernel"] == 12 * 10 + 4 * 101 + 8 * 100 * 3 * 9

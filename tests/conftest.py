"""Shared fixtures.  `-m gpu` marks the tests that need a B200 (the CUDA
library's parity tests); everything else runs on the CPU."""

import sys
from pathlib import Path

import numpy as np
import pytest

REPO = Path(__file__).resolve().parents[1]
GOLDEN = Path(__file__).resolve().parent / "golden"
for p in (str(REPO), str(REPO / "oracle")):
    if p not in sys.path:
        sys.path.insert(0, p)

GOLDEN_PANELS = ("akm_small", "akm_weighted", "akm_components")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


def load_golden(name):
    return dict(np.load(GOLDEN / f"{name}.npz"))


def golden_rows(g):
    """The golden panel's rows in pass 0's layout."""
    from hdfe_stream_b200.simulate import Rows
    w = g["w"] if len(g["w"]) else None
    return Rows(gcode=g["gcode"], codes=g["codes_rows"], V=g["V"], w=w,
                n_levels=[int(x) for x in g["n_levels"]], n_groups=int(g["n_groups"]),
                names=["log_earn", "age_squared", "age_cubed"])


@pytest.fixture(params=GOLDEN_PANELS)
def golden(request):
    return request.param, load_golden(request.param)

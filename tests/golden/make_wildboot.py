"""Golden vectors for the wild cluster bootstrap, made by the reference's own
core/wildboot.py (`_draws`, `_Test`): seeded per-cluster sums H_g, s_g, a
beta and a small-sample factor; for each weight distribution, restricted and
unrestricted, the t statistic and every bootstrap t* for a fixed seed (and the
Rademacher enumeration when 2^G < reps).  Outputs go to
tests/golden/wildboot.npz.

    python tests/golden/make_wildboot.py /path/to/hdfe-stream
"""

from __future__ import annotations

import importlib
import sys
from pathlib import Path
from types import SimpleNamespace

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE))

from make_golden import import_reference  # noqa: E402

CASES = [("rademacher", True, 40, 999, 11), ("rademacher", False, 40, 999, 12),
         ("mammen", True, 25, 499, 13), ("webb", True, 30, 499, 14),
         ("norm", False, 35, 499, 15), ("rademacher", True, 8, 999, 16)]


def main(root):
    import_reference(root)
    wb = importlib.import_module("hdfe_stream.core.wildboot")
    out = {}
    for c, (kind, null, G, reps, seed) in enumerate(CASES):
        rng = np.random.default_rng(100 + c)
        k = 3
        h = rng.standard_normal((G, 20, k))
        AG = np.einsum("gia,gib->gab", h, h)
        sG = rng.standard_normal((G, k)) * 0.3
        beta = rng.standard_normal(k) * 0.1
        adj = 1.0 + 1.0 / G
        res = SimpleNamespace(_boot={"AG": AG, "sG": sG, "adj": adj}, beta=beta)
        test = wb._Test(res, 1, null)
        tstar = np.concatenate([test.tstar(V) for V in wb._draws(kind, G, reps, seed)])
        out[f"c{c}_AG"], out[f"c{c}_sG"], out[f"c{c}_beta"] = AG, sG, beta
        out[f"c{c}_adj"] = np.array([adj])
        out[f"c{c}_t"] = np.array([test.t])
        out[f"c{c}_tstar"] = tstar
        print(kind, null, G, reps, test.t, tstar[:3])
    np.savez_compressed(HERE / "wildboot.npz", **out)


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else "/root/reference")

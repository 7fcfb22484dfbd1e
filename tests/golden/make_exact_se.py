"""Exact observation-level KSS standard errors and the exact weak-
identification diagnostic for the panel of exact.npz, by the reference's
dense prototype (prototypes/kss_exact.py:848-889 `kss_se` with the smoothed
sigma2 and :918-952 `weak_id`: S^-1, C, P_ii and the eigenvalues of S^- Q
formed densely).

Run once, in a container where the reference tree is readable, after
make_exact.py:

    python tests/golden/make_exact_se.py /path/to/hdfe-stream

Outputs go to tests/golden/exact_se.npz: per component (var(psi),
var(alpha), cov(psi, alpha)) theta, V and its two terms; the three leading
eigenvalues, sum lambda^2, q and the first-stage F.  Nothing at test time
reads the reference.
"""

from __future__ import annotations

import importlib.util
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parents[1]))
sys.path.insert(0, str(HERE))

from make_golden import import_reference  # noqa: E402

NAMES = ("var(psi)", "var(alpha)", "cov(psi, alpha)")


def main(root):
    import_reference(root)          # the package's modules, for the shared smoother
    spec = importlib.util.spec_from_file_location("kss_exact",
                                                  Path(root) / "prototypes" / "kss_exact.py")
    ke = importlib.util.module_from_spec(spec)
    sys.modules["kss_exact"] = ke
    spec.loader.exec_module(ke)
    g = np.load(HERE / "exact.npz")
    kp = ke.Panel(worker=g["gcode"].astype(np.int64), firm=g["codes_rows"][:, 0].astype(np.int64),
                  y=g["V"][:, 0].copy())
    out = {}
    se = ke.kss_se(kp, sigma2_rule="smooth")
    for field in ("theta", "V", "V_first_term", "V_trace_term", "plug_in", "bias"):
        out[f"se_{field}"] = np.array([se[n][field] for n in NAMES])
    print({n: {f: se[n][f] for f in ("theta", "V", "V_first_term", "V_trace_term")}
           for n in NAMES})
    wid = ke.weak_id(kp)
    for k, n in enumerate(NAMES):
        out[f"weak_eig{k}"] = np.array(wid[n]["eigenvalues"])
        out[f"weak_ratio{k}"] = np.array(wid[n]["ratios"])
    out["weak_sum_sq"] = np.array([wid[n]["sum_sq"] for n in NAMES])
    out["weak_q"] = np.array([wid[n]["q"] for n in NAMES])
    out["weak_f_stat"] = np.array([wid[n]["f_stat"] for n in NAMES])
    print(wid)
    np.savez_compressed(HERE / "exact_se.npz", **out)


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else "/root/reference")

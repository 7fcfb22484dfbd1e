"""Exact KSS components for a 1,500-worker panel, by the reference's dense
prototype (prototypes/kss_exact.py `kss`, S^-1 formed densely).

Run once, in a container where the reference tree is readable:

    python tests/golden/make_exact.py /path/to/hdfe-stream

The panel (worker and firm effects only, unweighted) is restricted to its
leave-one-out connected set by the reference's own core/connected.py:503-557
`_leave_one_out`; the rows, the exact leverages and the exact plug-in, bias
and leave-out components -- leaving out an observation (`kss`) and a match
(`kss_match`, centering "reference", with its per-match sigma2 and stayer
flags) -- go to tests/golden/exact.npz.  The prototype divides
the components by n; hdfe-stream by n - 1.  Nothing at test time reads the
reference.
"""

from __future__ import annotations

import importlib.util
import sys
from pathlib import Path

import numpy as np

REPO = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(REPO))
sys.path.insert(0, str(Path(__file__).resolve().parent))

from hdfe_stream_b200.simulate import pass0_layout, simulate_panel  # noqa: E402
from make_golden import import_reference  # noqa: E402
from make_se import loo_keep  # noqa: E402


def main(root):
    mods = import_reference(root)
    spec = importlib.util.spec_from_file_location("kss_exact",
                                                  Path(root) / "prototypes" / "kss_exact.py")
    ke = importlib.util.module_from_spec(spec)
    sys.modules["kss_exact"] = ke
    spec.loader.exec_module(ke)
    panel = simulate_panel(1_500, 150, 8, spell=(2, 8), p_move=0.15, seed=77)
    rows = pass0_layout(panel, loo_keep(mods, panel), year_fe=False)
    kp = ke.Panel(worker=rows.gcode.astype(np.int64), firm=rows.codes[:, 0].astype(np.int64),
                  y=rows.V[:, 0].copy())
    res = ke.kss(kp)
    A, _, _ = ke.design(kp)
    P_ii = ke.leverages(A, ke._dense_inverse(A, None), None)
    keys = list(res.plug_in)
    out = dict(gcode=rows.gcode, codes_rows=rows.codes, V=rows.V,
               n_levels=np.array(rows.n_levels, np.int64), n_groups=np.array([rows.n_groups]),
               keys=np.array(keys), plug_in=np.array([res.plug_in[k] for k in keys]),
               bias=np.array([res.bias[k] for k in keys]),
               kss=np.array([res.kss[k] for k in keys]), P_ii=np.asarray(P_ii))
    mres = ke.kss_match(kp)
    out.update(match_plug_in=np.array([mres.plug_in[k] for k in keys]),
               match_bias=np.array([mres.bias[k] for k in keys]),
               match_kss=np.array([mres.kss[k] for k in keys]),
               match_sigma2=np.asarray(mres.diagnostics["sigma2"]),
               match_stayer=np.asarray(mres.diagnostics["stayer"]),
               match_worker=np.asarray(mres.diagnostics["worker"]),
               match_firm=np.asarray(mres.diagnostics["firm"]))
    print(res.summary())
    print(mres.summary())
    np.savez_compressed(Path(__file__).resolve().parent / "exact.npz", **out)


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else "/root/reference")

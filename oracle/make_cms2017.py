"""Writes mkfit_b200/geom/cms2017.npz: the CMS-2017 detector description and
the finding configuration of its ten iterations, exported from the
reference's own geometry plugin (Geoms/CMS-2017.cc, run in-process through
the oracle build in oracle/_ref). Iteration 0's arrays sit under their own
names; every iteration's steering, search windows and parameters are also
stacked under "it_<name>" (index = iteration).

    python oracle/make_cms2017.py

A build-time exporter beside the oracle it runs: the product package only
loads the committed file (mkfit_b200/geometry.py). The GPU path needs the
same layer table, layer plans, search-window and material-map numbers as
the reference to reproduce its results; exporting them from the running
plugin (instead of transcribing its source tables) keeps them identical.
tests/test_find_prep.py re-exports and compares.
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

from mkfit_b200.geometry import ITER_KEYS, N_ITERATIONS  # noqa: E402
from oracle.oracle import RefLib, cms2017_export  # noqa: E402

OUT = os.path.join(ROOT, "mkfit_b200", "geom", "cms2017.npz")


def export_all(ref):
    g = cms2017_export(ref, 0)
    per = [cms2017_export(ref, it) for it in range(N_ITERATIONS)]
    mp = max(e["plans"].shape[1] for e in per)
    for k in ITER_KEYS:
        rows = []
        for e in per:
            v = e[k]
            if k == "plans" and v.shape[1] < mp:
                v = np.pad(v, ((0, 0), (0, mp - v.shape[1])), constant_values=-1)
            rows.append(v)
        g["it_" + k] = np.stack(rows)
    return g


if __name__ == "__main__":
    g = export_all(RefLib())
    np.savez_compressed(OUT, **g)
    print("wrote", OUT)

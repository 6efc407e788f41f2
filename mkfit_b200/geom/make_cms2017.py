"""Writes mkfit_b200/geom/cms2017.npz: the CMS-2017 detector description and
iteration-0 finding configuration, exported from the reference's own
geometry plugin (Geoms/CMS-2017.cc, run in-process through the oracle
build in oracle/_ref).

    python mkfit_b200/geom/make_cms2017.py

The GPU path needs the same layer table, layer plans, search-window and
material-map numbers as the reference to reproduce its results; exporting
them from the running plugin (instead of transcribing its source tables)
keeps them identical. tests/test_geometry.py re-exports and compares.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from oracle.oracle import RefLib, cms2017_export  # noqa: E402

if __name__ == "__main__":
    g = cms2017_export(RefLib())
    np.savez_compressed(os.path.join(HERE, "cms2017.npz"), **g)
    print("wrote", os.path.join(HERE, "cms2017.npz"))

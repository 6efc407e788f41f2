"""Generates the golden fit fixtures from the reference's own CPU path.

    python tests/golden/make_golden.py

Runs the reference MkFitter fit (oracle/_ref, compiled from the reference
sources) on small seeded toy-MC inputs and stores inputs and outputs in
tests/golden/*.npz. The fixtures pin the oracle and the GPU path without
needing the reference build at test time.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from mkfit_b200 import synth  # noqa: E402
from oracle.oracle import RefLib  # noqa: E402


def make_fit(name, n, seed, pflags):
    ev = synth.gen_fit_event(n, seed=seed)
    ref = RefLib()
    par, err, chg, _ = ref.fit(ev.par, ev.err, ev.chg, ev.hit_pos, ev.hit_err, ev.rl_grid,
                               ev.xi_grid, pflags=pflags)
    # Material grids are regenerated from the radii by the tests (they are
    # 2 x 144 KB); only the radii are stored.
    np.savez_compressed(os.path.join(HERE, name), par=ev.par, err=ev.err, chg=ev.chg,
                        hit_pos=ev.hit_pos, hit_err=ev.hit_err, radii=ev.radii,
                        pflags=np.int32(pflags), seed=np.int64(seed), ref_par=par, ref_err=err,
                        ref_chg=chg, matriplex_width=np.int32(ref.width()))
    print("wrote", name)


if __name__ == "__main__":
    make_fit("fit_toy64_material.npz", 64, 1234, 2)
    make_fit("fit_toy64_nomaterial.npz", 64, 4321, 0)

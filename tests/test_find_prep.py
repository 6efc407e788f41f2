"""Host-side preparation of the finder against the reference (no GPU):
the per-layer hit bins and sorted ranks (LayerOfHits::SuckInHits) and the
seed partition + order (MkBuilder::import_seeds with partitionSeeds1) must
be bit-identical."""
import numpy as np
import pytest

from mkfit_b200 import synth
from mkfit_b200.finder import FindConfig, prepare_event_host
from oracle.oracle import ref_event_prep


@pytest.mark.parametrize("seed,n,noise", [(1, 800, 0.01), (7, 2500, 0.05), (11, 50, 0.0)])
def test_prep_matches_reference(reflib, seed, n, noise):
    ev = synth.gen_cms_event(n, seed=seed, noise_frac=noise)
    a = prepare_event_host(ev)
    b = ref_event_prep(reflib, ev)
    for k in ("bins", "srank", "seed_order", "seed_region"):
        np.testing.assert_array_equal(a[k], b[k], err_msg=k)


def test_prep_empty_layers_and_no_seeds(reflib):
    ev = synth.gen_cms_event(3, seed=5, noise_frac=0.0)
    a = prepare_event_host(ev)
    b = ref_event_prep(reflib, ev)
    np.testing.assert_array_equal(a["bins"], b["bins"])
    assert (np.diff(ev.layer_begin) == 0).any()


def test_geometry_matches_reference_export(reflib):
    """The committed geometry file equals what the reference plugin exports,
    for every iteration's configuration."""
    from mkfit_b200.geometry import ITER_KEYS, N_ITERATIONS, cms2017
    from oracle.oracle import cms2017_export
    for it in range(N_ITERATIONS):
        g = cms2017(it)
        e = cms2017_export(reflib, it)
        for k, v in e.items():
            got = g.arrays[k]
            if k == "plans":
                assert (got[:, v.shape[1]:] == -1).all()
                got = got[:, :v.shape[1]]
            np.testing.assert_array_equal(got, v, err_msg=f"iteration {it}: {k}")
        assert FindConfig(g).c.n_layers == 72
    # Iterations differ where the plugin makes them differ.
    assert not np.array_equal(cms2017(7).plans, cms2017(0).plans)
    assert cms2017(6).iter_params[0] != cms2017(0).iter_params[0]
    assert all(k in cms2017().arrays for k in ["it_" + k for k in ITER_KEYS])

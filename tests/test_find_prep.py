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
    """The committed geometry file equals what the reference plugin exports."""
    from mkfit_b200.geometry import cms2017
    from oracle.oracle import cms2017_export
    g = cms2017()
    e = cms2017_export(reflib)
    for k, v in e.items():
        np.testing.assert_array_equal(g.arrays[k], v, err_msg=k)
    assert FindConfig(g).c.n_layers == 72

"""Detector description and finding configuration (CMS-2017).

The numbers come from the reference's own geometry plugin, exported once
into geom/cms2017.npz by oracle/make_cms2017.py (layer table, per-region
layer plans, search-window parameters, iteration parameters, propagation
flags and the (z, r) material grid), for each of the ten CMS-2017
iterations (initialStep, highPtTripletStep, lowPtQuadStep,
lowPtTripletStep, detachedQuadStep, detachedTripletStep, mixedTripletStep,
pixelLessStep, tobTecStep, pixelPairStep).
"""
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))

# Column meaning of Geometry.layer_desc (one row per layer).
LAYER_FIELDS = ["is_barrel", "rin", "rout", "zmin", "zmax", "propagate_to", "q_bin",
                "has_hole", "hole_min", "hole_max", "is_pix", "is_stereo",
                "min_dphi", "max_dphi", "min_dq", "max_dq",
                "c_dp_sf", "c_dp_0", "c_dp_1", "c_dp_2",
                "c_dq_sf", "c_dq_0", "c_dq_1", "c_dq_2",
                "c_c2_sf", "c_c2_0", "c_c2_1", "c_c2_2",
                "layer_type", "is_seed", "subdet", "pad"]

# Region indices (TrackerInfo::EtaRegion).
REG_ENDCAP_NEG, REG_TRANSITION_NEG, REG_BARREL, REG_TRANSITION_POS, REG_ENDCAP_POS = range(5)


# Iteration-dependent arrays (stacked under "it_<name>" in the file).
ITER_KEYS = ("layer_desc", "plans", "plan_len", "pickup", "bkfit_last", "bksearch_pickup",
             "region_order", "iter_params", "bk_iter_params", "bk_flags")
N_ITERATIONS = 10


class Geometry:
    """The layer table with one iteration's configuration (IterationConfig
    of Config::ItrInfo[iteration])."""

    def __init__(self, path=None, iteration=0):
        d = np.load(path or os.path.join(HERE, "geom", "cms2017.npz"))
        self.arrays = {k: d[k] for k in d.files}
        self.iteration = int(iteration)
        if self.iteration:
            if not 0 <= self.iteration < N_ITERATIONS or "it_plans" not in self.arrays:
                raise ValueError(f"no configuration for iteration {iteration}")
            for k in ITER_KEYS:
                self.arrays[k] = self.arrays["it_" + k][self.iteration]
        self.layer_desc = self.arrays["layer_desc"].astype(np.float32)
        self.n_layers = self.layer_desc.shape[0]
        self.plans = self.arrays["plans"]
        self.plan_len = self.arrays["plan_len"]
        self.pickup = self.arrays["pickup"]
        self.bkfit_last = self.arrays["bkfit_last"]
        self.bksearch_pickup = self.arrays["bksearch_pickup"]
        self.region_order = self.arrays["region_order"]
        self.iter_params = self.arrays["iter_params"]
        # The backward search's IterationParams (m_backward_params) and
        # {m_backward_drop_seed_hits, m_backward_fit_min_hits}.
        self.bk_iter_params = self.arrays["bk_iter_params"]
        self.bk_flags = self.arrays["bk_flags"]
        self.flags = self.arrays["flags"]
        self.eta = self.arrays["eta"]
        self.rl = self.arrays["rl"]
        self.xi = self.arrays["xi"]

    def field(self, name):
        return self.layer_desc[:, LAYER_FIELDS.index(name)]

    def layer(self, i):
        return {k: float(self.layer_desc[i, j]) for j, k in enumerate(LAYER_FIELDS)}

    @property
    def n_regions(self):
        return self.plans.shape[0]

    def plan(self, region):
        return [int(x) for x in self.plans[region, :self.plan_len[region]]]


_cache = {}


def cms2017(iteration=0):
    """CMS-2017 with the configuration of `iteration` (0-9)."""
    if iteration not in _cache:
        _cache[iteration] = Geometry(iteration=iteration)
    return _cache[iteration]

"""The synthetic workloads the benchmark measures, defined once so that the
benchmark and the parity tests generate the same events.

No public dataset is involved: the reference benchmarks on CMSSW samples
that are not available, so seeded generators (synth.py) stand in with the
sizes and distributions of each workload.

* Batched finding: 64 CMS-2017 events, Poisson(3000) tracks clipped to
  [500, 12000], noise 1% of the signal hits times a per-layer ramp up to 20x
  (hit density varying ~20x across layers), maxCandsPerSeed 6, chi2 cut 30
  with the dynamic chi2 terms zeroed.
* Plain finding: one CMS-2017 event of 800 tracks, 1% noise.
* PU200-like finding: 16 events of 10,000 helices, pT log-uniform
  0.3-50 GeV, |eta| < 2.5, vertex sigma_z 5 cm, 5% noise raised with
  uniform pileup-like noise to a noise fraction of 2.16 (~600k hits per
  event).
* Fit: toy MC, 20,000 tracks per event, 10 barrel layers, material on.
* Differentiable fit: 50,000 toy tracks on a misaligned detector (r-phi and
  z offsets N(0, 20 um), material scale 1 +- 0.1).
"""
import numpy as np

from .dist import rank_seed

FIND_EVENTS = 64
FIND_MEAN_TRACKS = 3000
FIND_MIN_TRACKS = 500
FIND_MAX_TRACKS = 12000
FIND_NOISE = 0.01
FIND_DENSITY_RATIO = 20.0
FIND_MAX_CANDS = 6
FIND_CHI2_CUT = 30.0

PLAIN_TRACKS = 800

PU_EVENTS = 16
PU_TRACKS = 10000
PU_NOISE = 2.16

FIT_TRACKS_PER_EVENT = 20000
FIT_EVENTS = 16
FIT_LAYERS = 10

ADJ_TRACKS = 50000


def find_event_args(n_events=FIND_EVENTS, rank=0):
    """gen_cms_event arguments of the batched-finding events of `rank`."""
    from . import synth
    from .geometry import cms2017
    sizes = synth.batch_event_sizes(n_events, FIND_MEAN_TRACKS, FIND_MIN_TRACKS, FIND_MAX_TRACKS,
                                    seed=rank_seed(0xB200, rank))
    ramp = synth.density_ramp(cms2017().n_layers, FIND_DENSITY_RATIO)
    return [dict(n_tracks=int(n), seed=rank_seed(0xE000, rank) + i, noise_frac=FIND_NOISE,
                 noise_scale=ramp) for i, n in enumerate(sizes)]


def plain_event_args(rank=0):
    return dict(n_tracks=PLAIN_TRACKS, seed=0xC0DE + rank, noise_frac=0.01)


def pu_event_args(rank=0, n_events=PU_EVENTS):
    """gen_cms_event arguments of the PU200-like events of `rank`."""
    return [dict(n_tracks=PU_TRACKS, seed=0x9200 + 1000 * rank + i, pt_range=(0.3, 50.0),
                 eta_max=2.5, noise_frac=PU_NOISE) for i in range(n_events)]


def find_config_kwargs():
    """FindConfig arguments of the finding workloads."""
    return dict(max_cands=FIND_MAX_CANDS, chi2_cut=FIND_CHI2_CUT, zero_c2=True)


def fit_batch(n_events=FIT_EVENTS, rank=0):
    """The fit workload: n_events toy events of FIT_TRACKS_PER_EVENT tracks
    concatenated into one FitEvent."""
    from . import synth
    evs = [synth.gen_fit_event(FIT_TRACKS_PER_EVENT, seed=0xC0FFEE + 1000 * rank + e)
           for e in range(n_events)]

    def cat(k, ax):
        return np.ascontiguousarray(np.concatenate([getattr(e, k) for e in evs], axis=ax))
    return synth.FitEvent(par=cat("par", 1), err=cat("err", 1), chg=cat("chg", 0),
                          hit_pos=cat("hit_pos", 2), hit_err=cat("hit_err", 2),
                          rl_grid=evs[0].rl_grid, xi_grid=evs[0].xi_grid, radii=evs[0].radii)


def adjoint_event(rank=0, n_tracks=ADJ_TRACKS):
    """The differentiable-fit workload of `rank`."""
    from . import synth
    rng = np.random.default_rng(0xAD1 + rank)
    return synth.gen_fit_event(n_tracks, seed=0xAD10 + rank,
                               align_rphi=rng.normal(0, 0.002, FIT_LAYERS),
                               align_z=rng.normal(0, 0.002, FIT_LAYERS),
                               mat_scale=1 + rng.uniform(-0.1, 0.1, FIT_LAYERS))

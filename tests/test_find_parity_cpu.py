"""The mismatch classifier of the finding parity tests (tests/find_parity.py)
on fabricated result dicts (CPU, no GPU): ties and order swaps are
recognised, a planted real difference is left unexplained, and the
perturbation and task-cut checks are consulted only for what remains."""
import numpy as np

from tests import find_parity as fp

M = 3


def result(cands_per_seed):
    """A finding result with, per seed, a list of (hits, score, chi2,
    counters) candidates; hits as [(index, layer), ...]."""
    ns = len(cands_per_seed)
    o = dict(n_cands=np.zeros(ns, np.int32), ntot=np.zeros(ns * M, np.int32),
             hit_idx=np.zeros((ns * M, 64), np.int32), hit_lyr=np.zeros((ns * M, 64), np.int32),
             score=np.zeros(ns * M, np.float32), chi2=np.zeros(ns * M, np.float32),
             nfound=np.zeros(ns * M, np.int32), noverlap=np.zeros(ns * M, np.int32),
             ninside=np.zeros(ns * M, np.int32), ntail=np.zeros(ns * M, np.int32))
    for s, cands in enumerate(cands_per_seed):
        o["n_cands"][s] = len(cands)
        for c, (hits, score, chi2) in enumerate(cands):
            k = s * M + c
            o["ntot"][k] = len(hits)
            o["hit_idx"][k, :len(hits)] = [h for h, _ in hits]
            o["hit_lyr"][k, :len(hits)] = [lyr for _, lyr in hits]
            o["score"][k], o["chi2"][k] = score, chi2
            o["nfound"][k] = sum(h >= 0 for h, _ in hits)
    return o


A = [(1, 0), (2, 1), (3, 2)]
B = [(1, 0), (2, 1), (4, 2)]
PAIR = [(1, 0), (7, 4), (8, 4), (-1, 5)]
SWAPPED = [(1, 0), (8, 4), (7, 4), (-1, 5)]


def never(ev):
    raise AssertionError("not consulted")


def dummy_event():
    from mkfit_b200 import synth
    return synth.CmsEvent(hit_pos=np.ones((3, 4), np.float32), seed_par=np.ones((6, 1), np.float32))


def test_rank_tie_and_swap_tie_and_unexplained():
    gpu = result([[(A, 10.0, 5.0), (B, 10.0005, 5.0)],      # rank swapped within tolerance
                  [(SWAPPED, 20.0, 3.0)],                   # overlap order swapped, same score
                  [(A, 10.0, 5.0)]])                        # a real difference
    ref = result([[(B, 10.0005, 5.0), (A, 10.0, 5.0)],
                  [(PAIR, 20.0, 3.0)],
                  [(B, 14.0, 1.0)]])
    calls = []

    def same_as_ref(ev):
        calls.append(1)
        return ref

    cls = fp.classify(gpu, ref, dummy_event(), M, range(3), same_as_ref, lambda ev: gpu,
                      n_perturb=2, run_ref_partition=lambda ev, mode, k: ref)
    assert cls["best"]["tie"] == [0]
    assert cls["best"]["swap_tie"] == [1]
    assert cls["best"]["unexplained"] == [2]
    assert cls["any"]["unexplained"] == [2]
    assert calls  # the perturbation checks ran for the unexplained seed


def test_rank_gap_beyond_tolerance_is_not_a_tie():
    gpu = result([[(A, 10.0, 5.0), (B, 11.0, 5.0)]])
    ref = result([[(B, 11.0, 5.0), (A, 10.0, 5.0)]])
    kind, gap = fp.rank_tie(gpu, ref, 0, M)
    assert kind is None and gap == 1.0


def test_swap_tie_needs_equal_scores():
    gpu = result([[(SWAPPED, 20.0, 3.0)]])
    ref = result([[(PAIR, 26.0, 3.0)]])
    assert not fp.swap_tie(gpu, ref, 0, M, best_only=True)
    assert fp.canonical(PAIR) == fp.canonical(SWAPPED)


def test_reference_reproducing_the_gpu_explains():
    gpu = result([[(A, 10.0, 5.0)]])
    ref = result([[(B, 14.0, 1.0)]])
    cls = fp.classify(gpu, ref, dummy_event(), M, range(1), lambda ev: gpu, never, n_perturb=1,
                      run_ref_partition=None)
    assert cls["best"]["ref_flips"] == [0] and cls["best"]["unexplained"] == []
    cls = fp.classify(gpu, ref, dummy_event(), M, range(1), lambda ev: ref, never, n_perturb=0,
                      run_ref_partition=lambda ev, mode, k: gpu)
    assert cls["best"]["ref_partition"] == [0]


def test_perturbed_event_moves_by_one_ulp_at_most():
    from mkfit_b200 import synth
    ev = synth.gen_cms_event(40, seed=3, noise_frac=0.0)
    p = fp.perturbed(ev, np.random.default_rng(0))
    for k in ("hit_pos", "seed_par"):
        a, b = getattr(ev, k).astype(np.float32), getattr(p, k)
        ulps = np.abs(a.view(np.int32).astype(np.int64) - b.view(np.int32).astype(np.int64))
        assert ulps.max() <= 1 and (ulps == 1).any()

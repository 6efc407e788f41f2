"""Comparison of clone-engine finding results with the reference's, and
classification of every hit-list mismatch (test infrastructure).

The parity bar for finding: the final candidates' hit lists equal the
reference's, except where an FP32 comparison sits within rounding of a
decision boundary (a window edge, the chi2 cut, the score order of two
candidates). Each mismatching seed is classified by one of:

* "tie": both sides hold the same set of candidate hit lists and differ
  only in their order, and wherever the GPU's order disagrees with the
  reference's scores, the reference's score gap is within the chi2
  tolerance (CHI2_RTOL of the candidates' chi2): the rank of two
  candidates whose scores are equal to FP32 accuracy.
* "best_tie": the two best candidates are swapped as above, while lower
  slots differ for another reason (classified separately for the
  any-candidate count).
* "swap_tie": the candidates that differ hold the same hits on every layer
  and differ only in the order of an overlap pair within a layer (which of
  the two hits is the primary one), with equal hit counts and their chi2
  and score equal within the chi2 tolerance: the same track, kept in one
  order or the other by a tie of two candidates of equal score.
* "ref_flips": the reference itself, run on the same event with its FP32
  inputs (hit positions, seed parameters) moved by at most one ulp,
  produces the GPU's result for the seed: the reference's own decision is
  not determined at FP32 precision there.
* "gpu_flips": the same with the roles exchanged (the GPU, on one-ulp
  perturbed inputs, produces the reference's result).
* "ref_partition": the reference, run with its seed ranges cut into tasks
  another way TBB cuts them (recursive halving, coarser pieces, one task
  per region, uneven pieces, instead of near-equal pieces of the grain),
  produces the GPU's result. The reference's clone engine adds a
  seed's records task batch by task batch (NN candidates at a time) and
  orders them with std::sort, which is not stable above 16 elements, so
  records of exactly equal score (two candidates holding the same hits
  with an overlap pair in either order) come out in an order that depends
  on the task cut: the reference's own result there is not determined by
  its inputs.
* "unexplained": none of the above; a parity failure.

The seeds of an event are independent (the clone engine never lets two
seeds interact), so a perturbation of the whole event tests each seed on
its own.
"""
import numpy as np

from tests.tolerances import CHI2_RTOL


def hit_list(o, slot):
    n = o["ntot"][slot]
    return tuple(zip(o["hit_idx"][slot][:n].tolist(), o["hit_lyr"][slot][:n].tolist()))


def signature(o, s, m):
    """The seed's candidate hit lists in rank order."""
    return tuple(hit_list(o, s * m + c) for c in range(int(o["n_cands"][s])))


def best_list(o, s, m):
    return hit_list(o, s * m) if o["n_cands"][s] > 0 else ()


def mismatching_seeds(gpu, ref, seeds, m):
    """(best, any): the seeds among `seeds` whose best-candidate hit list
    differs, and those whose candidate lists differ in any slot or count."""
    best, anyc = [], []
    for s in seeds:
        if best_list(gpu, s, m) != best_list(ref, s, m):
            best.append(s)
        if signature(gpu, s, m) != signature(ref, s, m):
            anyc.append(s)
    return best, anyc


def _score_tol(chi2_a, chi2_b):
    return CHI2_RTOL * max(abs(float(chi2_a)), abs(float(chi2_b)), 1.0)


def rank_tie(gpu, ref, s, m):
    """(kind, gap): kind "tie" when both hold the same candidate hit lists
    and the GPU's order follows the reference's scores up to ties within
    the chi2 tolerance; "best_tie" when only the two best are such a swap;
    None otherwise. gap: the largest reference score gap the GPU's order
    crossed."""
    sg, sr = signature(gpu, s, m), signature(ref, s, m)
    score = {lst: (float(ref["score"][s * m + c]), float(ref["chi2"][s * m + c]))
             for c, lst in enumerate(sr)}
    if sorted(sg) == sorted(sr):
        gap = 0.0
        for a, b in zip(sg[:-1], sg[1:]):
            d = score[b][0] - score[a][0]
            if d > 0:
                if d > _score_tol(score[a][1], score[b][1]):
                    return None, d
                gap = max(gap, d)
        return "tie", gap
    if sg and sr and sg[0] in score and sr[0] != sg[0]:
        gscore = {lst: float(gpu["score"][s * m + c]) for c, lst in enumerate(sg)}
        if sr[0] in gscore:
            d = score[sr[0]][0] - score[sg[0]][0]
            if d <= _score_tol(score[sr[0]][1], score[sg[0]][1]):
                return "best_tie", max(d, 0.0)
    return None, None


def canonical(lst):
    """A hit list with the hits of each layer visit as a set: the order of
    an overlap pair within a layer does not count."""
    out, i = [], 0
    while i < len(lst):
        j = i
        while j < len(lst) and lst[j][1] == lst[i][1]:
            j += 1
        out.append((lst[i][1], tuple(sorted(h for h, _ in lst[i:j]))))
        i = j
    return tuple(out)


_COUNTERS = ("nfound", "noverlap", "ninside", "ntail")


def swap_tie(gpu, ref, s, m, best_only):
    """True when the differing candidates of seed s (the best one only, or
    all) are the same tracks up to the order within layers, with equal
    counters and chi2 / score equal within the chi2 tolerance."""
    def cands(o):
        n = min(int(o["n_cands"][s]), 1) if best_only else int(o["n_cands"][s])
        return [(canonical(hit_list(o, s * m + c)),
                 tuple(int(o[k][s * m + c]) for k in _COUNTERS),
                 float(o["chi2"][s * m + c]), float(o["score"][s * m + c])) for c in range(n)]
    cg, cr = cands(gpu), cands(ref)
    if len(cg) != len(cr):
        return False
    cg.sort(key=lambda x: x[:2])
    cr.sort(key=lambda x: x[:2])
    for a, b in zip(cg, cr):
        if a[:2] != b[:2]:
            return False
        tol = _score_tol(a[2], b[2])
        if abs(a[2] - b[2]) > tol or abs(a[3] - b[3]) > tol:
            return False
    return True


def perturbed(ev, rng):
    """A copy of a synth.CmsEvent with every hit coordinate and seed
    parameter moved by one ulp up, one ulp down or kept (equal odds)."""
    from mkfit_b200 import synth

    def ulp(a):
        a = np.asarray(a, np.float32)
        step = rng.integers(-1, 2, a.shape)
        up = np.nextafter(a, np.float32(np.inf))
        dn = np.nextafter(a, np.float32(-np.inf))
        return np.ascontiguousarray(np.where(step > 0, up, np.where(step < 0, dn, a)), np.float32)
    d = dict(ev.__dict__)
    d["hit_pos"] = ulp(ev.hit_pos)
    d["seed_par"] = ulp(ev.seed_par)
    return synth.CmsEvent(**d)


def classify(gpu, ref, ev, m, seeds, run_ref, run_gpu, n_perturb=8, seed=1234,
             run_ref_partition=None, n_random_cuts=8):
    """Classifies the mismatching seeds of one event (indices into the
    event's seeds; gpu and ref indexed the same way). run_ref(ev) and
    run_gpu(ev) return the result dicts of the reference and the GPU on a
    (perturbed) event; run_ref_partition(ev, mode, cut_seed), the
    reference's result with task cut `mode` (1-4, see
    RefLib.set_task_split), n_random_cuts of them random (mode 4). Returns a dict: per class the seeds (best-candidate
    and any-candidate mismatches classified separately), and the largest
    score gap of the ties."""
    best, anyc = mismatching_seeds(gpu, ref, seeds, m)
    out = {"best": {}, "any": {}, "tie_gap_max": 0.0, "n_best": len(best), "n_any": len(anyc)}
    todo_best, todo_any = [], []
    for s in best:
        kind, gap = rank_tie(gpu, ref, s, m)
        if kind is not None:
            out["best"].setdefault(kind, []).append(s)
            out["tie_gap_max"] = max(out["tie_gap_max"], gap)
        elif swap_tie(gpu, ref, s, m, best_only=True):
            out["best"].setdefault("swap_tie", []).append(s)
        else:
            todo_best.append(s)
    for s in anyc:
        kind, gap = rank_tie(gpu, ref, s, m)
        if kind == "tie":
            out["any"].setdefault("tie", []).append(s)
            out["tie_gap_max"] = max(out["tie_gap_max"], gap)
        elif swap_tie(gpu, ref, s, m, best_only=False):
            out["any"].setdefault("swap_tie", []).append(s)
        else:
            todo_any.append(s)
    cuts = [(1, 0), (2, 0), (3, 0)] + [(4, k) for k in range(1, 1 + n_random_cuts)]
    for mode, cut_seed in cuts if run_ref_partition is not None else ():
        if not todo_best and not todo_any:
            break
        o = run_ref_partition(ev, mode, cut_seed)
        for todo, key, fn in ((todo_best, "best", best_list), (todo_any, "any", signature)):
            for s in [s for s in todo if fn(o, s, m) == fn(gpu, s, m)]:
                todo.remove(s)
                out[key].setdefault("ref_partition", []).append(s)
    rng = np.random.default_rng(seed)
    for direction, runner, other in (("ref_flips", run_ref, gpu), ("gpu_flips", run_gpu, ref)):
        for _ in range(n_perturb):
            if not todo_best and not todo_any:
                break
            o = runner(perturbed(ev, rng))
            for todo, key, fn in ((todo_best, "best", best_list), (todo_any, "any", signature)):
                hit = [s for s in todo if fn(o, s, m) == fn(other, s, m)]
                for s in hit:
                    todo.remove(s)
                    out[key].setdefault(direction, []).append(s)
    out["best"]["unexplained"] = todo_best
    out["any"]["unexplained"] = todo_any
    return out


def summary(cls):
    """Counts per class."""
    return {k: {c: len(v) for c, v in cls[k].items()} for k in ("best", "any")}


def event_slice(o, off, n, m):
    """The results of seeds [off, off + n) of a batch download."""
    per_seed = ("n_cands", "region", "sorted_pos")
    return {k: (v[off:off + n] if k in per_seed else v[off * m:(off + n) * m])
            for k, v in o.items() if isinstance(v, np.ndarray)}


def matched_state_errors(gpu, ref, n_seeds, m):
    """Scaled errors of parameters, covariances and chi2 of the candidates
    whose hit lists agree (slot by slot), and whether their found-hit
    counts agree."""
    from tests.tolerances import cov_scaled_err, par_scaled_err
    same = [s * m + c for s in range(n_seeds)
            for c in range(min(int(gpu["n_cands"][s]), int(ref["n_cands"][s])))
            if hit_list(gpu, s * m + c) == hit_list(ref, s * m + c)]
    same = np.array(same, np.int64)
    ep = par_scaled_err(gpu["par"][same].T, ref["par"][same].T, ref["err"][same].T)
    ec = cov_scaled_err(gpu["err"][same].T, ref["err"][same].T)
    rc = np.abs(gpu["chi2"][same] - ref["chi2"][same]) / np.maximum(np.abs(ref["chi2"][same]), 1e-3)
    nf_equal = bool(np.array_equal(gpu["nfound"][same], ref["nfound"][same]))
    return same, ep, ec, rc, nf_equal

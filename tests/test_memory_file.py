"""memoryFile event files (mkfg_mf_*): parity with the reference's own
DataFile / Event::write_out / read_in (Event.cc:123-444) in both directions,
round trips with every extra section, and the error paths, on the CPU (the
reader and writer are host code); on the GPU, finding on an event read back
from a file equals finding on the original.

Bar: bit-exact — every field the format carries comes back unchanged."""
import os

import numpy as np
import pytest

from mkfit_b200 import capi, memory_file as mf, synth
from oracle.oracle import ref_mf_read, ref_mf_write

ALL = mf.SIM_TRACK_STATES | mf.SEEDS | mf.CMSSW_TRACKS | mf.HIT_ITER_MASKS | mf.BEAM_SPOT


def tracks_like(rng, n, n_layers=72, max_hits=12):
    """A track vector with every field set (holes and -9 hits included)."""
    nh = rng.integers(0, max_hits + 1, n)
    hb = np.concatenate([[0], np.cumsum(nh)]).astype(np.int32)
    tot = int(hb[-1])
    idx = rng.integers(-3, 5000, tot).astype(np.int32)
    idx[rng.random(tot) < 0.05] = -9
    return dict(par=rng.normal(size=(6, n)).astype(np.float32),
                err=rng.normal(size=(21, n)).astype(np.float32),
                charge=rng.choice([-1, 1], n).astype(np.int32),
                chi2=rng.random(n).astype(np.float32) * 50,
                score=rng.normal(size=n).astype(np.float32),
                status=rng.integers(0, 2 ** 31, n).astype(np.uint32),
                label=rng.integers(-1, 10 ** 6, n).astype(np.int32), hits_begin=hb,
                hit_index=idx, hit_layer=rng.integers(0, n_layers, tot).astype(np.int32))


def full_event(seed, n_tracks=150):
    """A synthetic CMS-2017 event with every section populated."""
    rng = np.random.default_rng(seed)
    ev = synth.gen_cms_event(n_tracks, seed=seed)
    d = mf.from_cms_event(ev)
    nh = ev.n_hits
    d["hit_masks"] = rng.integers(0, 2 ** 63, nh, dtype=np.uint64)
    d["sim"] = tracks_like(rng, 40)
    d["cmssw"] = tracks_like(rng, 25)
    d["seeds"]["chi2"] = rng.random(ev.n_seeds).astype(np.float32)
    d["seeds"]["status"] = rng.integers(0, 2 ** 31, ev.n_seeds).astype(np.uint32)
    d["sim_states"] = dict(par=rng.normal(size=(6, 30)).astype(np.float32),
                           err=rng.normal(size=(21, 30)).astype(np.float32),
                           charge=rng.choice([-1, 1], 30).astype(np.int32))
    d["beam_spot"] = rng.normal(size=8).astype(np.float32)
    return d


def assert_tracks_equal(a, b, what, nfound=True):
    n = len(b["charge"])
    assert len(a["charge"]) == n, what
    for k in ("par", "err", "charge", "chi2", "score", "status", "label", "hits_begin",
              "hit_index", "hit_layer") + (("nfound",) if nfound else ()):
        if k in b and k in a:
            np.testing.assert_array_equal(np.asarray(a[k]), np.asarray(b[k]), err_msg=f"{what}.{k}")


def assert_event_equal(a, b, sections):
    assert a["n_layers"] == b["n_layers"]
    for k in ("layer_begin", "hit_pos", "hit_err", "hit_mcid", "hit_packed", "mc_info"):
        np.testing.assert_array_equal(np.asarray(a[k]), np.asarray(b[k]), err_msg=k)
    if sections & mf.HIT_ITER_MASKS:
        np.testing.assert_array_equal(a["hit_masks"], b["hit_masks"])
    assert_tracks_equal(a["sim"], b["sim"], "sim")
    if sections & mf.SEEDS:
        assert_tracks_equal(a["seeds"], b["seeds"], "seeds")
    if sections & mf.CMSSW_TRACKS:
        assert_tracks_equal(a["cmssw"], b["cmssw"], "cmssw")
    if sections & mf.SIM_TRACK_STATES:
        for k in ("par", "err", "charge"):
            np.testing.assert_array_equal(a["sim_states"][k], b["sim_states"][k])
    if sections & mf.BEAM_SPOT:
        np.testing.assert_array_equal(a["beam_spot"], b["beam_spot"])


def with_nfound(t):
    """nFoundHits as Track::addHitIdx counts it (hits >= 0 or -9)."""
    t = dict(t)
    hb, idx = t["hits_begin"], t["hit_index"]
    t["nfound"] = np.array([int(((idx[a:b] >= 0) | (idx[a:b] == -9)).sum())
                            for a, b in zip(hb[:-1], hb[1:])], np.int32)
    return t


@pytest.mark.parametrize("sections", [ALL, mf.SEEDS, 0], ids=["all", "seeds", "none"])
def test_reference_written_file_reads_back(reflib, tmp_path, sections):
    events = [full_event(11), full_event(12, 60)]
    path = tmp_path / "ref.bin"
    assert ref_mf_write(reflib, path, events, sections) == 2
    hdr, got = mf.read(path)
    assert hdr == dict(format_version=6, n_layers=72, n_events=2, extra_sections=sections)
    for ev, g in zip(events, got):
        exp = dict(ev, sim=with_nfound(ev["sim"]), seeds=with_nfound(ev["seeds"]),
                   cmssw=with_nfound(ev["cmssw"]))
        assert_event_equal(g, exp, sections)
        assert (g["sim"]["valid"] == 1).all()


@pytest.mark.parametrize("sections", [ALL, mf.SEEDS | mf.BEAM_SPOT], ids=["all", "seeds+bs"])
def test_written_file_reads_in_reference(reflib, tmp_path, sections):
    events = [full_event(21), full_event(22, 80), full_event(23, 30)]
    path = tmp_path / "ours.bin"
    mf.write(path, events, n_layers=72, sections=sections)
    for i, ev in enumerate(events):
        ref = ref_mf_read(reflib, path, i)
        exp = dict(ev, sim=with_nfound(ev["sim"]), seeds=with_nfound(ev["seeds"]),
                   cmssw=with_nfound(ev["cmssw"]))
        assert_event_equal(ref, exp, sections)


def test_round_trip_and_finder_input(tmp_path):
    ev = synth.gen_cms_event(300, seed=31)
    path = tmp_path / "rt.bin"
    mf.write(path, [mf.from_cms_event(ev)], n_layers=ev.n_layers, sections=mf.SEEDS)
    with mf.Reader(path) as r:
        assert len(r) == 1
        back = mf.to_cms_event(r[0])
    for k in ("layer_begin", "hit_pos", "hit_err", "hit_detid", "seed_par", "seed_err", "seed_chg",
              "seed_nhits"):
        np.testing.assert_array_equal(getattr(back, k), getattr(ev, k), err_msg=k)
    for i in range(ev.n_seeds):
        n = ev.seed_nhits[i]
        np.testing.assert_array_equal(back.seed_hit_index[i, :n], ev.seed_hit_index[i, :n])
        np.testing.assert_array_equal(back.seed_hit_layer[i, :n], ev.seed_hit_layer[i, :n])
    # The charge-per-cm code (what the strip cut reads) survives; pixel hits
    # come back as -1.
    code = lambda c: np.where(c < 0, 0xff, np.where(c < 1620, 0,  # noqa: E731
                                                    np.minimum(0xff, ((c - 1620) >> 3) + 1)))
    np.testing.assert_array_equal(code(back.hit_cpcm.astype(np.int64)),
                                  code(ev.hit_cpcm.astype(np.int64)))


def test_errors(tmp_path):
    ev = mf.from_cms_event(synth.gen_cms_event(50, seed=41))
    good = tmp_path / "good.bin"
    mf.write(good, [ev, ev], n_layers=72, sections=mf.SEEDS)
    raw = good.read_bytes()
    with pytest.raises(capi.MkfgError, match="cannot open"):
        mf.read(tmp_path / "missing.bin")
    bad = tmp_path / "magic.bin"
    bad.write_bytes(b"\x00\x00\x00\x00" + raw[4:])
    with pytest.raises(capi.MkfgError, match="magic"):
        mf.read(bad)
    cut = tmp_path / "cut.bin"
    cut.write_bytes(raw[:len(raw) - 100])
    with pytest.raises(capi.MkfgError, match="2 events, 1 complete"):
        mf.read(cut)
    with mf.Reader(good) as r:
        with pytest.raises(capi.MkfgError, match="out of range"):
            r[2]
    with pytest.raises(capi.MkfgError, match="n_layers"):
        mf.write(tmp_path / "x.bin", [ev], n_layers=71)
    # A seed with more hits than the finder takes (16) is refused.
    ev17 = dict(ev)
    s = dict(ev["seeds"])
    s["hits_begin"] = np.concatenate([[0], np.full(len(s["charge"]), 17).cumsum()]).astype(np.int32)
    s["hit_index"] = np.zeros(17 * len(s["charge"]), np.int32)
    s["hit_layer"] = np.zeros(17 * len(s["charge"]), np.int32)
    ev17["seeds"] = s
    p17 = tmp_path / "seventeen.bin"
    mf.write(p17, [ev17], n_layers=72, sections=mf.SEEDS)
    with pytest.raises(capi.MkfgError, match="17 hits"):
        mf.to_cms_event(mf.read(p17)[1][0])
    assert os.path.getsize(good) == len(raw)


@pytest.mark.gpu
def test_finding_on_file_event_equals_original(gpu_ctx, tmp_path):
    """An event written to a memoryFile and read back gives the finder the
    same input: identical candidates."""
    from mkfit_b200.finder import FindConfig, Finder
    ev = synth.gen_cms_event(800, seed=51)
    path = tmp_path / "f.bin"
    mf.write(path, [mf.from_cms_event(ev)], n_layers=72, sections=mf.SEEDS)
    back = mf.to_cms_event(mf.read(path)[1][0])
    outs = []
    for e in (ev, back):
        f = Finder(gpu_ctx, FindConfig(max_cands=6))
        f.upload(e)
        f.run()
        outs.append(f.download(e.n_seeds))
    for k in outs[0]:
        np.testing.assert_array_equal(outs[0][k], outs[1][k], err_msg=k)

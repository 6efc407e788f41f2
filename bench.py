#!/usr/bin/env python3
"""Benchmark of the B200 Kalman-filter tracking hot path.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Prints one JSON line on rank 0. Headline: combinatorial track finding
(clone engine, CMS-2017 geometry) in events built per second for the
batched form -- a batch of 64 synthetic events of uneven size found by one
graph-captured launch sequence -- beside the plain one-event form and the
reference CPU build. A "step" is one pass over the batch with the inputs
resident in HBM. Secondary: the Kalman fit in tracks fit per second.

Under torchrun (N > 1) each rank finds its own batch (weak scaling, no
data-path collective); the step time is the max over ranks.

--impl reference times the reference's own CPU implementation (the
trackreco/mkFit sources compiled in oracle/_ref) on the host cores with all
threads, several events in flight, on a bounded sample of the same events.
"""
import argparse
import json
import multiprocessing as mp
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402

from mkfit_b200 import workloads as W  # noqa: E402

# Workloads (mkfit_b200/workloads.py): batched finding, 64 CMS-2017 events,
# Poisson(3000) tracks clipped to [500, 12000], noise 1% x a per-layer ramp
# up to 20x; the plain one-event form on 800 tracks; the fit; the
# differentiable fit; PU200-like finding.
FIND_EVENTS = W.FIND_EVENTS
FIND_MEAN_TRACKS = W.FIND_MEAN_TRACKS
FIND_NOISE = W.FIND_NOISE
FIND_DENSITY_RATIO = W.FIND_DENSITY_RATIO
FIND_MAX_CANDS = W.FIND_MAX_CANDS
FIND_CHI2_CUT = W.FIND_CHI2_CUT
# Batches in flight in the end-to-end measurement (one context each).
E2E_IN_FLIGHT = 3
PLAIN_TRACKS = W.PLAIN_TRACKS
# Algorithmic FLOPs per unit of work (counted from the generated products
# and the restated arithmetic): propagation of a
# candidate to a layer + hit selection; propagation to a hit + chi2; the
# update step (propagation to the hit + Kalman update).
FLOP_LAYER_PROP = 1000
FLOP_HIT_CHI2 = 950
FLOP_UPDATE = 1150
# Algorithmic HBM bytes per unit: the candidate state read (27 floats +
# charge) and the propagated state written (27 floats); the hit (9 floats)
# and the propagated state read per pair; state in + hit + state out per
# update.
BYTES_LAYER_PROP = 112 + 108
BYTES_HIT_CHI2 = 36 + 108
BYTES_UPDATE = 112 + 36 + 112
# Kernels per layer-plan step in the graph form.
KERNELS_PER_LAYER_STEP = 5
FIT_TRACKS_PER_EVENT = W.FIT_TRACKS_PER_EVENT
FIT_EVENTS = W.FIT_EVENTS
FIT_LAYERS = W.FIT_LAYERS
FLOP_FIT_TRACK_LAYER = 1130
ADJ_TRACKS = W.ADJ_TRACKS
PU_EVENTS = W.PU_EVENTS
PU_TRACKS = W.PU_TRACKS
PU_NOISE = W.PU_NOISE
# Events of each workload the CPU baselines find (the whole batched-finding
# step; half of the PU200-like step).
CPU_FIND_EVENTS = FIND_EVENTS
CPU_PU_EVENTS = 8
CPU_FIT_TRACKS = 320_000   # the whole fit step (16 x 20000)
CPU_ADJ_TRACKS = 5_000


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=20)
    p.add_argument("--warmup", type=int, default=5)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--events", type=int, default=FIND_EVENTS)
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-e2e", action="store_true")
    p.add_argument("--no-fit", action="store_true")
    p.add_argument("--no-pu", action="store_true")
    p.add_argument("--no-autotune", action="store_true",
                   help="keep the default launch configuration (fixed launch counts for profiling)")
    p.add_argument("--step-profile", action="store_true",
                   help="print per layer-plan step work and launch times to stderr")
    return p.parse_args()


# ----------------------------------------------------------------------------- inputs
def find_event_args(n_events, rank):
    return W.find_event_args(n_events, rank)


def generate(args_list):
    """Generates events in a spawn process pool (started before CUDA)."""
    from mkfit_b200 import synth
    n = min(len(args_list), os.cpu_count() or 1)
    if n <= 1:
        return [synth.gen_cms_event(**a) for a in args_list]
    with mp.get_context("spawn").Pool(n) as pool:
        return pool.map(synth.gen_cms_event_args, args_list)


def make_fit_batch(n_events, rank):
    return W.fit_batch(n_events, rank)


# ----------------------------------------------------------------------------- utilities
class ClockSampler:
    """nvidia-smi clock / throttle sampling during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index):
        self.dev = device_index
        self.proc = None
        self.tmp = None

    def start(self):
        try:
            self.tmp = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.dev), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=self.tmp, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.tmp.flush()
        rows = [ln.strip().split(",") for ln in open(self.tmp.name) if ln.strip()]
        os.unlink(self.tmp.name)
        sm, smax, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            try:
                sm.append(float(r[1]))
                smax = max(smax, float(r[2]))
                for nm, v in zip(names, r[5:9]):
                    if v.strip().lower() == "active":
                        reasons.add(nm)
            except (ValueError, IndexError):
                continue
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm)}


def load_measured_peaks():
    try:
        return json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "source": "fallback"}


def fp32_peak(ctx):
    import ctypes
    v = ctypes.c_double(0)
    rc = ctx.lib.mkfg_probe_fp32_peak(ctx.handle, 4000, ctypes.byref(v))
    return v.value if rc == 0 else None


def print_step_profile(prof):
    """Per layer-plan step: work counters and launch times (us), to stderr."""
    keys = list(prof)
    print("step " + " ".join(k[:12].rjust(12) for k in keys), file=sys.stderr)
    for i in range(len(prof[keys[0]])):
        cells = [(f"{int(prof[k][i]):12d}" if prof[k].dtype.kind == "i" else
                  f"{1000 * float(prof[k][i]):12.1f}") for k in keys]
        print(f"{i + 1:4d} " + " ".join(cells), file=sys.stderr)


def timed_events(stream, fn, steps):
    """Per-step CUDA-event timing on `stream`; returns per-step ms."""
    import torch
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(steps)]
    for s in range(steps):
        starts[s].record(stream)
        fn()
        ends[s].record(stream)
    torch.cuda.synchronize()
    return [a.elapsed_time(b) for a, b in zip(starts, ends)]


# Algorithmic bytes of the clone step (k_clone): per candidate of a cloned
# seed, its record-presence mask, hole/extra code, extra stop node and 11
# counters read (56 B); per record present, the 16-byte record; per new
# candidate, the parent's 27-float state read and written to the new slot
# and 9 counters written (108 + 108 + 36 B); per Kalman update listed, its
# hit-on-track node (12 B) and update-list entry (8 B).
CLONE_BYTES_PER_CAND = 56
CLONE_BYTES_PER_RECORD = 16
CLONE_BYTES_PER_NEW_CAND = 252
CLONE_BYTES_PER_UPDATE = 20


# DRAM traffic of k_clone per new candidate written, from one ncu capture
# (dram__bytes_read.sum + dram__bytes_write.sum over the 42 clone launches
# of one replay of an 8-event batch of the same workload, 1.866 GB for
# 3,427,364 new candidates; profiles/clone_kernel_cms2017_batch.md).
CLONE_DRAM_BYTES_PER_NEW_CAND = 544.4


def clone_traffic_per_launch(work):
    if CLONE_DRAM_BYTES_PER_NEW_CAND is None:
        return None
    return CLONE_DRAM_BYTES_PER_NEW_CAND * work["new_cands"] / work["steps"]


def kernel_rooflines(work, kt, fp32_peak_tf, peaks):
    """Rooflines of the finding kernels from one timed replay (kt: ms per
    step per kernel) and the step's work counters: the dominant kernel by
    time against its bound, and the dominant FP32 kernel against the FP32
    peak."""
    steps = work["steps"]
    hbm = peaks.get("hbm_gbs")
    fp = {"propagate": (work["active_cands"], FLOP_LAYER_PROP, BYTES_LAYER_PROP),
          "chi2": (work["hit_pairs"], FLOP_HIT_CHI2, BYTES_HIT_CHI2),
          "update": (work["updates"], FLOP_UPDATE, BYTES_UPDATE)}
    clone_bytes = (CLONE_BYTES_PER_CAND * work["active_cands"] +
                   CLONE_BYTES_PER_RECORD * work["records"] +
                   CLONE_BYTES_PER_NEW_CAND * work["new_cands"] +
                   CLONE_BYTES_PER_UPDATE * work["updates"])
    f_dom = max(fp, key=lambda k: kt[k])
    units, f_unit, b_unit = fp[f_dom]
    f_tf = units * f_unit / (kt[f_dom] * 1e-3) / 1e12
    fp32 = {"kernel": f"k_{f_dom}", "bound": "fp32", "achieved": f_tf, "peak": fp32_peak_tf,
            "unit": "TFLOP/s", "frac": f_tf / fp32_peak_tf if fp32_peak_tf else None,
            "peak_source": "measured FP32 FMA probe (mkfg_probe_fp32_peak), same run (of measured)",
            "per_launch_ms": kt[f_dom] / steps, "units_per_step": units, "flop_per_unit": f_unit,
            "bytes_per_unit": b_unit,
            "hbm_achieved_gbs": units * b_unit / (kt[f_dom] * 1e-3) / 1e9}
    by_time = max((k for k in kt if k not in ("reset", "merge")), key=lambda k: kt[k])
    if by_time == "clone":
        gbs = clone_bytes / (kt["clone"] * 1e-3) / 1e9
        dom = {"kernel": "k_clone", "bound": "hbm", "achieved": gbs, "peak": hbm, "unit": "GB/s",
               "frac": gbs / hbm if hbm else None,
               "peak_source": ("fallback HBM copy bandwidth, no MEASURED_PEAKS.json on this "
                               "machine (of fallback)" if peaks.get("source") == "fallback"
                               else "MEASURED_PEAKS.json hbm_gbs (of measured)"),
               "per_launch_ms": kt["clone"] / steps,
               "algorithmic_bytes_per_launch": clone_bytes / steps,
               "bytes_model": {"per_candidate": CLONE_BYTES_PER_CAND,
                               "per_record": CLONE_BYTES_PER_RECORD,
                               "per_new_candidate": CLONE_BYTES_PER_NEW_CAND,
                               "per_update": CLONE_BYTES_PER_UPDATE},
               "traffic": clone_traffic_per_launch(work),
               "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum of k_clone "
                                 "per new candidate, scaled to this launch "
                                 "(profiles/clone_kernel_cms2017_batch.md)"}
    else:
        dom = dict(fp32)
    return {"dominant": dom, "fp32": fp32, "fp32_peak": fp32_peak_tf}


def find_config_line(events, world):
    """The `config` of the batched-finding line, shared by both arms."""
    n_seeds = sum(e.n_seeds for e in events)
    n_hits = sum(e.n_hits for e in events)
    return {
        "workload": (f"batched clone-engine finding: {len(events)} CMS-2017 events per step, "
                     f"Poisson({FIND_MEAN_TRACKS}) tracks clipped to [500, 12000], "
                     f"noise {FIND_NOISE:.0%} x per-layer ramp up to {FIND_DENSITY_RATIO:.0f}x, "
                     f"maxCandsPerSeed {FIND_MAX_CANDS}, chi2 cut {FIND_CHI2_CUT:.0f}"),
        "events_per_step": len(events), "seeds_per_step": n_seeds, "hits_per_step": n_hits,
        "l2": "inputs + candidate state ~%.0f MB per step (L2 126 MB); no flush" % (
            (n_hits * 40 + n_seeds * 8 * 37 * 4 * 3) / 1e6),
        "parallelism": f"dp{world} (independent event batches per GPU)",
    }


# ----------------------------------------------------------------------------- ours
def run_ours(args):
    rank = int(os.environ.get("RANK", "0"))
    # Inputs first (process pool before any CUDA call).
    events = generate(find_event_args(args.events, rank))
    from mkfit_b200 import synth
    plain_ev = synth.gen_cms_event(**W.plain_event_args(rank))
    fit_batch = None if args.no_fit else make_fit_batch(FIT_EVENTS, rank)
    # One sample for all ranks: the differentiable fit splits its tracks.
    adj_ev = None if args.no_fit else adjoint_event(0)
    pu_events = None if args.no_pu else generate(pu_event_args(rank))

    import torch
    from mkfit_b200 import Context
    from mkfit_b200.finder import FindConfig, Finder
    from mkfit_b200 import dist as mdist
    world, rank, local = mdist.setup()
    torch.cuda.set_device(local)
    ctx = Context(local)
    stream = ctx.torch_stream()
    finder = Finder(ctx, FindConfig(max_cands=FIND_MAX_CANDS, chi2_cut=FIND_CHI2_CUT, zero_c2=True))
    n_events = len(events)
    n_seeds = sum(e.n_seeds for e in events)
    n_hits = sum(e.n_hits for e in events)

    # Plain form: one event per upload, eager launch sequence per run.
    finder.upload(plain_ev)
    for _ in range(2):
        finder.run()
    ctx.synchronize()
    plain_cfg1_ms = statistics.median(timed_events(stream, finder.run, max(3, args.steps // 2)))
    # Plain form on one event of the batch (same event size class).
    finder.upload(events[0])
    finder.run()
    ctx.synchronize()
    plain_b_ms = statistics.median(timed_events(stream, finder.run, max(3, args.steps // 2)))

    # Batched form: all events resident, one graph replay per step, in the
    # launch configuration the autotuner picks on this batch (untimed).
    finder.upload_batch(events)
    tuning = finder.graph_tuning() if args.no_autotune else finder.autotune_graph(reps=2)
    for _ in range(args.warmup):
        finder.run_graph()
    ctx.synchronize()
    # Work counters of the step: one eager run of the same sequence, which
    # also counts the clone step's records and new candidates.
    finder.run()
    work = finder.work()
    peak = fp32_peak(ctx)
    sampler = ClockSampler(local)
    mdist.barrier(world)
    torch.cuda.synchronize()
    sampler.start()
    t_load = time.perf_counter() + 1.5  # let the sampler see the clocks under load
    while time.perf_counter() < t_load:
        for _ in range(4):
            finder.run_graph()
        ctx.synchronize()
    step_ms = timed_events(stream, finder.run_graph, args.steps)
    clocks = sampler.stop()
    mdist.barrier(world)
    total_ms = sum(step_ms)
    total_ms_max = mdist.max_over_ranks(total_ms, world)
    value = mdist.aggregate_rate(n_events, args.steps, total_ms_max * 1e-3, world)
    ms_step = total_ms / args.steps

    flops = (work["active_cands"] * FLOP_LAYER_PROP + work["hit_pairs"] * FLOP_HIT_CHI2 +
             work["updates"] * FLOP_UPDATE)
    achieved_tf = flops / (ms_step * 1e-3) / 1e12

    # Per-kernel device times: one replay of the same step as the plain
    # launch sequence with a CUDA event after every kernel (outside the
    # timed region), for the rooflines of the kernels.
    kt = finder.run_timed()
    kt_total = sum(kt.values())
    rl = kernel_rooflines(work, kt, peak, load_measured_peaks())
    # The best candidate per seed of this step, for the comparison with the
    # reference CPU run on the same events.
    gpu_best = finder.download_best(n_seeds)
    if args.step_profile and rank == 0:
        print_step_profile(finder.step_profile())

    # End to end through the C ABI from host buffers: upload (seed partition
    # and initial candidates on the host, H2D, device hit-index build), run,
    # download (export + D2H into the caller's arrays, reused across steps).
    e2e = None
    if not args.no_e2e:
        e_steps = max(4, args.steps // 2)
        # One batch at a time: upload, run, download.
        ts = []
        out = None
        for _ in range(e_steps + 1):
            t0 = time.perf_counter()
            finder.upload_batch(events)
            finder.run_graph()
            out = finder.download_best(n_seeds, out)
            ts.append(time.perf_counter() - t0)
        t_serial = statistics.median(ts[1:])
        # E2E_IN_FLIGHT batches in flight on as many contexts (the reference
        # keeps events in flight the same way): the host work of a batch's
        # upload overlaps the device runs of the earlier ones. Every step
        # still copies its inputs from host memory and its results back to
        # host memory; a context's results are read before it takes the
        # next batch.
        extra = [Context(local) for _ in range(E2E_IN_FLIGHT - 1)]
        ring = [finder] + [Finder(c, FindConfig(max_cands=FIND_MAX_CANDS, chi2_cut=FIND_CHI2_CUT,
                                                zero_c2=True)) for c in extra]
        outs = [out] + [None] * (E2E_IN_FLIGHT - 1)

        def pipelined(steps):
            pending = []
            for i in range(steps):
                k = i % E2E_IN_FLIGHT
                if len(pending) == E2E_IN_FLIGHT:
                    j = pending.pop(0)
                    outs[j] = ring[j].download_best(n_seeds, outs[j])
                ring[k].upload_batch(events)
                ring[k].run_graph()
                pending.append(k)
            for j in pending:
                outs[j] = ring[j].download_best(n_seeds, outs[j])

        pipelined(E2E_IN_FLIGHT)
        t0 = time.perf_counter()
        pipelined(e_steps)
        t = (time.perf_counter() - t0) / e_steps
        # Every context found the same candidates.
        for o in outs[1:]:
            for k in ("n_cands", "hit_idx", "hit_lyr", "par"):
                if not np.array_equal(outs[0][k], o[k]):
                    raise RuntimeError(f"pipelined contexts disagree on {k}")
        for c in extra:
            c.close()
        h2d = sum(e.hit_pos.nbytes + e.hit_err.nbytes + e.hit_detid.nbytes + e.hit_cpcm.nbytes +
                  e.seed_par.nbytes + e.seed_err.nbytes + e.seed_chg.nbytes for e in events)
        d2h = sum(v.nbytes for v in out.values())
        e2e = {"value": n_events / t, "unit": "events/s", "h2d_bytes_per_step": int(h2d),
               "d2h_bytes_per_step": int(d2h), "ms_per_step": t * 1e3,
               "batches_in_flight": E2E_IN_FLIGHT,
               "one_batch_at_a_time": {"value": n_events / t_serial, "ms_per_step": t_serial * 1e3},
               "entry": "mkfg_find_upload_batch + mkfg_find_run_graph + mkfg_find_download_best "
                        "(seed partition and initial candidates on the host, copies, device "
                        "hit-index build, export of the best candidate per seed as "
                        "MkBuilder::export_best_comb_cands into reused host arrays); "
                        f"{E2E_IN_FLIGHT} contexts take batches in turn"}

    stages = None if args.no_e2e else run_iteration_stages(ctx, stream, finder, events, n_seeds)
    fit = None if fit_batch is None else run_fit(ctx, stream, fit_batch, args)
    adjoint = None if adj_ev is None else run_adjoint(ctx, stream, adj_ev, args, world, rank)
    pu200, pu_best = (None, None) if pu_events is None else run_pu200(ctx, stream, finder,
                                                                      pu_events, args)

    peaks = load_measured_peaks()
    line = {
        "metric": "events built/s",
        "value": value,
        "unit": "events/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": total_ms_max / args.steps,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32",
        "data": "synthetic (seeded, mkfit_b200.synth.gen_cms_event on the CMS-2017 layer table)",
        "config": find_config_line(events, world),
        "rates": {"seeds_per_s": n_seeds * world / (total_ms_max / args.steps * 1e-3),
                  "candidate_hit_evals_per_s": work["hit_pairs"] * world /
                                               (total_ms_max / args.steps * 1e-3),
                  "note": "the batched-finding workload in two more units: seeds found and "
                          "(candidate, hit) chi2 evaluations per second, whole job"},
        "plain_form": {
            "cms_800_tracks": {"events_per_launch_sequence": 1, "value": 1e3 / plain_cfg1_ms,
                               "unit": "events/s", "ms_per_event": plain_cfg1_ms,
                               "seeds": plain_ev.n_seeds},
            "batch_event0": {"value": 1e3 / plain_b_ms, "unit": "events/s",
                             "ms_per_event": plain_b_ms, "seeds": events[0].n_seeds},
            "batched_over_plain": (value / world) / (1e3 / plain_b_ms),
        },
        "roofline": dict(rl["dominant"], kernel_ms_per_step=dict(kt),
                         kernel_share={k: v / kt_total for k, v in kt.items()},
                         fp32_kernel=rl["fp32"],
                         step={"scope": "whole finding step (all kernels of the graph)",
                               "achieved_tflops": achieved_tf,
                               "fp32_frac": achieved_tf / rl["fp32_peak"] if rl["fp32_peak"] else None,
                               "flop_per_step": flops, "work_per_step": work}),
        "e2e": e2e,
        "gpu_launches": args.steps * (2 + KERNELS_PER_LAYER_STEP * work["steps"]),
        "gpu_launches_note": (f"kernels in the timed region: one CUDA graph replay per step = reset + "
                              f"{KERNELS_PER_LAYER_STEP} kernels x {work['steps']} layer steps + merge"),
        "clocks": clocks,
        "fit": fit,
        "adjoint": adjoint,
        "pu200": pu200,
        "iteration_stages": stages,
        "autotune": dict(tuning, knobs="grid of the propagate, chi2, clone and update kernels as a "
                                       "multiple of their resident blocks; bin staging",
                         note="mkfg_find_autotune_graph on the step's batch before timing; "
                              "ms_before / ms_after: summed per-launch device times of one run"),
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        if fit is not None:
            fit["cpu_baseline"] = cpu_baseline_fit(fit_batch, min(CPU_FIT_TRACKS, fit_batch.n))
        if adjoint is not None:
            adjoint["cpu_baseline"] = cpu_baseline_adjoint(adj_ev, CPU_ADJ_TRACKS)
        line["cpu_baseline"] = cpu_baseline_find(events, gpu_best)
        if pu_events is not None:
            line["cpu_baseline"]["pu200"] = cpu_baseline_find(pu_events, pu_best,
                                                              n_sample=CPU_PU_EVENTS)
    if rank == 0:
        emit(line)
    ctx.close()
    mdist.teardown(world)


def run_fit(ctx, stream, batch, args):
    from mkfit_b200 import FitBuffers
    ctx.set_material(batch.rl_grid, batch.xi_grid)
    dev = FitBuffers.upload(batch)
    out = FitBuffers.outputs(batch.n)
    for _ in range(args.warmup):
        ctx.fit_device(dev, out)
    ctx.synchronize()
    ms = timed_events(stream, lambda: ctx.fit_device(dev, out), args.steps)
    t = sum(ms) / len(ms)
    flops = batch.n * FIT_LAYERS * FLOP_FIT_TRACK_LAYER
    return {"metric": "tracks fit/s", "value": batch.n / (t * 1e-3), "unit": "tracks/s",
            "ms_per_step": t, "tracks_per_step": batch.n,
            "workload": f"toy-MC Kalman fit, {FIT_EVENTS} events x {FIT_TRACKS_PER_EVENT} tracks x "
                        f"{FIT_LAYERS} barrel layers, material on, one launch",
            "achieved_tflops": flops / (t * 1e-3) / 1e12}


def cpu_baseline_fit(batch, n_sample):
    """The reference's MkFitter fitting loop (runFittingTestPlex:
    InputTracksForFit + FitTracksWithInterSlurp + OutputFittedTracks over
    NN-track chunks, mkFit/fittestMPlex.cc:65-100) on all host threads,
    best of 3, on the first n_sample tracks of the step."""
    from oracle.oracle import RefLib
    ref = RefLib()
    threads = os.cpu_count()
    ref.set_threads(threads)
    sub = batch.tracks(0, n_sample)
    _, _, _, secs = ref.fit(sub.par, sub.err, sub.chg, sub.hit_pos, sub.hit_err, sub.rl_grid,
                            sub.xi_grid, pflags=2, repeat=3)
    return {"value": n_sample / secs, "unit": "tracks/s", "cores": threads, "kind": "reference",
            "sample": (f"{n_sample} of the step's {batch.n} tracks, reference MkFitter loop over "
                       f"NN-track chunks on a {threads}-thread pool, AVX2 Matriplex (NN=8), "
                       f"material on, best of 3")}


def cpu_baseline_adjoint(ev, n_sample):
    """The FP64 restatement of the forward fit + adjoint (the oracle's port:
    the reference has no gradient) on one host thread, on the first
    n_sample tracks."""
    from oracle.oracle import adj_f64_grad
    sub = ev.tracks(0, n_sample)
    theta = np.zeros((sub.hit_pos.shape[0], 3))
    theta[:, 2] = 1.0
    t0 = time.perf_counter()
    adj_f64_grad(sub.par, sub.err, sub.chg, sub.hit_pos, sub.hit_err, theta, sub.rl_grid,
                 sub.xi_grid, material=True)
    secs = time.perf_counter() - t0
    return {"value": n_sample / secs, "unit": "tracks/s", "cores": 1, "kind": "port",
            "sample": (f"{n_sample} of the step's {ev.n} tracks, FP64 forward fit + adjoint of "
                       "the 30 layer parameters (oracle/adjoint_f64.cc), one thread, wall clock")}


def adjoint_event(rank):
    return W.adjoint_event(rank)


def run_adjoint(ctx, stream, ev, args, world=1, rank=0):
    """Forward (summed chi2, checkpoints) + adjoint (30-parameter gradient)
    through the C ABI, timed per step with CUDA events. With N ranks the
    tracks are split into one share per rank and each step ends with one
    all-reduce of the 31 sums (strong scaling: the sample is the same)."""
    import ctypes
    import torch
    from mkfit_b200 import capi
    from mkfit_b200 import dist as mdist
    from mkfit_b200.align import AlignedFit, _bind
    begin, end = mdist.track_share(ev.n, world, rank)
    fit = AlignedFit(ctx, ev.tracks(begin, end), material=True)
    lib = ctx.lib
    _bind(lib)
    th = fit.nominal()
    n = end - begin
    dev = th.device
    ckpt = torch.empty((fit.n_steps, 27, n), dtype=torch.float32, device=dev)
    sums = torch.empty(1 + 3 * fit.n_steps, dtype=torch.float64, device=dev)
    total, grad = sums[:1], sums[1:]
    gout = torch.ones((), dtype=torch.float32, device=dev)
    a = fit._args(th, ckpt, total)
    torch.cuda.synchronize()

    def step():
        capi.check(lib.mkfg_align_chi2_forward(ctx.handle, ctypes.byref(a)))
        capi.check(lib.mkfg_align_chi2_backward(ctx.handle, ctypes.byref(a), gout.data_ptr(),
                                                grad.data_ptr()))
        if world > 1:
            import torch.distributed as tdist
            with torch.cuda.stream(stream):
                tdist.all_reduce(sums)
    for _ in range(args.warmup):
        step()
    ctx.synchronize()
    mdist.barrier(world)
    ms = timed_events(stream, step, args.steps)
    t = mdist.max_over_ranks(sum(ms) / len(ms), world)
    g = grad.cpu().numpy()
    return {"metric": "tracks/s (forward + adjoint)", "value": ev.n / (t * 1e-3),
            "unit": "tracks/s", "ms_per_step": t, "tracks_per_step": ev.n,
            "scaling": "strong" if world > 1 else None,
            "workload": (f"differentiable fit: {ev.n} toy tracks x {FIT_LAYERS} barrel layers, "
                         "misaligned detector (offsets N(0, 20 um), material scale 1 +- 0.1), "
                         "summed chi2 and its gradient w.r.t. 30 layer parameters at nominal, "
                         "FP32 forward with per-layer checkpoints + FP32 adjoint, 2 launches"
                         + (f", tracks split over {world} ranks + one all-reduce of the 31 "
                            "sums per step" if world > 1 else "")),
            "chi2_sum": float(total.item()),
            "grad_norm": float(np.linalg.norm(g)),
            "accuracy": "gradient vs FP64 central finite differences: tests/test_adjoint_gpu.py"}


def pu_event_args(rank):
    return W.pu_event_args(rank)


def run_iteration_stages(ctx, stream, finder, events, n_seeds):
    """Time of the steps of run_OneIteration around the finding, on the
    same batch (median of 5; CUDA events on the context stream around each
    call, so host-side setup inside the call counts): the backward fit, the
    backward search, the output selection, a quality filter, and the seed
    cleaning of the
    batch's seeds with 20% near-duplicates added (host-buffer call, wall
    clock)."""
    import torch
    from mkfit_b200 import synth
    from mkfit_b200.seed_clean import clean_seeds

    def dev_ms(fn, pre=None, reps=5):
        out = []
        for _ in range(reps):
            finder.run_graph()
            if pre is not None:
                pre()
            torch.cuda.synchronize()
            a = torch.cuda.Event(enable_timing=True)
            b = torch.cuda.Event(enable_timing=True)
            a.record(stream)
            fn()
            b.record(stream)
            b.synchronize()
            out.append(a.elapsed_time(b))
        return statistics.median(out)

    from mkfit_b200.finder import QF_N_LAYERS
    bk = dev_ms(finder.backward_fit)
    bs = dev_ms(finder.backward_search, pre=finder.backward_fit)
    sel = dev_ms(lambda: finder.select(n_seeds))
    # The costliest quality filter (a walk of every best candidate's hit
    # chain), verdicts copied to the host.
    qf = dev_ms(lambda: finder.filter(n_seeds, QF_N_LAYERS, beam_spot=(0.0, 0.0)))
    sds = [synth.with_duplicate_seeds(e, frac=0.2, seed=i) for i, e in enumerate(events)]
    begin = np.cumsum([0] + [len(d["chg"]) for d in sds]).astype(np.int32)
    cat = lambda k, ax: np.concatenate([d[k] for d in sds], axis=ax)  # noqa: E731
    args = (begin, cat("par", 1), cat("chg", 0), cat("nhits", 0), cat("hit_layer", 0),
            cat("hit_index", 0))
    clean_seeds(ctx, *args)
    ts = []
    for _ in range(5):
        t0 = time.perf_counter()
        keep = clean_seeds(ctx, *args)[0]
        ts.append(time.perf_counter() - t0)
    return {"events": len(events), "seeds": int(n_seeds),
            "backward_fit_ms": bk, "backward_search_ms": bs, "select_ms": sel,
            "quality_filter_ms": qf,
            "seed_cleaning": {"seeds_in": int(begin[-1]), "kept": int(keep.sum()),
                              "ms_host_buffers": statistics.median(ts) * 1e3},
            "note": "stream times of the calls around the finding of the bench batch; seed "
                    "cleaning on the batch's seeds plus 20% near-duplicates, through "
                    "mkfg_clean_seeds with host buffers (wall clock)"}


def run_pu200(ctx, stream, finder, events, args):
    finder.upload_batch(events)
    for _ in range(max(args.warmup, 1)):
        finder.run_graph()
    ctx.synchronize()
    ms = timed_events(stream, finder.run_graph, max(3, args.steps // 2))
    t = sum(ms) / len(ms)
    work = finder.work()
    best = finder.download_best(sum(e.n_seeds for e in events))
    flops = (work["active_cands"] * FLOP_LAYER_PROP + work["hit_pairs"] * FLOP_HIT_CHI2 +
             work["updates"] * FLOP_UPDATE)
    return {"metric": "events built/s", "value": len(events) / (t * 1e-3), "unit": "events/s",
            "ms_per_step": t, "events_per_step": len(events),
            "seeds_per_step": sum(e.n_seeds for e in events),
            "hits_per_event": float(np.mean([e.n_hits for e in events])),
            "workload": (f"PU200-like finding: {len(events)} events x {PU_TRACKS} helices "
                         "(pT log-uniform 0.3-50 GeV, |eta| < 2.5, vertex sigma_z 5 cm), 5% noise "
                         f"plus uniform pileup-like noise (noise fraction {PU_NOISE} in total) to "
                         "reach ~600k hits per event, one CUDA-graph replay per step"),
            "achieved_tflops": flops / (t * 1e-3) / 1e12, "work_per_step": work}, best


def best_mismatch(ref, gpu_best):
    """Seeds whose best-candidate hit list (or candidate presence) differs
    between the reference (ref_find_batch summaries) and the GPU
    (download_best), over the seeds both hold."""
    n = min(len(ref["n_cands"]), len(gpu_best["n_cands"]))
    bad = 0
    for s in range(n):
        rc, gc = int(ref["n_cands"][s]) > 0, int(gpu_best["n_cands"][s]) > 0
        if rc != gc:
            bad += 1
            continue
        if not rc:
            continue
        k = int(ref["ntot"][s])
        if (k != int(gpu_best["ntot"][s]) or
                not np.array_equal(ref["hit_idx"][s, :k], gpu_best["hit_idx"][s, :k]) or
                not np.array_equal(ref["hit_lyr"][s, :k], gpu_best["hit_lyr"][s, :k])):
            bad += 1
    return bad, n


def cpu_baseline_find(events, gpu_best=None, n_sample=None):
    """The reference CPU clone engine on the host cores (all threads, events
    in flight), best of 3, on the first n_sample events (all by default);
    with gpu_best (the GPU's best candidate per seed of the same events),
    also the best-candidate hit-list mismatch rate against the GPU."""
    from oracle.oracle import RefLib, ref_find_batch
    ref = RefLib()
    threads = os.cpu_count()
    ref.set_threads(threads)
    sample = events if n_sample is None else events[:n_sample]
    t0 = time.perf_counter()
    o = ref_find_batch(ref, sample, max_cands=FIND_MAX_CANDS, chi2_cut=FIND_CHI2_CUT, repeat=3)
    wall = time.perf_counter() - t0
    line = {"value": len(sample) / o["seconds"], "unit": "events/s", "cores": threads,
            "kind": "reference",
            "sample": (f"{len(sample)} of the step's {len(events)} events "
                       f"({sum(e.n_seeds for e in sample)} seeds), "
                       f"reference find_tracks_load_seeds + FindTracksCloneEngine, events in flight "
                       f"on a {threads}-thread pool, AVX2 Matriplex (NN=8), best of 3, "
                       f"{wall:.1f} s wall incl. hit-index build")}
    if gpu_best is not None:
        bad, n = best_mismatch(o, gpu_best)
        line["mismatch"] = {"best_candidate_hit_list": bad / max(n, 1), "seeds_differing": bad,
                            "seeds_compared": n,
                            "note": "GPU batched form vs the reference on the same events; every "
                                    "mismatch class is checked by tests/test_find_measured_gpu.py"}
    return line


# ----------------------------------------------------------------------------- reference
def run_reference(args):
    """The reference's own CPU clone engine (the unmodified sources compiled
    in oracle/_ref) on the host cores with all threads and every event of
    the batch in flight, on the same events and configuration as the GPU
    arm; each step finds the whole batch."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from oracle.oracle import RefLib, have_ref, ref_find_batch
    if not have_ref():
        emit({"impl": "reference", "unavailable":
              "reference CPU build oracle/_ref missing (built by __graft_entry__.build "
              "from the reference sources)"})
        return
    events = generate(find_event_args(args.events, 0))
    ref = RefLib()
    threads = os.cpu_count()
    ref.set_threads(threads)
    for _ in range(max(1, min(args.warmup, 2))):
        ref_find_batch(ref, events, max_cands=FIND_MAX_CANDS, chi2_cut=FIND_CHI2_CUT)
    secs = []
    for _ in range(args.steps):
        o = ref_find_batch(ref, events, max_cands=FIND_MAX_CANDS, chi2_cut=FIND_CHI2_CUT)
        secs.append(o["seconds"])
    total = sum(secs)
    value = len(events) * args.steps / total
    line = {
        "impl": "reference",
        "metric": "events built/s", "value": value, "unit": "events/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": total / args.steps * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded, mkfit_b200.synth.gen_cms_event on the CMS-2017 layer table)",
        # The same config object as this workload's line from the GPU arm at
        # this world size (rank 0's batch); the reference runs it on rank 0's
        # host cores alone.
        "config": find_config_line(events, world),
        "cpu_baseline": {"value": value, "unit": "events/s", "cores": threads, "kind": "reference",
                         "sample": f"all {len(events)} events of the step, in flight on a "
                                   f"{threads}-thread pool, reference find_tracks_load_seeds + "
                                   "MkBuilder::FindTracksCloneEngine timed region, AVX2 "
                                   "Matriplex (NN=8)"},
        "e2e": {"value": value, "unit": "events/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
        "gpu_launches": 0,
    }
    emit(line)


def spawn_ranks(args):
    """`--gpus N` without a launcher: starts N ranks of this script (one per
    GPU) with torch.distributed.run on 127.0.0.1 and returns their exit
    status; rank 0 prints the line."""
    import socket
    with socket.socket(socket.AF_INET, socket.SOCK_STREAM) as sk:
        sk.bind(("127.0.0.1", 0))
        port = sk.getsockname()[1]
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1",
           f"--nproc-per-node={args.gpus}", "--master-addr", "127.0.0.1",
           f"--master-port={port}", os.path.abspath(__file__)] + sys.argv[1:]
    return subprocess.call(cmd)


_RESULT_FD = None


def emit(line):
    """Prints the result line on the process's real standard output."""
    data = (json.dumps(line) + "\n").encode()
    if _RESULT_FD is None:
        sys.stdout.write(data.decode())
        sys.stdout.flush()
    else:
        os.write(_RESULT_FD, data)


def keep_stdout_for_result():
    """Sends everything else written to file descriptor 1 (the reference
    library's own printf lines among it) to standard error, so that
    standard output carries the one JSON line alone."""
    global _RESULT_FD
    sys.stdout.flush()
    _RESULT_FD = os.dup(1)
    os.dup2(2, 1)


def main():
    args = parse()
    if args.gpus > 1 and "WORLD_SIZE" not in os.environ:
        sys.exit(spawn_ranks(args))
    keep_stdout_for_result()
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()

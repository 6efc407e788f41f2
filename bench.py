#!/usr/bin/env python3
"""Benchmark of the B200 Kalman-filter hot path.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

One JSON line on rank 0. A "step" is one pass of the hot path over one batch
of seeded synthetic input resident in HBM (see DESIGN.md for the workload
definition). For N > 1 the script runs under torchrun, one process per GPU,
each rank processing its own batch (weak scaling, no data-path collective);
the step time is the max over ranks of the device time.

--impl reference runs the reference's own CPU implementation (the
trackreco/mkFit sources compiled in oracle/_ref) on the host cores with all
available threads, on the same workload and metric; rank 0 only.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402

FIT_TRACKS_PER_EVENT = 20000
FIT_LAYERS = 10
FIT_EVENTS_PER_STEP = 64
# Algorithmic work of one barrel fit step (track-layer): FLOPs from the
# generated similarity/update products plus the hand-counted propagation,
# material and update arithmetic, bytes moved from/to HBM.
FLOP_PER_TRACK_LAYER = 1130
BYTES_PER_TRACK_FIXED = 2 * (27 * 4 + 4)   # state in + state out
BYTES_PER_TRACK_LAYER = 9 * 4 + 4          # hit (pos 3 + err 6) + hit index


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=50)
    p.add_argument("--warmup", type=int, default=5)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-e2e", action="store_true")
    p.add_argument("--events", type=int, default=FIT_EVENTS_PER_STEP,
                   help="events of 20k tracks per step (profiling uses fewer)")
    return p.parse_args()


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


# --------------------------------------------------------------------------- helpers
def dist_setup(args):
    import torch
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    return world, rank, local


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(x, world):
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def make_fit_batch(n_events, rank):
    """One batch of n_events toy-MC events (20k tracks x 10 layers each),
    concatenated: the batched form fits all of them in one launch."""
    from mkfit_b200 import synth
    evs = [synth.gen_fit_event(FIT_TRACKS_PER_EVENT, seed=0xC0FFEE + 1000 * rank + e)
           for e in range(n_events)]
    cat = lambda k, ax: np.ascontiguousarray(np.concatenate([getattr(e, k) for e in evs], axis=ax))
    return synth.FitEvent(par=cat("par", 1), err=cat("err", 1), chg=cat("chg", 0),
                          hit_pos=cat("hit_pos", 2), hit_err=cat("hit_err", 2),
                          rl_grid=evs[0].rl_grid, xi_grid=evs[0].xi_grid, radii=evs[0].radii)


def cpu_reference_fit_rate(seconds_target=10.0, threads=None):
    """Reference CPU MkFitter fit (oracle/_ref) on the host cores: tracks/s
    on a bounded sample of the toy-MC workload."""
    from oracle.oracle import RefLib
    from mkfit_b200 import synth
    ref = RefLib()
    threads = threads or os.cpu_count()
    ref.set_threads(threads)
    ev = synth.gen_fit_event(FIT_TRACKS_PER_EVENT * 4, seed=0xBEEF)
    _, _, _, t1 = ref.fit(ev.par, ev.err, ev.chg, ev.hit_pos, ev.hit_err, ev.rl_grid, ev.xi_grid,
                          pflags=2, repeat=1)
    reps = max(1, int(seconds_target / max(t1, 1e-4) / max(threads, 1)))
    t0 = time.perf_counter()
    _, _, _, best = ref.fit(ev.par, ev.err, ev.chg, ev.hit_pos, ev.hit_err, ev.rl_grid,
                            ev.xi_grid, pflags=2, repeat=reps)
    wall = time.perf_counter() - t0
    return ev.n / best, threads, reps, ev.n, wall


# --------------------------------------------------------------------------- ours
def run_ours(args):
    import torch
    from mkfit_b200 import Context, FitBuffers

    world, rank, local = dist_setup(args)
    torch.cuda.set_device(local)
    ctx = Context(local)
    stream = ctx.torch_stream()

    n_events = args.events
    batch = make_fit_batch(n_events, rank)
    ctx.set_material(batch.rl_grid, batch.xi_grid)
    dev = FitBuffers.upload(batch)
    out = FitBuffers.outputs(batch.n)
    n_tracks = batch.n

    # Device-resident timing: one batched launch per step.
    for _ in range(args.warmup):
        ctx.fit_device(dev, out)
    ctx.synchronize()
    peak = ctypes_probe(ctx)
    sampler = ClockSampler(local)
    barrier(world)
    torch.cuda.synchronize()
    sampler.start()
    # Untimed back-to-back launches for ~1.5 s so that the clock sampler
    # (100 ms period) observes the clocks the timed steps run at.
    t_load = time.perf_counter() + 1.5
    while time.perf_counter() < t_load:
        for _ in range(10):
            ctx.fit_device(dev, out)
        ctx.synchronize()
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    for s in range(args.steps):
        starts[s].record(stream)
        ctx.fit_device(dev, out)
        ends[s].record(stream)
    ctx.synchronize()
    torch.cuda.synchronize()
    clocks = sampler.stop()
    barrier(world)
    step_ms = [a.elapsed_time(b) for a, b in zip(starts, ends)]
    total_ms = sum(step_ms)
    total_ms_max = max_over_ranks(total_ms, world)
    value = world * n_tracks * args.steps / (total_ms_max * 1e-3)

    # Plain form: one launch per event (20k tracks), same data.
    plain_ms = time_plain_fit(ctx, stream, dev, out, n_events, FIT_TRACKS_PER_EVENT,
                              max(2, args.steps // 4))

    # End to end through the host-buffer C-ABI entry (pinned host memory,
    # H2D + kernel + D2H inside the timed region).
    e2e = None if args.no_e2e else time_e2e_fit(ctx, batch, max(2, args.steps // 4), args.warmup)

    kernel_ms = total_ms / args.steps
    flops = n_tracks * FIT_LAYERS * FLOP_PER_TRACK_LAYER
    bytes_alg = n_tracks * (BYTES_PER_TRACK_FIXED + FIT_LAYERS * BYTES_PER_TRACK_LAYER)
    achieved_tf = flops / (kernel_ms * 1e-3) / 1e12
    achieved_gbs = bytes_alg / (kernel_ms * 1e-3) / 1e9
    peaks = load_measured_peaks()
    hbm_peak = peaks.get("hbm_gbs")

    line = {
        "metric": "tracks fit/s",
        "value": value,
        "unit": "tracks/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": total_ms_max / args.steps,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32",
        "data": "synthetic (seeded toy MC, mkfit_b200.synth.gen_fit_event)",
        "config": {
            "workload": (f"Kalman fit, toy MC: {n_events} events x "
                         f"{FIT_TRACKS_PER_EVENT} tracks x {FIT_LAYERS} barrel layers per step, "
                         "one batched launch (the reference's MkFitter fit)"),
            "tracks_per_step": n_tracks,
            "layers": FIT_LAYERS,
            "pflags": "apply_material",
            "l2": "inputs larger than L2 (%.0f MB per step)" % (bytes_alg / 1e6),
            "parallelism": f"dp{world} (independent events per GPU)",
        },
        "plain_form": {"events_per_launch": 1, "tracks_per_launch": FIT_TRACKS_PER_EVENT,
                       "value": n_tracks / (plain_ms * 1e-3), "unit": "tracks/s",
                       "ms_per_step": plain_ms,
                       "launches_per_step": n_events},
        "roofline": {
            "bound": "fp32",
            "kernel": "fit_kernel<false>",
            "achieved": achieved_tf,
            "peak": peak,
            "unit": "TFLOP/s",
            "frac": achieved_tf / peak if peak else None,
            "peak_source": "measured FP32 FMA probe (mkfg_probe_fp32_peak), same run",
            "flop_per_launch": flops,
            "traffic": None,
            "hbm": {"achieved": achieved_gbs, "peak": hbm_peak, "unit": "GB/s",
                    "frac": achieved_gbs / hbm_peak if hbm_peak else None,
                    "bytes_per_launch": bytes_alg, "peak_source": "MEASURED_PEAKS.json hbm_gbs"},
        },
        "e2e": e2e,
        "gpu_launches": args.steps,
        "clocks": clocks,
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        rate, threads, reps, sample_n, wall = cpu_reference_fit_rate()
        line["cpu_baseline"] = {
            "value": rate, "unit": "tracks/s", "cores": threads, "kind": "reference",
            "sample": (f"reference MkFitter fit (oracle/_ref, AVX2 Matriplex) of {sample_n} "
                       f"toy-MC tracks x {FIT_LAYERS} layers, best of {reps} repeats, "
                       f"{wall:.1f} s wall")}
    if rank == 0:
        print(json.dumps(line), flush=True)
    ctx.close()
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


def ctypes_probe(ctx):
    import ctypes
    v = ctypes.c_double(0)
    rc = ctx.lib.mkfg_probe_fp32_peak(ctx.handle, 20000, ctypes.byref(v))
    return v.value if rc == 0 else None


def time_plain_fit(ctx, stream, dev, out, n_events, per_event, steps):
    """One launch per event: the plain drop-in form of the fit."""
    import torch
    from mkfit_b200 import capi
    t0 = torch.cuda.Event(enable_timing=True)
    t1 = torch.cuda.Event(enable_timing=True)
    ms = []
    for s in range(steps + 1):
        t0.record(stream)
        for e in range(n_events):
            ctx_fit_slice(ctx, dev, out, e * per_event, per_event)
        t1.record(stream)
        ctx.synchronize()
        if s > 0:
            ms.append(t0.elapsed_time(t1))
    return sum(ms) / len(ms)


def ctx_fit_slice(ctx, dev, out, begin, count):
    """Fit tracks [begin, begin+count) of the device batch (views with the
    batch stride)."""
    import ctypes
    from mkfit_b200 import capi
    n = dev["n"]
    a = capi.MkfgFitArgs()
    f4 = 4
    a.in_ = capi.MkfgTracks(dev["par"].data_ptr() + begin * f4, dev["err"].data_ptr() + begin * f4,
                            dev["chg"].data_ptr() + begin * f4, count, n)
    a.out = capi.MkfgTracks(out["par"].data_ptr() + begin * f4, out["err"].data_ptr() + begin * f4,
                            out["chg"].data_ptr() + begin * f4, count, n)
    a.hits = capi.MkfgHits(dev["hit_pos"].data_ptr(), dev["hit_err"].data_ptr(),
                           dev["layer_begin"].data_ptr(), dev["n_layers"], dev["n_hits"])
    a.hot_index = dev["hot"].data_ptr() + begin * f4
    a.hot_stride = n
    a.n_steps = dev["n_layers"]
    hl = np.arange(dev["n_layers"], dtype=np.int32)
    a._hl = hl
    a.hit_layer = hl.ctypes.data
    a.endcap_mask = 0
    a.pflags = capi.PF_MATERIAL
    a.out_chi2 = None
    capi.check(ctx.lib.mkfg_fit(ctx.handle, ctypes.byref(a)))


def time_e2e_fit(ctx, batch, steps, warmup):
    import torch
    n = batch.n
    nl = batch.hit_pos.shape[0]
    pin = lambda a: torch.from_numpy(np.ascontiguousarray(a)).pin_memory().numpy()
    par, err, chg = pin(batch.par), pin(batch.err), pin(batch.chg)
    hp = pin(batch.hit_pos.transpose(1, 0, 2).reshape(3, nl * n))
    he = pin(batch.hit_err.transpose(1, 0, 2).reshape(6, nl * n))
    out = dict(par=pin(np.zeros((6, n), np.float32)), err=pin(np.zeros((21, n), np.float32)),
               chg=pin(np.zeros(n, np.int32)), chi2=pin(np.zeros(n, np.float32)))
    for _ in range(max(1, warmup // 2)):
        ctx.fit_host(par, err, chg, hp, he, out=out)
    ts = []
    for _ in range(steps):
        t0 = time.perf_counter()
        ctx.fit_host(par, err, chg, hp, he, out=out)
        ts.append(time.perf_counter() - t0)
    t = sum(ts) / len(ts)
    h2d = par.nbytes + err.nbytes + chg.nbytes + hp.nbytes + he.nbytes + 4 * (nl + 1) + 4 * nl * n
    d2h = out["par"].nbytes + out["err"].nbytes + out["chg"].nbytes
    return {"value": n / t, "unit": "tracks/s", "h2d_bytes_per_step": int(h2d),
            "d2h_bytes_per_step": int(d2h), "ms_per_step": t * 1e3,
            "entry": "mkfg_fit_host (pinned host buffers; H2D + fit + D2H + sync)"}


def load_measured_peaks():
    try:
        return json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "source": "fallback"}


# --------------------------------------------------------------------------- reference
def run_reference(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from oracle.oracle import RefLib, have_ref
    from mkfit_b200 import synth
    if not have_ref():
        print(json.dumps({"impl": "reference", "unavailable":
                          "reference CPU build oracle/_ref missing (built by __graft_entry__.build "
                          "from /root/reference)"}))
        return
    ref = RefLib()
    threads = os.cpu_count()
    ref.set_threads(threads)
    # A step is a bounded sample of the same workload: 4 events of 20k tracks.
    n_ev = 4
    ev = make_fit_batch(n_ev, 0)
    for _ in range(args.warmup):
        ref.fit(ev.par, ev.err, ev.chg, ev.hit_pos, ev.hit_err, ev.rl_grid, ev.xi_grid, pflags=2)
    times = []
    for _ in range(args.steps):
        _, _, _, t = ref.fit(ev.par, ev.err, ev.chg, ev.hit_pos, ev.hit_err, ev.rl_grid,
                             ev.xi_grid, pflags=2)
        times.append(t)
    total = sum(times)
    value = ev.n * args.steps / total
    line = {
        "impl": "reference",
        "metric": "tracks fit/s", "value": value, "unit": "tracks/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": total / args.steps * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded toy MC, mkfit_b200.synth.gen_fit_event)",
        "config": {"workload": (f"Kalman fit, toy MC: {n_ev} events x {FIT_TRACKS_PER_EVENT} "
                                f"tracks x {FIT_LAYERS} barrel layers per step (bounded sample "
                                f"of the GPU arm's {FIT_EVENTS_PER_STEP}-event step)"),
                   "tracks_per_step": ev.n, "layers": FIT_LAYERS, "pflags": "apply_material"},
        "cpu_baseline": {"value": value, "unit": "tracks/s", "cores": threads, "kind": "reference",
                         "sample": f"{ev.n} tracks per step, reference MkFitter fit, TBB-shim "
                                   f"thread pool of {threads} threads, AVX2 Matriplex (NN=8)"},
        "e2e": {"value": value, "unit": "tracks/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
        "gpu_launches": 0,
    }
    print(json.dumps(line), flush=True)


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()

"""Multi-GPU plumbing: one process per GPU.

Finding: each rank finds its own batch of events (events are independent,
as the reference's events in flight are: mkFit/mkFit.cc:308-425), no
data-path collective. Only the timing uses a collective: the step time is
the maximum over ranks, and the throughput counts the events of all ranks.

Differentiable fit: the tracks are split into contiguous shares, one per
rank; each rank computes its share's summed chi2 and the gradient with
respect to the per-layer parameters, and one all-reduce (sum) of those
1 + 3 * n_layers numbers gives every rank the whole-sample result.

Backend "nccl" on GPUs; "gloo" (CPU tensors) for the host-side tests.
"""
import datetime
import os


def setup(backend=None, timeout_s=120):
    """Initialises the process group from the torchrun environment (RANK,
    LOCAL_RANK, WORLD_SIZE, MASTER_ADDR/PORT). Returns (world, rank, local)."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import torch
        import torch.distributed as dist
        backend = backend or "nccl"
        kw = dict(timeout=datetime.timedelta(seconds=timeout_s))
        if backend == "nccl":
            torch.cuda.set_device(local)
            kw["device_id"] = torch.device("cuda", local)
        dist.init_process_group(backend, **kw)
    return world, rank, local


def _device():
    import torch
    import torch.distributed as dist
    return torch.device("cuda") if dist.get_backend() == "nccl" else torch.device("cpu")


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(x, world):
    """The maximum of a per-rank float (a timed region) over all ranks."""
    if world == 1:
        return float(x)
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(x)], dtype=torch.float64, device=_device())
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(x, world):
    if world == 1:
        return float(x)
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(x)], dtype=torch.float64, device=_device())
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def track_share(n, world, rank):
    """The contiguous share [begin, end) of n tracks that `rank` takes:
    shares differ by at most one track."""
    base, extra = divmod(int(n), int(world))
    begin = rank * base + min(rank, extra)
    return begin, begin + base + (1 if rank < extra else 0)


def allreduce_sum(values, world):
    """Element-wise sum over ranks of a float64 vector (one all-reduce);
    returns a numpy array."""
    import numpy as np
    v = np.asarray(values, np.float64).ravel()
    if world == 1:
        return v.copy()
    import torch
    import torch.distributed as dist
    t = torch.from_numpy(v.copy()).to(_device())
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return t.cpu().numpy()


def rank_seed(base, rank):
    """Seed of a rank's synthetic workload: distinct per rank, fixed per
    (base, rank) so a rank's events are reproducible."""
    return int(base) + 1000 * int(rank)


def aggregate_rate(units_per_rank_step, steps, max_seconds, world):
    """Whole-job throughput: the units all ranks processed over the slowest
    rank's timed region (weak scaling: every rank holds the same amount)."""
    return world * units_per_rank_step * steps / max_seconds


def teardown(world):
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()

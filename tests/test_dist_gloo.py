"""Multi-process plumbing of the batched finder (mkfit_b200.dist), run as
two gloo ranks on the CPU: each rank gets its own reproducible event batch,
the step time is the maximum over ranks, the throughput counts the events
of both ranks, and the ranks shut down cleanly."""
import os
import socket
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket(socket.AF_INET, socket.SOCK_STREAM) as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    sys.path.insert(0, ROOT)
    os.environ.update(RANK=str(rank), LOCAL_RANK=str(rank), WORLD_SIZE=str(world),
                      MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    try:
        import bench
        from mkfit_b200 import dist
        w, r, _ = dist.setup(backend="gloo", timeout_s=60)
        args = bench.find_event_args(3, r)
        again = bench.find_event_args(3, r)
        m = dist.max_over_ranks(r + 1.5, w)
        n_all = dist.sum_over_ranks(len(args), w)
        dist.barrier(w)
        rate = dist.aggregate_rate(len(args), 10, m, w)
        same = [(a["seed"], a["n_tracks"]) for a in args] == [(a["seed"], a["n_tracks"]) for a in again]
        q.put((r, [a["seed"] for a in args], [a["n_tracks"] for a in args], same, m, n_all, rate))
        dist.teardown(w)
    except Exception as e:  # reported to the parent, which fails the test
        q.put((rank, "error", repr(e)))


def test_two_gloo_ranks():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    try:
        res = sorted(q.get(timeout=180) for _ in procs)
    finally:
        for p in procs:
            p.join(timeout=60)
            if p.is_alive():
                p.kill()
    for r in res:
        assert r[1] != "error", r
    (r0, seeds0, n0, rep0, m0, all0, rate0), (r1, seeds1, n1, rep1, m1, all1, rate1) = res
    assert (r0, r1) == (0, 1)
    assert rep0 and rep1                      # a rank's batch is reproducible
    assert not set(seeds0) & set(seeds1)      # ranks find different events
    assert m0 == m1 == 2.5                    # slowest rank's time
    assert all0 == all1 == 6
    assert rate0 == rate1 == pytest.approx(2 * 3 * 10 / 2.5)
    assert all(p.exitcode == 0 for p in procs)


def _grad_worker(rank, world, port, q):
    sys.path.insert(0, ROOT)
    os.environ.update(RANK=str(rank), LOCAL_RANK=str(rank), WORLD_SIZE=str(world),
                      MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    try:
        import numpy as np
        from mkfit_b200 import dist, workloads
        from mkfit_b200.align import distributed_chi2_grad
        from oracle.oracle import adj_f64_grad
        w, r, _ = dist.setup(backend="gloo", timeout_s=60)
        ev = workloads.adjoint_event(0, n_tracks=301)
        theta = np.zeros((ev.hit_pos.shape[0], 3))
        theta[:, 2] = 1.0

        def grad_fn(e, th):
            return adj_f64_grad(e.par, e.err, e.chg, e.hit_pos, e.hit_err, th, e.rl_grid,
                                e.xi_grid)
        c2, g = distributed_chi2_grad(None, ev, theta, w, r, grad_fn=grad_fn)
        q.put((r, c2, g.tolist(), dist.track_share(ev.n, w, r)))
        dist.teardown(w)
    except Exception as e:  # reported to the parent, which fails the test
        q.put((rank, "error", repr(e)))


def test_split_adjoint_sums_to_one_rank_result():
    """The differentiable fit's track split: two gloo ranks each take half of
    the tracks (301: shares of 151 and 150), compute their summed chi2 and
    gradient (here with the FP64 evaluation of the same adjoint), and one
    all-reduce gives both ranks the one-rank result of the whole sample."""
    import numpy as np
    import torch.multiprocessing as mp
    from mkfit_b200 import workloads
    from oracle.oracle import adj_f64_grad
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_grad_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    try:
        res = sorted(q.get(timeout=180) for _ in procs)
    finally:
        for p in procs:
            p.join(timeout=60)
            if p.is_alive():
                p.kill()
    for r in res:
        assert r[1] != "error", r
    ev = workloads.adjoint_event(0, n_tracks=301)
    theta = np.zeros((ev.hit_pos.shape[0], 3))
    theta[:, 2] = 1.0
    c2, g = adj_f64_grad(ev.par, ev.err, ev.chg, ev.hit_pos, ev.hit_err, theta, ev.rl_grid,
                         ev.xi_grid)
    (r0, c0, g0, s0), (r1, c1, g1, s1) = res
    assert s0 == (0, 151) and s1 == (151, 301)
    assert c0 == c1 and g0 == g1                # every rank holds the same sum
    assert c0 == pytest.approx(c2, rel=1e-12)
    np.testing.assert_allclose(np.array(g0), g, rtol=1e-10, atol=1e-9 * np.abs(g).max())
    assert all(p.exitcode == 0 for p in procs)

"""The multi-rank logic of bench.py on CPU: two gloo ranks over 127.0.0.1.

Each rank decodes its own frames (weak scaling, no data-path collective):
the ranks' seeds differ, the timed region is the max over ranks, and the
aggregate throughput counts every rank's frames over that time.  A rank that
never joins ends the others' collective with an error after the process
group's timeout instead of a hang."""
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, q):
    sys.path.insert(0, ROOT)
    os.environ.update({"MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port), "RANK": str(rank),
                       "WORLD_SIZE": str(world), "LOCAL_RANK": str(rank)})
    import torch.distributed as dist

    import bench
    w, r, local = bench.rank_env()
    bench.init_ranks(w, "gloo", timeout_s=30)
    ms = bench.max_over_ranks(10.0 * (r + 1), w, "cpu")  # rank 1 is the slow one
    value = bench.aggregate_gbps(w, 4096, 38880, ms)
    seeds = [bench.rank_seed(r, k) for k in range(7)]
    dist.barrier()
    dist.destroy_process_group()
    q.put((r, w, local, ms, value, seeds))


def _lone_rank(port, q):
    sys.path.insert(0, ROOT)
    os.environ.update({"MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port), "RANK": "0", "WORLD_SIZE": "2",
                       "LOCAL_RANK": "0"})
    import bench
    try:
        bench.init_ranks(2, "gloo", timeout_s=3)
        q.put("joined")
    except Exception as e:  # the peer never comes: a timeout, not a hang
        q.put("error: " + type(e).__name__)


def test_two_gloo_ranks_weak_scaling():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    res = sorted(q.get(timeout=120) for _ in ps)
    for p in ps:
        p.join(timeout=60)
        assert p.exitcode == 0
    (r0, w0, l0, ms0, v0, s0), (r1, w1, l1, ms1, v1, s1) = res
    assert (r0, r1, w0, w1, l0, l1) == (0, 1, 2, 2, 0, 1)
    assert ms0 == ms1 == 20.0  # both ranks report the slowest rank's time
    assert v0 == v1 == pytest.approx(2 * 4096 * 38880 / 0.020 / 1e9)
    assert not set(s0) & set(s1)  # every rank decodes its own frames


def test_missing_rank_times_out():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    p = ctx.Process(target=_lone_rank, args=(_free_port(), q))
    p.start()
    msg = q.get(timeout=120)
    p.join(timeout=60)
    assert msg.startswith("error"), msg


def _grad_rank(rank, world, port, q):
    sys.path.insert(0, ROOT)
    os.environ.update({"MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port), "RANK": str(rank),
                       "WORLD_SIZE": str(world), "LOCAL_RANK": str(rank)})
    import torch
    import torch.distributed as dist

    from dvbrx_b200 import train
    dist.init_process_group("gloo", world_size=world, rank=rank, timeout=__import__("datetime").timedelta(seconds=30))
    w, r = train.dist_world()
    # two parameters shaped like the learned tables, rank-dependent gradients
    a = torch.zeros(12, 4, requires_grad=True)
    b = torch.zeros(12, 4, requires_grad=True)
    (a * (r + 1)).sum().backward()
    (b * (2 * r + 3)).sum().backward()
    train.average_gradients([a, b], w)
    seeds = [train.rank_seed(7, r)]
    dist.barrier()
    dist.destroy_process_group()
    q.put((r, w, float(a.grad.mean()), float(b.grad.mean()), float(a.grad.std()), seeds))


def test_training_gradients_averaged_over_ranks():
    """Data-parallel training: one all-reduce gives every rank the mean
    gradient of the learned tables (so the tables stay identical), and the
    ranks draw different minibatches."""
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_grad_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    res = sorted(q.get(timeout=120) for _ in ps)
    for p in ps:
        p.join(timeout=60)
        assert p.exitcode == 0
    (r0, w0, a0, b0, s0, seed0), (r1, w1, a1, b1, s1, seed1) = res
    assert (w0, w1) == (2, 2)
    assert a0 == a1 == 1.5 and b0 == b1 == 4.0  # means of (1, 2) and (3, 5)
    assert s0 == s1 == 0.0
    assert seed0 != seed1

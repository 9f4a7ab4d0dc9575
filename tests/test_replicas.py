"""Multi-rank plumbing of the replica mode (fmm-fft_b200/replicas.py) as world-size-2 gloo
process groups on CPU: the same calls bench.py makes under NCCL, one process per rank."""
import os
import socket
import sys
import time

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "..", "fmm-fft_b200"))

import replicas  # noqa: E402


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _env(world, rank, port):
    return {"WORLD_SIZE": str(world), "RANK": str(rank), "LOCAL_RANK": str(rank),
            "MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)}


def _rank_timing(rank, world, port, q):
    os.environ.update(_env(world, rank, port))
    try:
        info = replicas.rank_info()
        dist = replicas.init_group(info, "gloo", timeout_s=30)
        # each replica "took" a different time; everybody must see the slowest
        my_ms = 10.0 + 7.5 * rank
        tot = replicas.max_over_ranks(my_ms, dist)
        rate = replicas.whole_job_rate(1 << 20, 4, info.world, tot)
        seed = replicas.replica_seed(0, info.rank)
        replicas.barrier(dist)
        replicas.finish(dist)
        q.put((rank, tot, rate, seed))
    except Exception as e:  # pragma: no cover - reported to the parent
        q.put((rank, "error", repr(e), None))


def _rank_leaves(rank, world, port, q):
    os.environ.update(_env(world, rank, port))
    info = replicas.rank_info()
    dist = replicas.init_group(info, "gloo", timeout_s=5)
    replicas.barrier(dist)
    if rank == 1:
        os._exit(0)  # leaves between steps, with nothing in flight
    t0 = time.time()
    try:
        replicas.max_over_ranks(1.0, dist)
        q.put((rank, "returned", time.time() - t0))
    except Exception as e:
        q.put((rank, "error:" + type(e).__name__, time.time() - t0))


def _spawn(fn, world):
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=fn, args=(r, world, port, q)) for r in range(world)]
    for p in ps:
        p.start()
    return ps, q


def test_rank_info_defaults_and_validation():
    assert replicas.rank_info({}) == replicas.RankInfo(1, 0, 0)
    assert replicas.rank_info({"WORLD_SIZE": "4", "RANK": "3"}) == replicas.RankInfo(4, 3, 3)
    with pytest.raises(ValueError):
        replicas.rank_info({"WORLD_SIZE": "2", "RANK": "2"})
    assert replicas.init_group(replicas.RankInfo(1, 0, 0), "gloo") is None
    assert replicas.max_over_ranks(3.5, None) == 3.5


def test_whole_job_rate():
    # 2 ranks x 3 steps x 2^24 samples in 6 ms (slowest rank) -> 16.8e9 samples/s
    assert replicas.whole_job_rate(1 << 24, 3, 2, 6.0) == pytest.approx((1 << 24) * 3 * 2 / 6e-3)
    with pytest.raises(ValueError):
        replicas.whole_job_rate(1, 1, 1, 0.0)


def test_two_ranks_agree_on_slowest_time():
    ps, q = _spawn(_rank_timing, 2)
    got = sorted(q.get(timeout=120) for _ in ps)
    for p in ps:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [g[1] for g in got] == [17.5, 17.5], got  # max of 10.0 and 17.5 on both ranks
    assert got[0][2] == got[1][2] == pytest.approx((1 << 20) * 4 * 2 / 17.5e-3)
    assert [g[3] for g in got] == [0, 1]  # each replica transforms its own seeded input


def test_rank_that_leaves_ends_the_collective_with_an_error():
    ps, q = _spawn(_rank_leaves, 2)
    res = q.get(timeout=120)
    for p in ps:
        p.join(timeout=60)
    assert res[0] == 0
    assert res[1].startswith("error"), res
    assert res[2] < 60.0  # bounded by the process-group timeout, not a hang

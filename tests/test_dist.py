"""Multi-rank host logic of the replica (independent signals per GPU) path,
run as two gloo processes on CPU."""
import os
import socket

import pytest

from so3_b200 import dist


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def test_shard_covers_every_signal_once():
    for n in (0, 1, 7, 16, 513):
        for world in (1, 2, 3, 8):
            seen = []
            for r in range(world):
                seen.extend(dist.shard(n, r, world))
            assert seen == list(range(n))
            sizes = [len(dist.shard(n, r, world)) for r in range(world)]
            assert max(sizes) - min(sizes) <= 1


def test_seeds_distinct_across_ranks():
    seeds = {dist.signal_seed(7, r, i) for r in range(8) for i in range(64)}
    assert len(seeds) == 8 * 64


def _worker(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    try:
        info = dist.init(backend="gloo", timeout_s=30)
        # each rank "processes" its shard with a rank-dependent duration
        shard = dist.shard(10, info.rank, info.world)
        elapsed = 0.5 + info.rank
        tmax = dist.max_over_ranks(elapsed)
        total = dist.sum_over_ranks(len(shard))
        dist.barrier()
        q.put((info.rank, tmax, total, dist.job_throughput(total, tmax)))
        dist.finalize()
    except Exception as e:  # report instead of hanging the parent
        q.put((rank, "error", repr(e), None))


def test_two_rank_gloo_max_time_and_job_throughput():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = [q.get(timeout=120) for _ in range(2)]
    for p in procs:
        p.join(timeout=60)
    for rank, tmax, total, thr in out:
        assert tmax != "error", total
        assert tmax == pytest.approx(1.5)
        assert total == 10
        assert thr == pytest.approx(10 / 1.5)

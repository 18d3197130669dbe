"""The multi-rank plumbing of bench.py and serving on the host: two gloo ranks on the CPU
(one process each, rendezvous on 127.0.0.1) join, meet at a barrier, agree on the maximum and
the sum of their values, compute the same request shards, gather every shard's results on
every rank (the sharded serve's p50/p99 come from them), and leave; shards cover every request
once and stay within one request of the average."""

import os
import socket

import pytest
import torch.multiprocessing as mp

from nabladyn_b200.replicas import Ranks, shard_requests


def _free_port() -> int:
    with socket.socket() as probe:
        probe.bind(("127.0.0.1", 0))
        return probe.getsockname()[1]


def _rank_main(rank: int, world: int, port: int, queue) -> None:
    os.environ.update({"RANK": str(rank), "WORLD_SIZE": str(world), "LOCAL_RANK": str(rank),
                       "MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
    ranks = Ranks("gloo", timeout_s=60)
    ranks.barrier()
    largest = ranks.max(rank + 1.5)
    total = ranks.sum(rank + 1.0)
    work = [float(k % 7 + 1) for k in range(23)]
    shards = shard_requests(work, ranks.world)
    # A sharded serve: each rank "serves" its share and every rank gathers all results.
    served = ranks.gather([(k, work[k] * 10.0) for k in shards[rank]])
    ranks.barrier()
    ranks.close()
    queue.put((rank, largest, total, shards, served))


def test_two_gloo_ranks_agree():
    world, port = 2, _free_port()
    context = mp.get_context("spawn")
    queue = context.Queue()
    processes = [context.Process(target=_rank_main, args=(r, world, port, queue))
                 for r in range(world)]
    for process in processes:
        process.start()
    results = sorted(queue.get(timeout=120) for _ in range(world))
    for process in processes:
        process.join(timeout=60)
        assert process.exitcode == 0
    assert [r[1] for r in results] == [2.5, 2.5]
    assert [r[2] for r in results] == [3.0, 3.0]
    assert results[0][3] == results[1][3]
    for result in results:  # every request's result reaches every rank exactly once
        served = result[4]
        assert sorted(k for k, _ in served) == list(range(23))
        assert all(latency == (k % 7 + 1) * 10.0 for k, latency in served)


@pytest.mark.parametrize("world", [1, 2, 3, 8])
def test_shards_cover_every_request_once_and_balance(world):
    work = [float((k * 37) % 101 + 1) for k in range(200)]
    shards = shard_requests(work, world)
    assert sorted(i for shard in shards for i in shard) == list(range(200))
    loads = [sum(work[i] for i in shard) for shard in shards]
    assert max(loads) - sum(work) / world <= max(work)


def test_single_rank_needs_no_group():
    ranks = Ranks("gloo")
    assert (ranks.rank, ranks.world) == (0, 1)
    assert ranks.max(4.0) == 4.0 and ranks.sum(2.0) == 2.0
    assert ranks.gather([1, 2]) == [1, 2]
    ranks.barrier()
    ranks.close()

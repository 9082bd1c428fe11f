"""Host logic of the multi-GPU replicas, on CPU with two gloo ranks.

bench.py --gpus N runs one independent structure per rank (no collective on the data
path); the collectives are the barrier and the max over ranks of the measured times, and a
batch of structures is split into contiguous blocks.  These run here as two processes with
the gloo backend: max over ranks, partition coverage, and the aggregate throughput.
"""
import os
import socket

import pytest
import torch.multiprocessing as mp

import numpy as np

from voronota_ltr import workloads as W
from voronota_ltr.replicas import Ranks, partition, partition_weighted, replica_throughput


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q):
    os.environ.update({"RANK": str(rank), "WORLD_SIZE": str(world), "LOCAL_RANK": str(rank),
                       "MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
    R = Ranks(backend="gloo", timeout_s=30)
    R.barrier()
    ms = 10.0 + 5.0 * rank  # rank 1 is the slowest
    m = R.max(ms)
    start, stop = partition(4096, world, rank)
    sizes = W.batch_sizes(4096)
    ws, we = partition_weighted(sizes, world, rank)
    balls = float(sizes[ws:we].sum())
    total = R.max(balls)
    R.close()
    q.put((rank, m, start, stop, ws, we, balls, total))


def test_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [o[1] for o in out] == [15.0, 15.0]  # every rank sees the max
    assert out[0][2:4] == (0, 2048) and out[1][2:4] == (2048, 4096)
    assert replica_throughput(100_000, 2, out[0][1]) == pytest.approx(2 * 100_000 / 0.015)
    # the batch split by balls: contiguous, complete, balanced
    assert out[0][4] == 0 and out[0][5] == out[1][4] and out[1][5] == 4096
    sizes = W.batch_sizes(4096)
    assert out[0][6] + out[1][6] == float(sizes.sum())
    assert abs(out[0][6] - out[1][6]) <= sizes.max()


def test_partition_covers_everything_once():
    for count in (0, 1, 7, 4096, 4097):
        for world in (1, 2, 3, 8):
            blocks = [partition(count, world, r) for r in range(world)]
            assert blocks[0][0] == 0 and blocks[-1][1] == count
            assert all(blocks[i][1] == blocks[i + 1][0] for i in range(world - 1))
            sizes = [b - a for a, b in blocks]
            assert max(sizes) - min(sizes) <= 1
    with pytest.raises(ValueError):
        partition(10, 2, 2)


def test_partition_weighted_balances_and_covers():
    sizes = W.batch_sizes(4096)
    for world in (1, 2, 3, 4, 8):
        blocks = [partition_weighted(sizes, world, r) for r in range(world)]
        assert blocks[0][0] == 0 and blocks[-1][1] == len(sizes)
        assert all(blocks[i][1] == blocks[i + 1][0] for i in range(world - 1))
        loads = [sizes[a:b].sum() for a, b in blocks]
        assert max(loads) - min(loads) <= 2 * sizes.max()
    assert partition_weighted([], 4, 2) == (0, 0)
    assert [partition_weighted([5], 3, r) for r in range(3)] in ([(0, 1), (1, 1), (1, 1)], [(0, 0), (0, 1), (1, 1)],
                                                                  [(0, 0), (0, 0), (0, 1)])
    with pytest.raises(ValueError):
        partition_weighted([1, 2], 2, 2)


def test_single_rank_needs_no_process_group():
    for k in ("RANK", "WORLD_SIZE", "LOCAL_RANK"):
        os.environ.pop(k, None)
    R = Ranks(backend="gloo")
    assert R.world == 1 and R.max(3.5) == 3.5
    R.close()

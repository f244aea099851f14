"""The N>1 host path on CPU: two gloo ranks shard frames and reduce the timing
with a max over ranks, as bench.py --gpus 2 does with NCCL."""
import os
import socket

import pytest
import torch.multiprocessing as mp

import multiframe


def test_shard_covers_every_frame_once():
    sizes = [4096 * 4096] * 8 + [2048 * 4096] * 16 + [1024 * 1024] * 24 + [512 * 512] * 16
    for world in (1, 2, 3, 4, 8):
        got = sorted(i for r in range(world) for i in multiframe.shard(len(sizes), r, world, sizes))
        assert got == list(range(len(sizes)))
        loads = [sum(sizes[i] for i in multiframe.shard(len(sizes), r, world, sizes)) for r in range(world)]
        assert max(loads) - min(loads) <= 4096 * 4096


def _worker(rank, world, port, q):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    mine = multiframe.shard(10, rank, world)
    dist.barrier()
    t = multiframe.max_over_ranks([float(len(mine)) + rank, 1.0 - rank], dist)
    q.put((rank, mine, t))
    dist.barrier()
    dist.destroy_process_group()


def test_two_gloo_ranks():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in range(2))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert res[0][1] == [0, 2, 4, 6, 8] and res[1][1] == [1, 3, 5, 7, 9]
    assert res[0][2] == res[1][2] == [6.0, 1.0]

"""Host logic of the multi-GPU benchmark on CPU ranks (gloo, world size 2): every rank
takes its own config-1 task blocks (no two ranks share one), the job time is the slowest
rank's and the work the sum over ranks — the same helpers bench.py uses over NCCL."""
import os
import socket
import sys

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, steps, out):
    sys.path.insert(0, ROOT)
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    blocks = bench.rank_blocks(rank, world, steps)
    # a rank's "time" and "work": distinct per rank so the reductions are checked
    t, w = bench.reduce_time_and_work(dist, 10.0 + rank, 100.0 * (rank + 1), "cpu")
    out[rank] = (blocks, t, w)
    dist.barrier()
    dist.destroy_process_group()


def test_two_ranks_shard_blocks_and_reduce_time():
    world, steps = 2, 4
    port = _free_port()
    with mp.Manager() as m:
        out = m.dict()
        mp.spawn(_worker, args=(world, port, steps, out), nprocs=world, join=True)
        res = dict(out)
    b0, b1 = res[0][0], res[1][0]
    assert len(b0) == len(b1) == steps and not set(b0) & set(b1)
    assert sorted(b0 + b1) == list(range(world * steps))
    for r in range(world):
        assert res[r][1] == 11.0 and res[r][2] == 300.0


def test_single_rank_needs_no_collective():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.reduce_time_and_work(None, 3.5, 7.0, "cpu") == (3.5, 7.0)
    assert bench.rank_blocks(0, 1, 3) == [0, 1, 2]

"""bench.py's multi-rank timing on the CPU (gloo, world size 2): every rank takes the same steps, the
reported per-step time is the maximum over ranks, and the whole-job value scales with the ranks."""
import os
import socket

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank_main(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    import time

    import bench
    calls = {"n": 0}

    def step():  # rank 1 is the slow replica
        calls["n"] += 1
        time.sleep(0.02 if rank == 1 else 0.002)

    ms = bench.timed_region(step, steps=4, warmup=3, dist=dist)
    out[rank] = (ms, calls["n"])
    dist.barrier()
    dist.destroy_process_group()


def test_max_over_ranks_gloo():
    world = 2
    port = _free_port()
    with mp.Manager() as m:
        out = m.dict()
        mp.spawn(_rank_main, args=(world, port, out), nprocs=world, join=True)
        res = dict(out)
    (ms0, n0), (ms1, n1) = res[0], res[1]
    assert n0 == n1 == 7                 # 3 warm-up + 4 timed steps on every rank
    assert ms0 == ms1                    # both ranks report the same (max) time
    assert ms0 >= 20.0                   # ... which is the slow rank's
    value = world * 1.0 / (ms0 / 1e3)    # whole-job throughput for 1 unit per step per rank
    assert value == pytest.approx(2.0 / (ms0 / 1e3))

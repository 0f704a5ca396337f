"""The multi-GPU path of bench.py is replicas: each rank corrects its own frame and the only
collective is the max-over-ranks timing.  Exercised here with two gloo ranks on the CPU."""
import os
import socket
import sys
from pathlib import Path

import torch.multiprocessing as mp

ROOT = Path(__file__).resolve().parents[1]


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    sys.path.insert(0, str(ROOT))
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    import bench
    ms, value = bench.aggregate(100.0 * (rank + 1), steps=5, iterations=6, world=world)
    out[rank] = (ms, value)
    dist.barrier()
    dist.destroy_process_group()


def test_replica_timing_is_the_max_over_ranks():
    world, port = 2, _free_port()
    with mp.Manager() as m:
        out = m.dict()
        mp.spawn(_rank, args=(world, port, out), nprocs=world, join=True)
        res = dict(out)
    for rank in range(world):
        ms, value = res[rank]
        assert ms == 200.0  # the slower rank's time
        assert abs(value - world * 5 * 6 / 0.2) < 1e-9


def test_single_rank_needs_no_collective():
    sys.path.insert(0, str(ROOT))
    import bench
    ms, value = bench.aggregate(50.0, steps=2, iterations=6, world=1)
    assert ms == 50.0 and abs(value - 12 / 0.05) < 1e-9

"""The multi-GPU form is replicas (every rank solves its own copy, no
collective on the data path); what bench.py reduces over ranks is the device
time of the slowest rank.  Checked with two gloo ranks on the CPU."""
import os
import sys
from pathlib import Path

import torch.multiprocessing as mp

ROOT = Path(__file__).resolve().parent.parent


def _rank(rank, world, port, out):
    sys.path.insert(0, str(ROOT))
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    import bench
    ms = bench.max_over_ranks(10.0 + 5.0 * rank, dist, device="cpu")
    out[rank] = (ms, bench.aggregate_rate(1_000_000, world, ms))
    dist.barrier()
    dist.destroy_process_group()


def test_two_rank_max_and_aggregate():
    world = 2
    port = 29500 + os.getpid() % 1000
    with mp.Manager() as m:
        out = m.dict()
        mp.spawn(_rank, args=(world, port, out), nprocs=world, join=True)
        res = dict(out)
    for rank in range(world):
        ms, rate = res[rank]
        assert ms == 15.0                           # the slowest rank's time
        assert abs(rate - 2 * 1e6 / 15e-3 / 1e6) < 1e-9

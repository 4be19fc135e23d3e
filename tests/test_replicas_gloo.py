"""Multi-rank host logic of bench.py on CPU: two gloo ranks, the job value taken over the slowest rank."""
import os
import sys
from pathlib import Path

import torch.multiprocessing as mp

ROOT = Path(__file__).resolve().parent.parent


def _rank(rank, world, port, out):
    import torch.distributed as dist
    sys.path.insert(0, str(ROOT))
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        ms = bench.slowest_rank_ms(100.0 + 50.0 * rank, world, "cpu")     # rank 1 is the slow one
        out[rank] = bench.job_throughput(ms, world, steps=10)
    finally:
        dist.destroy_process_group()


def test_two_replicas_value_uses_slowest_rank():
    port = 29500 + os.getpid() % 1000
    with mp.Manager() as m:
        out = m.dict()
        mp.start_processes(_rank, args=(2, port, out), nprocs=2, start_method="spawn", join=True)
        vals = dict(out)
    # both ranks see the slowest rank's 150 ms: 2 ranks x 10 reconstructions / 0.15 s
    assert abs(vals[0] - 2 * 10 / 0.150) < 1e-9 and vals[0] == vals[1]

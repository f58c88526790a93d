"""The multi-GPU plumbing of bench.py on CPU ranks (gloo, world size 2): replicas time
the same workload independently and rank 0 reports the slowest rank's time.  The
H-matvec itself does not shard across GPUs in this engine (replicas only)."""
import os
import socket

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    import sys
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        import bench
        got = bench.max_over_ranks([10.0 + rank, 5.0 - rank], world, "cpu")
        out[rank] = got
        dist.barrier()
    finally:
        dist.destroy_process_group()


@pytest.mark.timeout(120)
def test_max_over_ranks_gloo():
    world = 2
    mgr = mp.Manager()
    out = mgr.dict()
    mp.spawn(_rank, args=(world, _free_port(), out), nprocs=world, join=True)
    assert out[0] == out[1] == [11.0, 5.0]


def test_single_rank_passthrough():
    import bench
    assert bench.max_over_ranks([1.5, 2.5], 1) == [1.5, 2.5]

"""The multi-GPU path is replicas only: each rank runs its own transforms and the
only cross-rank step is the max over ranks of the step time. This exercises that
aggregation with world_size 2 over gloo on the CPU."""
import os
import socket

import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, results):
    import sys
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        local_ms = [4.0, 5.5][rank]  # rank 1 is slower
        ms, value = bench.replica_throughput(local_ms, 8, world, device="cpu")
        results[rank] = (ms, value)
    finally:
        dist.destroy_process_group()


def test_replica_throughput_takes_max_over_ranks():
    world = 2
    port = _free_port()
    with mp.Manager() as m:
        results = m.dict()
        mp.spawn(_worker, args=(world, port, results), nprocs=world, join=True)
        for rank in range(world):
            ms, value = results[rank]
            assert ms == 5.5
            assert abs(value - world * 8 / 5.5e-3) < 1e-6


def test_single_rank_needs_no_collective():
    import sys
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import bench
    ms, value = bench.replica_throughput(2.0, 8, 1)
    assert ms == 2.0 and value == 4000.0

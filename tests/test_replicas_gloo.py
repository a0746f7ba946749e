"""The multi-GPU path of bench.py is N independent replicas (one chain per
GPU, no data-path collective): every rank times its own sweep pair and rank 0
reports the maximum over ranks.  This runs that reduction as two gloo ranks on
the CPU."""
import os
import socket

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def worker(rank, world, port, out):
    import datetime
    import sys
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import bench
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    dist.barrier()
    t = bench.max_over_ranks(0.25 + 0.5 * rank, dist, "cpu")
    out[rank] = t
    dist.barrier()
    dist.destroy_process_group()


@pytest.mark.parametrize("world", [2])
def test_max_over_ranks_gloo(world):
    port = free_port()
    manager = mp.get_context("spawn").Manager()  # no fork of a multi-threaded process
    out = manager.dict()
    mp.spawn(worker, args=(world, port, out), nprocs=world, join=True)
    assert [out[r] for r in range(world)] == [0.25 + 0.5 * (world - 1)] * world


def test_single_process_is_identity():
    import sys
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import bench
    assert bench.max_over_ranks(1.5, None, "cpu") == 1.5

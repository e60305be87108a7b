"""The multi-GPU path is replicas only (independent systems per rank, no
data-path collective); its one reduction -- the max over ranks of the
per-step times -- exercised with two gloo ranks on the CPU."""
import os
import socket

import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, out):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        import bench
        vals = [1.0 + rank, 5.0 - rank, 2.0]
        got = bench.max_over_ranks(vals, world, "cpu")
        out[rank] = got
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_two_gloo_ranks():
    world = 2
    with mp.Manager() as mgr:
        out = mgr.dict()
        mp.spawn(_worker, args=(world, _free_port(), out), nprocs=world, join=True)
        for r in range(world):
            assert out[r] == [2.0, 5.0, 2.0]

"""Data-parallel gradient averaging over world_size-2 gloo ranks on CPU (the
host logic of multi-GPU training; on GPUs the same calls run over NCCL)."""
import os

import torch
import torch.multiprocessing as mp


def _rank(rank, world, port, out):
    import torch.distributed as dist

    from nect_b200.trainer import reduce_gradients

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        g1 = torch.full((1000, 2), float(rank + 1))
        g2 = torch.arange(10, dtype=torch.float32) * (rank + 1)
        reduce_gradients([g1, g2])
        out[rank] = (float(g1.mean()), g2.tolist())
    finally:
        dist.destroy_process_group()


def test_gradients_are_averaged_over_ranks():
    ctx = mp.get_context("spawn")
    with ctx.Manager() as mgr:
        out = mgr.dict()
        port = 29500 + os.getpid() % 1000
        procs = [ctx.Process(target=_rank, args=(r, 2, port, out)) for r in range(2)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(120)
            assert p.exitcode == 0
        for r in range(2):
            mean, g2 = out[r]
            assert mean == 1.5
            assert g2 == [1.5 * k for k in range(10)]


def test_single_process_is_a_no_op():
    from nect_b200.trainer import reduce_gradients

    g = torch.ones(4)
    reduce_gradients([g])
    assert torch.equal(g, torch.ones(4))

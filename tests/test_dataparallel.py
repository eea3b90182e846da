"""The data-parallel exchange on CPU with gloo ranks (world size 2).

Each rank holds different render gradients and V_R bitmaps; after the exchange every rank must
hold the global-batch mean gradient, the union bitmap, and a variance gradient amplified by k
only when the reduced (global) gradient is negative.
"""

import os
import socket

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime

    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        from voxneus_b200.dataparallel import GradExchange, amplify_after_reduce

        torch.manual_seed(100 + rank)
        grid = torch.nn.Parameter(torch.zeros(4, 5, 6))
        grid.grad = torch.randn(4, 5, 6)
        var = torch.nn.Parameter(torch.tensor(0.3))
        # rank 0 pushes the variance gradient negative, rank 1 positive but smaller: global < 0
        var.grad = torch.tensor(-3.0 if rank == 0 else 1.0)
        bitmap = torch.zeros(8, dtype=torch.int32)
        bitmap[rank] = 1 << (3 + rank)
        bitmap[7] = 1 << rank
        grads_before = grid.grad.clone()
        ex = GradExchange()
        ex.reduce_grads([grid, var])
        ex.union_bitmap(bitmap)
        flag = amplify_after_reduce(var, 5.0)
        q.put((rank, grads_before, grid.grad.clone(), var.grad.clone(), bool(flag), bitmap.clone()))
    finally:
        dist.destroy_process_group()


@pytest.mark.timeout(120)
def test_gradient_mean_bitmap_union_and_global_sign_amplification():
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = sorted([q.get(timeout=90) for _ in range(world)], key=lambda x: x[0])
    for p in procs:
        p.join(timeout=30)
        assert p.exitcode == 0
    mean = (res[0][1] + res[1][1]) / 2
    for _, _, g, v, flag, bm in res:
        assert torch.allclose(g, mean, atol=1e-7)
        assert flag is True and torch.allclose(v, torch.tensor(-5.0))  # mean(-3, 1) = -1, times k = 5
        assert bm[0].item() == 1 << 3 and bm[1].item() == 1 << 4 and bm[7].item() == 3

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
        # numpy copies travel by value: a tensor would travel as a shared-memory handle that the
        # parent can only open while this process is still alive
        q.put((rank, grads_before.numpy(), grid.grad.numpy().copy(), var.grad.numpy().copy(), bool(flag),
               bitmap.numpy().copy()))
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
    res = [(r, *(torch.from_numpy(a) for a in (gb, g, v)), f, torch.from_numpy(bm)) for r, gb, g, v, f, bm in res]
    mean = (res[0][1] + res[1][1]) / 2
    for _, _, g, v, flag, bm in res:
        assert torch.allclose(g, mean, atol=1e-7)
        assert flag is True and torch.allclose(v, torch.tensor(-5.0))  # mean(-3, 1) = -1, times k = 5
        assert bm[0].item() == 1 << 3 and bm[1].item() == 1 << 4 and bm[7].item() == 3


def _scene(O):
    torch.manual_seed(7)
    from voxneus_b200 import synthetic

    grid = synthetic.sphere_grid(24, noise=0.02, seed=3).requires_grad_(True)
    emb = (torch.rand(16, 1024, 2) * 0.4 - 0.2).requires_grad_(True)
    l0, l1 = torch.nn.Linear(51, 64), torch.nn.Linear(64, 3)
    ps = [t.detach().clone().requires_grad_(True) for t in (l0.weight, l0.bias, l1.weight, l1.bias)]
    return O.OracleScene(grid, torch.tensor(0.3, requires_grad=True), emb, *ps)


def _batch():
    g = torch.Generator().manual_seed(11)
    o = torch.randn(64, 3, generator=g)
    o = 3.0 * o / o.norm(dim=-1, keepdim=True)
    d = -o / 3.0 + 0.15 * torch.randn(64, 3, generator=g)
    d = d / d.norm(dim=-1, keepdim=True)
    t = torch.rand(64, 3, generator=g)
    t_rand = torch.rand(64, 32, generator=g)
    us = [torch.rand(64, 8, generator=g) for _ in range(4)]
    return o, d, t, t_rand, us


RENDER = dict(n_samples=32, n_importance=32, steps=4, perturb=True)


def _half_batch_worker(rank, world, port, q):
    """One rank of the data-parallel step on the oracle: its half of the rays rendered and
    back-propagated, then GradExchange.exchange (reduce, union, amplify), then the regularizer
    on the union V_R: the order FusedTrainer(exchange=...) runs."""
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime

    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        from oracle import reference_path as O
        from voxneus_b200.dataparallel import GradExchange

        torch.set_num_threads(1)
        sc = _scene(O)
        o, d, t, t_rand, us = _batch()
        h = slice(32 * rank, 32 * rank + 32)
        near, far = O.near_far_from_sphere(o[h], d[h])
        out = sc.render(o[h], d[h], near, far, t_rand=t_rand[h], us=[u[h] for u in us], **RENDER)
        O.huber(out["rgb"], t[h]).backward()
        res = sc.res()
        _, lin = O.extract_active_vertices(out["corner_indices"], res)
        marks = torch.zeros(res[0] * res[1] * res[2], dtype=torch.int32)
        marks[lin] = 1
        ex = GradExchange(bucket_bytes=32 << 10)  # the grid and table in place, the MLP and s in one bucket
        flag = ex.exchange(sc.params(), marks, sc.variance, amplify_k=5.0)
        lin_all = marks.nonzero().reshape(-1)
        verts = torch.stack([lin_all // (res[1] * res[2]), (lin_all // res[2]) % res[1], lin_all % res[2]], dim=-1)
        verts = O.relax_filter(verts, sc.xyz_min.float(), sc.eps().float())
        g3 = sc.grid.detach().reshape(res)
        _, ge = O.eikonal(g3, verts, sc.eps(), res, weight=0.1)
        _, gc = O.curvature(g3, verts, sc.eps(), res, weight=5e-4)
        with torch.no_grad():
            sc.grid.grad.add_(ge.reshape(sc.grid.shape))
            sc.grid.grad.add_(gc.reshape(sc.grid.shape))
        q.put((rank, [p.grad.numpy().copy() for p in sc.params()], bool(flag), verts.shape[0], ex.collectives))
    finally:
        dist.destroy_process_group()


@pytest.mark.timeout(180)
def test_two_half_batches_through_the_exchange_equal_the_full_batch():
    from oracle import reference_path as O

    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_half_batch_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = sorted([q.get(timeout=150) for _ in range(world)], key=lambda x: x[0])
    for p in procs:
        p.join(timeout=30)
        assert p.exitcode == 0
    res = [(r, [torch.from_numpy(g) for g in gs], f, n, c) for r, gs, f, n, c in res]
    sc = _scene(O)
    o, d, t, t_rand, us = _batch()
    ref = sc.train_step(o, d, t, amplify_k=5.0, t_rand=t_rand, us=us, **RENDER)
    names = ("grid", "variance", "embeddings", "w0", "b0", "w1", "b1")
    for rank, grads, flag, n_active, collectives in res:
        assert collectives == 4  # grid, table, one bucket of the rest, the bitmap gather
        assert n_active == ref["n_active"]
        assert flag == ref["amplified"]
        for nm, g in zip(names, grads):
            r = ref["grads"][nm]
            err = float((g - r).abs().max()) / max(float(r.abs().max()), 1e-30)
            assert err < 1e-5, (rank, nm, err)
    for a, b in zip(res[0][1], res[1][1]):
        assert torch.equal(a, b)  # every rank holds the same gradients

"""The CUDA-graph training step against the eager step (training/trainer.py:166-393 as one unit).

Same seeded model, rays and default-generator draws; deterministic adjoints (sorted segmented
sums, no float atomics), so the two must agree bit for bit: parameters, Adam state, occupancy
grid and the step's outputs, across an occupancy refresh between replays, the cosine LR schedule
and the switch to the amplified-s variant (a second capture).
"""

import pytest
import torch

pytestmark = pytest.mark.gpu

DEV = torch.device("cuda", 0)


def _model():
    from voxneus_b200.models import VoxNeuS

    torch.manual_seed(3)
    m = VoxNeuS(grid_res=32, hash_log2_size=12, occupancy_res=16).to(DEV)
    with torch.no_grad():
        m.sdf_grid.grid.add_(0.01 * torch.randn_like(m.sdf_grid.grid))
        m.radiance_hash.encoder.embeddings.uniform_(-0.1, 0.1)
    return m


def _rays(n, seed, host=False):
    g = torch.Generator().manual_seed(seed)
    o = torch.randn(n, 3, generator=g)
    o = 3.0 * o / o.norm(dim=-1, keepdim=True)
    d = -o / 3.0 + 0.05 * torch.randn(n, 3, generator=g)
    d = d / d.norm(dim=-1, keepdim=True)
    t = torch.rand(n, 3, generator=g)
    if host == "packed":  # the three slices of one pinned (3, N, 3) tensor: one copy
        hb = torch.stack([o, d, t]).pin_memory()
        return hb[0], hb[1], hb[2]
    if host:
        return o.pin_memory(), d.pin_memory(), t.pin_memory()
    return o.to(DEV), d.to(DEV), t.to(DEV)


def _run(cuda_graph, steps, warmup_s, host=False, grid_adam="torch", exchange=None):
    from voxneus_b200.rendering import RaySampler
    from voxneus_b200.training import FusedTrainer

    m = _model()
    tr = FusedTrainer(m, RaySampler(16, 16, perturb=True), band_voxels=3.0, s_warmup_steps=warmup_s,
                      total_steps=10, occupancy_update_interval=3, cuda_graph=cuda_graph, grid_adam=grid_adam,
                      exchange=exchange)
    torch.manual_seed(11)  # the sampler's and occupancy refresh's draws (default CUDA generator)
    hist = []
    for i in range(steps):
        o, d, t = _rays(256, 100 + i, ("packed" if i % 2 else True) if host else False)
        out = tr.step(o, d, t, step=i)
        hist.append({k: v.clone() for k, v in out.items()})
    torch.cuda.synchronize()
    return m, tr, hist


@pytest.mark.parametrize("grid_adam", ["torch", "cuda"])
def test_graph_step_is_bitwise_the_eager_step(grid_adam):
    """grid_adam: "torch", the plain-PyTorch mode's formula (the default), or "cuda", the reference
    extension's (masked_adam_upd; in the graph its step size is read from device memory)."""
    from voxneus_b200 import ops

    ops.set_deterministic(True)
    try:
        me, te, he = _run(False, 8, 5, grid_adam=grid_adam)
        mg, tg, hg = _run(True, 8, 5, grid_adam=grid_adam)
    finally:
        ops.set_deterministic(False)
    assert tg.graph() is not None and tg.graph().amplify  # captured, and recaptured with amplification
    assert tg.replayed_launches > 0
    for i, (a, b) in enumerate(zip(he, hg)):
        for k in a:
            assert torch.equal(a[k], b[k]), (i, k)
    for (n, pa), pb in zip(me.named_parameters(), mg.parameters()):
        assert torch.equal(pa, pb), n
    for name in ("sdf_optimizer", "net_optimizer"):
        oe, og = te.optimizers[name], tg.optimizers[name]
        for pa, pb in zip(me.parameters(), mg.parameters()):
            if pa in oe.state:
                sa, sb = oe.state[pa], og.state[pb]
                assert sa["step"] == sb["step"]
                assert torch.equal(sa["exp_avg"], sb["exp_avg"]) and torch.equal(sa["exp_avg_sq"], sb["exp_avg_sq"])
    assert torch.equal(me.occupancy_grid.density_grid, mg.occupancy_grid.density_grid)
    assert torch.equal(me.occupancy_grid.occupancy_mask, mg.occupancy_grid.occupancy_mask)


def test_graph_step_takes_pinned_host_inputs():
    """Pinned host rays and targets (copied by the step, in graph mode straight into the graph's
    input buffers; separate tensors and slices of one packed tensor alternate) give the bits of
    device inputs."""
    from voxneus_b200 import ops

    ops.set_deterministic(True)
    try:
        me, _, he = _run(False, 5, 100)
        mh, th, hh = _run(True, 5, 100, host=True)
    finally:
        ops.set_deterministic(False)
    assert th.graph() is not None
    for a, b in zip(he, hh):
        for k in a:
            assert torch.equal(a[k], b[k]), k
    for pa, pb in zip(me.parameters(), mh.parameters()):
        assert torch.equal(pa, pb)


def test_graph_mode_falls_back_to_eager_with_explicit_randoms():
    """Caller-supplied uniforms are not graph inputs: such a step runs eagerly (and drops the graph)."""
    from voxneus_b200.rendering import RaySampler
    from voxneus_b200.training import FusedTrainer

    m = _model()
    tr = FusedTrainer(m, RaySampler(16, 16, perturb=True), band_voxels=3.0, cuda_graph=True)
    for i in range(3):
        o, d, t = _rays(128, i)
        tr.step(o, d, t, step=i)
    assert tr.graph() is not None
    o, d, t = _rays(128, 9)
    randoms = m.draw_sampler_randoms(128, 16, 16, 4, DEV)
    out = tr.step(o, d, t, step=3, randoms=randoms)
    assert tr.graph() is None and torch.isfinite(out["loss_rgb"]).all()


def test_sampler_draws_are_the_separate_draws():
    """The per-step uniforms drawn in place into one tensor equal separate draws stacked (the same
    generator offsets: the reference's draw order is kept)."""
    m = _model()
    g1 = torch.Generator(device=DEV).manual_seed(21)
    t1, u1 = m.draw_sampler_randoms(300, 64, 64, 4, DEV, generator=g1)
    g2 = torch.Generator(device=DEV).manual_seed(21)
    t2 = torch.rand((300, 64), device=DEV, generator=g2)
    u2 = torch.stack([torch.rand((300, 16), device=DEV, generator=g2) for _ in range(4)])
    assert torch.equal(t1, t2) and torch.equal(u1, u2)


def test_graph_mode_recaptures_on_a_new_batch_shape():
    """A new ray count mid-run captures the step again; the steps stay the eager steps' bits."""
    from voxneus_b200 import ops
    from voxneus_b200.rendering import RaySampler
    from voxneus_b200.training import FusedTrainer

    sizes = [192, 192, 192, 256, 256, 192]

    def run(cuda_graph):
        m = _model()
        tr = FusedTrainer(m, RaySampler(16, 16, perturb=True), band_voxels=3.0, cuda_graph=cuda_graph)
        torch.manual_seed(13)
        outs = []
        for i, n in enumerate(sizes):
            o, d, t = _rays(n, 200 + i)
            outs.append(tr.step(o, d, t, step=i)["loss_rgb"].clone())
        torch.cuda.synchronize()
        return m, tr, outs

    ops.set_deterministic(True)
    try:
        me, _, le = run(False)
        mg, tg, lg = run(True)
    finally:
        ops.set_deterministic(False)
    assert tg.graph() is not None and tg.graph().o.shape[0] == sizes[-1]
    assert all(torch.equal(a, b) for a, b in zip(le, lg))
    for pa, pb in zip(me.parameters(), mg.parameters()):
        assert torch.equal(pa, pb)


def test_data_parallel_graph_step_is_bitwise_the_eager_step():
    """With a gradient exchange (here a one-rank NCCL group on this GPU) the step runs as two
    graphs, render + backward and regularizer + optimizers, with the exchange's collectives run
    eagerly between them (no collective inside a graph); it gives the eager data-parallel step's
    bits: parameters, Adam state and outputs, across the switch to the amplified variant."""
    import socket

    import torch.distributed as dist

    from voxneus_b200 import ops
    from voxneus_b200.dataparallel import GradExchange

    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        port = sk.getsockname()[1]
    dist.init_process_group("nccl", init_method=f"tcp://127.0.0.1:{port}", rank=0, world_size=1, device_id=DEV)
    try:
        ops.set_deterministic(True)
        try:
            me, te, he = _run(False, 8, 5, exchange=GradExchange())
            mg, tg, hg = _run(True, 8, 5, exchange=GradExchange())
        finally:
            ops.set_deterministic(False)
        assert tg.graph() is not None and tg.graph().graph2 is not None and tg.graph().amplify
        for i, (a, b) in enumerate(zip(he, hg)):
            for k in a:
                assert torch.equal(a[k], b[k]), (i, k)
        for (n, pa), pb in zip(me.named_parameters(), mg.parameters()):
            assert torch.equal(pa, pb), n
        for name in ("sdf_optimizer", "net_optimizer"):
            oe, og = te.optimizers[name], tg.optimizers[name]
            for pa, pb in zip(me.parameters(), mg.parameters()):
                if pa in oe.state:
                    sa, sb = oe.state[pa], og.state[pb]
                    assert sa["step"] == sb["step"]
                    assert torch.equal(sa["exp_avg"], sb["exp_avg"]) and torch.equal(sa["exp_avg_sq"], sb["exp_avg_sq"])
        del tg, mg
    finally:
        torch.cuda.synchronize()
        dist.destroy_process_group()

"""The fused training step against the reference's own trainer, and a reference checkpoint served.

`tests/golden/train_step.npz` holds steps 1 and 2 of the reference's VoxNeuSTrainer.train_step
(training/trainer.py:166-393), run by `make_golden.py` on a 20^3 scene with RaySampler(64, 64,
perturb=True) and s_warmup_steps = 0: the sampler's uniforms and the z it returned, the losses,
the amplification flag, the learning rates, and every parameter, gradient and Adam moment after
each step. Its targets make the s gradient negative at step 1 (amplified by k = 5, variance
learning rate x5) and positive at step 2 (neither), so both branches of
training/scheduler.py:14-33 and trainer.py:311-329 are pinned by the reference itself.

Step 1 runs from the fixture's initial state; step 2 from the reference's state after step 1
(parameters and Adam moments loaded into the fused trainer). Each step trains on the samples the
reference's sampler produced (FusedTrainer.step(z_vals=...)); the fused sampler is compared with
those samples separately, on the same uniforms. Tolerances: losses 1e-5 relative, gradients 1e-4
of their largest magnitude, the flag exact, the Adam moments 1e-4 of the scale the gradient gives
them, and the parameters equal to Adam (float64, the reference optimizer's torch formulas) of the
fused step's own state and gradients to float32 rounding (1e-6 of the parameter's scale plus the
largest update, lr / (1 - b1^t); Adam divides by sqrt(v), so where |g| is
near eps an allowed gradient difference moves the update by up to the learning rate).
"""

import math
import os

import pytest
import torch

pytestmark = pytest.mark.gpu

DEV = torch.device("cuda", 0)
GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
VAL_TOL = 1e-5
GRAD_TOL = 1e-4


def _close(a, b, tol, what, scale=None):
    a = torch.as_tensor(a).detach().double().cpu()
    b = torch.as_tensor(b).detach().double().cpu()
    assert a.shape == b.shape, (what, a.shape, b.shape)
    if scale is None:
        scale = float(b.abs().max()) if b.numel() else 0.0
    err = (a - b).abs()
    bad = err > tol * (b.abs() + max(scale, 1e-30))
    assert not bool(bad.any()), f"{what}: max err {float(err.max()):.3e} vs scale {scale:.3e} ({int(bad.sum())} bad)"


@pytest.fixture(scope="module")
def fx(golden):
    from voxneus_b200 import _lib

    _lib.load()
    return golden("train_step.npz")


def _model(fx, prefix):
    from voxneus_b200.models import VoxNeuS

    m = VoxNeuS(grid_res=20, hash_log2_size=7, occupancy_res=8).to(DEV)
    with torch.no_grad():
        for n, p in m.named_parameters():
            p.copy_(fx[f"{prefix}param/{n}"].to(DEV))
        m.occupancy_grid.occupancy_mask.copy_(fx["occupancy"].to(DEV))
    return m


def _load_adam(tr, m, fx, prefix):
    """The reference optimizers' state after a step, into the fused trainer's optimizers."""
    for n, p in m.named_parameters():
        opt = tr.optimizers["sdf_optimizer" if n == "sdf_grid.grid" else "net_optimizer"]
        opt.state[p] = {"step": int(fx[f"{prefix}adam_step/{n}"]), "exp_avg": fx[f"{prefix}exp_avg/{n}"].to(DEV).clone(),
                        "exp_avg_sq": fx[f"{prefix}exp_avg_sq/{n}"].to(DEV).clone()}


def _adam64(p, g, m, v, t, lr, b1, b2, eps, masked):
    p, g, m, v = (x.detach().double().cpu() for x in (p, g, m, v))
    m2 = b1 * m + (1 - b1) * g
    v2 = b2 * v + (1 - b2) * g * g
    p2 = p - (lr / (1 - b1 ** t)) * m2 / (v2.sqrt() / math.sqrt(1 - b2 ** t) + eps)
    if masked:
        keep = g == 0
        m2, v2, p2 = torch.where(keep, m, m2), torch.where(keep, v, v2), torch.where(keep, p, p2)
    return p2, m2, v2


def _trainer(m, fx):
    from voxneus_b200.rendering import RaySampler
    from voxneus_b200.training import FusedTrainer

    w_eik, w_curv = float(fx["step1/w_eik"]), float(fx["step1/w_curv"])
    assert (float(fx["step2/w_eik"]), float(fx["step2/w_curv"])) == (w_eik, w_curv)
    return FusedTrainer(m, RaySampler(64, 64, perturb=True), w_eik=w_eik, w_curv=w_curv, band_voxels=None,
                        s_warmup_steps=0, total_steps=40000, lr_sdf=0.1, lr_hash=0.01, lr_mlp=0.001,
                        lr_variance=0.0005, occupancy_update_interval=16)


@pytest.mark.parametrize("k", [1, 2])
def test_sampler_matches_reference_trainer_samples(fx, k):
    """The fused sampler on the step's inputs and uniforms against the z the reference's sampler
    returned inside its trainer. A ray whose reference samples are ill-conditioned at 1e-5 (an
    occupancy cell, the unit sphere or a flat CDF stretch within a few ulps) may move by up to an
    interval; at most one ray of the 32 is allowed outside 1e-5, and every ray within 1e-2."""
    from voxneus_b200 import ops

    m = _model(fx, "init/" if k == 1 else f"step{k - 1}/")
    lo, hi = m.sdf_grid.bounds()
    occ = m.occupancy_grid
    z, _, _ = ops.sample_multistep(m.sdf_grid.grid.detach(), lo, hi, fx["rays_o"].to(DEV), fx["rays_d"].to(DEV), None,
                                   None, 64, 64, 4, True, fx[f"step{k}/t_rand"].to(DEV), fx[f"step{k}/us"].to(DEV),
                                   occ.occupancy_mask, *occ.bounds(), want_z=True)
    zr = fx[f"step{k}/z"].double()
    err = (z.cpu().double() - zr).abs()
    bad = (err > VAL_TOL * (zr.abs() + float(zr.abs().max()))).any(dim=1)
    print(f"step {k}: fused z vs the reference trainer's z: {int(bad.sum())} of 32 rays outside 1e-5, "
          f"max |dz| {float(err.max()):.2e}")
    assert int(bad.sum()) <= 1
    assert float(err.max()) < 1e-2


@pytest.mark.parametrize("k", [1, 2])
def test_step_matches_reference_trainer(fx, k):
    m = _model(fx, "init/" if k == 1 else f"step{k - 1}/")
    tr = _trainer(m, fx)
    if k > 1:
        _load_adam(tr, m, fx, f"step{k - 1}/")
    before = {}
    for n, p in m.named_parameters():
        st = tr.optimizers["sdf_optimizer" if n == "sdf_grid.grid" else "net_optimizer"].state.get(p)
        before[n] = (p.detach().clone(), (int(st["step"]), st["exp_avg"].clone(), st["exp_avg_sq"].clone()) if st
                     else (0, torch.zeros_like(p), torch.zeros_like(p)))
    out = tr.step(fx["rays_o"].to(DEV), fx["rays_d"].to(DEV), fx["target"].to(DEV), step=k,
                  z_vals=fx[f"step{k}/z"].to(DEV))
    torch.cuda.synchronize()
    for key in ("loss_rgb", "loss_eik", "loss_curv"):
        _close(out[key], fx[f"step{k}/{key}"], VAL_TOL, f"step {k} {key}")
    amp = bool(tr.amp_flag.item())
    assert amp == bool(fx[f"step{k}/s_amplified"]), (k, amp)
    assert amp == (k == 1)  # the fixture's s gradient is negative at step 1 and positive at step 2
    f = tr.lr_factor(k)
    assert abs(tr.lr_hash * f - float(fx[f"step{k}/lr_hash"])) < 1e-12
    assert abs(tr.lr_mlp * f - float(fx[f"step{k}/lr_mlp"])) < 1e-12
    lr_var = tr.lr_variance * (tr.amplify_k if amp else 1.0)
    assert abs(lr_var - float(fx[f"step{k}/lr_s"])) < 1e-12
    lrs = {"sdf_grid.grid": 0.1, "variance_net.variance": lr_var, "radiance_hash.encoder.embeddings": tr.lr_hash * f}
    for n, p in m.named_parameters():
        g_ref = fx[f"step{k}/grad/{n}"]
        _close(p.grad, g_ref, GRAD_TOL, f"step {k} grad {n}")
        grid = n == "sdf_grid.grid"
        b1, b2 = (0.9, 0.99) if grid else (0.9, 0.999)
        lr = lrs.get(n, tr.lr_mlp * f)
        p0, (t0, m0, v0) = before[n]
        st = tr.optimizers["sdf_optimizer" if grid else "net_optimizer"].state[p]
        assert int(st["step"]) == t0 + 1 == int(fx[f"step{k}/adam_step/{n}"])
        pe, me, ve = _adam64(p0, p.grad, m0, v0, t0 + 1, lr, b1, b2, 1e-8, masked=grid)
        _close(st["exp_avg"], me, 1e-6, f"step {k} exp_avg {n} (Adam of the fused gradient)")
        _close(st["exp_avg_sq"], ve, 1e-5, f"step {k} exp_avg_sq {n} (Adam of the fused gradient)")
        _close(p, pe, 1e-6, f"step {k} param {n} (Adam of the fused gradient)",
               scale=float(p0.abs().max()) + lr / (1 - b1 ** (t0 + 1)))
        gmax = float(g_ref.abs().max())
        _close(st["exp_avg"], fx[f"step{k}/exp_avg/{n}"], GRAD_TOL, f"step {k} exp_avg {n}", scale=(1 - b1) * gmax)
        _close(st["exp_avg_sq"], fx[f"step{k}/exp_avg_sq/{n}"], 3 * GRAD_TOL, f"step {k} exp_avg_sq {n}",
               scale=(1 - b2) * gmax * gmax)
        print(f"step {k} {n}: max |p - p_reference| / lr = "
              f"{float((p.detach().cpu().double() - fx[f'step{k}/param/{n}'].double()).abs().max()) / lr:.2e}")


def test_reference_checkpoint_into_scene_store(golden):
    """A checkpoint written by the reference's save_checkpoint (training/checkpoint.py:11-33)
    loaded into the serving scene store, rendered directly and through the serving engine, against
    the reference's render of the same model (RaySampler(64, 64, perturb=False), scripts/render.py)."""
    from voxneus_b200 import _lib
    from voxneus_b200.rendering import RaySampler
    from voxneus_b200.serving import Request, SceneStore, ServingEngine

    _lib.load()
    ref = golden("checkpoint_render.npz")
    store = SceneStore(DEV)
    step = store.load_checkpoint("ck", os.path.join(GOLDEN, "checkpoint_step2.pt"))
    assert step == 2
    m = store.scenes["ck"]
    o, d = ref["rays_o"].to(DEV), ref["rays_d"].to(DEV)
    with torch.no_grad():
        out = m.render(o, d, RaySampler(64, 64, perturb=False), None, None)
    for key in ("rgb", "depth", "normal", "opacity"):
        _close(out[key], ref[key], VAL_TOL, f"render {key}", scale=1.0 if key != "depth" else None)
    eng = ServingEngine(store, render_buckets=(64,), query_buckets=(1024,))
    try:
        req = eng.submit(Request("ck", "render", (ref["rays_o"], ref["rays_d"]))).wait(120)
    finally:
        eng.close()
    _close(req.outputs["rgb"], ref["rgb"], VAL_TOL, "served rgb", scale=1.0)
    _close(req.outputs["depth"], ref["depth"], VAL_TOL, "served depth")

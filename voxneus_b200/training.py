"""Training step of the hot path (reference voxneus/training/{trainer,optimizer,scheduler}.py).

`FusedTrainer.step` is the timed unit of training/trainer.py:166-393 minus host logging:
fused render (sampler, geometry, appearance, MLP, compositing), Huber loss, backward through
the hand-written adjoints (with the k=5 s-gradient rule applied in-kernel), V_R from the
render's corner bitmap, the fused eikonal + curvature stencil into grid.grad, and the optimizer
steps (masked grid Adam kernel; one multi-tensor Adam launch for the hash table, MLP and
variance). No host synchronisation unless the s amplification is active (its LR rule needs the
flag).
"""

from __future__ import annotations

import math
from typing import Dict, Optional

import torch
from torch.optim import Optimizer

from . import ops
from .models import VoxNeuS
from .rendering import RaySampler, compute_huber_color_loss


def amplify_s_gradient(variance_param: torch.nn.Parameter, k: float = 5.0) -> bool:
    """grad <- k * grad when grad < 0 (training/scheduler.py:14-33); host read like the reference."""
    if variance_param.grad is None:
        return False
    with torch.no_grad():
        if variance_param.grad.item() < 0.0:
            variance_param.grad.mul_(k)
            return True
    return False


class SparseGridAdam(Optimizer):
    """Adam that skips grad == 0 voxels (training/optimizer.py:15-116) on the masked Adam kernel."""

    def __init__(self, params, lr: float = 1e-1, betas=(0.9, 0.999), eps: float = 1e-8, weight_decay: float = 0.0):
        if weight_decay != 0.0:
            raise ValueError("weight decay is not on the masked kernel path")
        super().__init__(params, dict(lr=lr, betas=betas, eps=eps, weight_decay=weight_decay))
        self.last_updated_count = 0

    @torch.no_grad()
    def step(self, closure=None):
        for group in self.param_groups:
            b1, b2 = group["betas"]
            for p in group["params"]:
                if p.grad is None:
                    continue
                st = self.state[p]
                if not st:
                    st["step"] = 0
                    st["exp_avg"] = torch.zeros_like(p)
                    st["exp_avg_sq"] = torch.zeros_like(p)
                st["step"] += 1
                ops.adam_update(p, p.grad.contiguous(), st["exp_avg"], st["exp_avg_sq"], st["step"], b1, b2,
                                group["lr"], group["eps"], masked=True)
        return None


class FusedAdam(Optimizer):
    """torch.optim.Adam (the network optimizer of training/optimizer.py:119-154) with every
    parameter of every group updated by one kernel launch per 8 tensors (`vx_adam_torch`).

    Same update, hyper-parameters and state names as torch.optim.Adam (step, exp_avg,
    exp_avg_sq); parameters whose grad is None are skipped, as there. No weight decay or amsgrad.
    """

    def __init__(self, params, lr: float = 1e-3, betas=(0.9, 0.999), eps: float = 1e-8, weight_decay: float = 0.0,
                 amsgrad: bool = False):
        if weight_decay != 0.0 or amsgrad:
            raise ValueError("weight decay and amsgrad are not on the fused Adam kernel")
        super().__init__(params, dict(lr=lr, betas=betas, eps=eps, weight_decay=weight_decay, amsgrad=amsgrad))

    @torch.no_grad()
    def step(self, closure=None):
        loss = None
        if closure is not None:
            with torch.enable_grad():
                loss = closure()
        batches: Dict[tuple, list] = {}
        for group in self.param_groups:
            b1, b2 = group["betas"]
            for p in group["params"]:
                if p.grad is None:
                    continue
                if p.grad.is_sparse:
                    raise RuntimeError("FusedAdam does not support sparse gradients")
                st = self.state[p]
                if not st:
                    st["step"] = 0
                    st["exp_avg"] = torch.zeros_like(p, memory_format=torch.contiguous_format)
                    st["exp_avg_sq"] = torch.zeros_like(p, memory_format=torch.contiguous_format)
                st["step"] += 1
                batches.setdefault((float(b1), float(b2), float(group["eps"])), []).append(
                    (p, p.grad.contiguous(), st["exp_avg"], st["exp_avg_sq"], st["step"], group["lr"]))
        for (b1, b2, eps), segs in batches.items():
            ops.adam_torch(segs, b1, b2, eps)
        return loss


def create_optimizer(model: VoxNeuS, lr_sdf=0.1, lr_hash=1e-2, lr_mlp=1e-3, lr_variance=1e-2, use_sparse_sdf=True):
    """Optimizer suite (training/optimizer.py:119-154)."""
    sdf_opt = (SparseGridAdam([model.sdf_grid.grid], lr=lr_sdf, betas=(0.9, 0.99)) if use_sparse_sdf
               else torch.optim.Adam([model.sdf_grid.grid], lr=lr_sdf, betas=(0.9, 0.99)))
    net_opt = FusedAdam([{"params": model.radiance_hash.parameters(), "lr": lr_hash},
                         {"params": model.radiance_mlp.parameters(), "lr": lr_mlp},
                         {"params": model.variance_net.parameters(), "lr": lr_variance}],
                        betas=(0.9, 0.999), eps=1e-8)
    return {"sdf_optimizer": sdf_opt, "net_optimizer": net_opt}


class FusedTrainer:
    """One training step of the fused path; returns device tensors (no host sync)."""

    def __init__(self, model: VoxNeuS, sampler: Optional[RaySampler] = None, w_eik: float = 0.1,
                 w_curv: float = 5e-4, band_voxels: Optional[float] = None, relax_radius: float = 1.2,
                 amplify_k: float = 5.0, s_warmup_steps: int = 5000, total_steps: int = 40000, lr_sdf: float = 0.1,
                 lr_hash: float = 0.01, lr_mlp: float = 0.001, lr_variance: float = 0.0005, up_sample_steps: int = 4,
                 huber_delta: float = 0.1, optimize: bool = True, exchange=None,
                 occupancy_update_interval: int = 16, occupancy_seed: int = 0):
        self.model = model
        self.exchange = exchange  # dataparallel.GradExchange for world_size > 1
        self.sampler = sampler or RaySampler(64, 64, perturb=True)
        self.w_eik, self.w_curv = w_eik, w_curv
        self.relax_radius = relax_radius
        self.amplify_k = amplify_k
        self.s_warmup_steps = s_warmup_steps
        self.total_steps = total_steps
        self.up_sample_steps = up_sample_steps
        self.huber_delta = huber_delta
        self.lr_hash, self.lr_mlp, self.lr_variance = lr_hash, lr_mlp, lr_variance
        self.optimize = optimize
        self.optimizers = create_optimizer(model, lr_sdf, lr_hash, lr_mlp, lr_variance) if optimize else {}
        dev = model.sdf_grid.grid.device
        self.res = [int(r) for r in model.sdf_grid.res]
        eps = model.sdf_grid.voxel_size_host()
        # |f| < band * eps_x, threshold rounded to float32 like a float32 tensor comparison
        self.band = float(torch.tensor(band_voxels * eps[0], dtype=torch.float32)) if band_voxels else 0.0
        self.bitmap = ops.new_bitmap(self.res, dev)
        self.filtered = ops.new_filtered(self.res, dev)
        self.counts = torch.zeros(4, dtype=torch.int64, device=dev)
        self.reg_losses = torch.zeros(2, device=dev)
        self.amp_flag = torch.zeros(1, dtype=torch.int32, device=dev)
        # training/trainer.py:171-173: occupancy refresh every `occupancy_update_interval` steps
        # (0 disables). Data-parallel ranks draw the cells from one shared seed so that their
        # masks stay identical; a single process draws from the default generator.
        self.occupancy_update_interval = int(occupancy_update_interval)
        self.occ_generator = None
        if exchange is not None:
            self.occ_generator = torch.Generator(device=dev)
            self.occ_generator.manual_seed(int(occupancy_seed))

    def step(self, rays_o, rays_d, target, step: int = 0, randoms=None) -> Dict[str, torch.Tensor]:
        m = self.model
        if [int(r) for r in m.sdf_grid.res] != self.res:
            raise RuntimeError("grid resolution changed; build a new FusedTrainer after scale_volume_grid")
        for opt in self.optimizers.values():
            opt.zero_grad(set_to_none=True)
        if not self.optimize:
            for p in m.parameters():
                p.grad = None
        if self.occupancy_update_interval > 0 and step % self.occupancy_update_interval == 0:
            m.update_occupancy_grid(subsample_ratio=0.25, generator=self.occ_generator)
        self.bitmap.zero_()
        self.counts.zero_()
        amp_k = self.amplify_k if step >= self.s_warmup_steps else 0.0
        ex = self.exchange
        out = m.render(rays_o, rays_d, self.sampler, None, None, up_sample_steps=self.up_sample_steps,
                       sphere_radius=1.0, randoms=randoms, vr_bitmap=self.bitmap, extras=False,
                       amplify_k=0.0 if ex is not None else amp_k, amp_flag=self.amp_flag)
        loss = compute_huber_color_loss(out["rgb"], target, self.huber_delta)
        loss.backward()
        if ex is not None:
            from .dataparallel import amplify_after_reduce

            ex.reduce_grads(list(m.parameters()))
            ex.union_bitmap(self.bitmap)
            if amp_k > 0:
                self.amp_flag.copy_(amplify_after_reduce(m.variance_net.variance, amp_k).reshape(1).int())
        grid = m.sdf_grid.grid
        lo, hi = m.sdf_grid.bounds()
        ops.vr_count(self.bitmap, grid.detach(), self.res, lo, hi, self.relax_radius, self.band, self.counts,
                     self.filtered)
        ops.reg_stencil(grid.detach(), self.filtered, self.res, lo, hi, self.relax_radius, self.band, self.counts,
                        self.w_eik, self.w_curv, grid.grad, self.reg_losses)
        if self.optimize:
            lr_factor = (math.cos(math.pi * step / max(self.total_steps, 1)) + 1.0) * 0.5 * (1.0 - 0.05) + 0.05
            net = self.optimizers["net_optimizer"]
            net.param_groups[0]["lr"] = self.lr_hash * lr_factor
            net.param_groups[1]["lr"] = self.lr_mlp * lr_factor
            amplified = bool(self.amp_flag.item()) if amp_k > 0 else False
            net.param_groups[2]["lr"] = self.lr_variance * (self.amplify_k if amplified else 1.0)
            for opt in self.optimizers.values():
                opt.step()
        return {"loss_rgb": loss.detach(), "loss_eik": self.reg_losses[0], "loss_curv": self.reg_losses[1],
                "n_active": ops.final_count(self.counts, self.relax_radius, self.band), "rgb": out["rgb"].detach()}

"""Training step of the hot path (reference voxneus/training/{trainer,optimizer,scheduler}.py).

`FusedTrainer.step` is the timed unit of training/trainer.py:166-393 minus host logging:
fused render (sampler, geometry, appearance, MLP, compositing), Huber loss, backward through
the hand-written adjoints (with the k=5 s-gradient rule applied in-kernel), V_R from the
render's corner bitmap, the fused eikonal + curvature stencil into grid.grad, and the optimizer
steps (masked grid Adam kernel; one multi-tensor Adam launch for the hash table, MLP and
variance). No host synchronisation unless the s amplification is active (its LR rule needs the
flag).

With `cuda_graph=True` (single process), the step from render to optimizer is captured once per
s-amplification setting into a CUDA graph and replayed: the step-dependent optimizer scalars
(cosine LR, bias corrections, the amplified variance LR picked on the device from the flag) are
computed on the host exactly as the eager optimizers compute them and copied to the device before
each replay; the occupancy refresh runs eagerly between replays.
"""

from __future__ import annotations

import math
from typing import Dict, Optional

import torch
from torch.optim import Optimizer

from . import ops
from .models import VoxNeuS
from .rendering import RaySampler


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
    """Adam that skips grad == 0 voxels (training/optimizer.py:15-116) on the masked Adam kernel.

    formula="torch" (default): the reference optimizer's vectorised PyTorch path
    (optimizer.py:86-113), p -= lr/(1-b1^t) * m / (sqrt(v)/sqrt(1-b2^t) + eps).
    formula="cuda": the update of the reference's extension kernel, which its optimizer
    dispatches to when that extension is built (optimizer.py:64-77, adam_upd_kernel.cu),
    p -= lr*sqrt(1-b2^t)/(1-b1^t) * m / (sqrt(v) + eps). They differ only in where eps enters.
    """

    def __init__(self, params, lr: float = 1e-1, betas=(0.9, 0.999), eps: float = 1e-8, weight_decay: float = 0.0,
                 formula: str = "torch"):
        if weight_decay != 0.0:
            raise ValueError("weight decay is not on the masked kernel path")
        if formula not in ("torch", "cuda"):
            raise ValueError(f"formula must be 'torch' or 'cuda', not {formula!r}")
        super().__init__(params, dict(lr=lr, betas=betas, eps=eps, weight_decay=weight_decay))
        self.formula = formula
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
                if self.formula == "torch":
                    ops.adam_torch([(p, p.grad.contiguous(), st["exp_avg"], st["exp_avg_sq"], st["step"], group["lr"])],
                                   b1, b2, group["eps"], masked=True)
                else:
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


def create_optimizer(model: VoxNeuS, lr_sdf=0.1, lr_hash=1e-2, lr_mlp=1e-3, lr_variance=1e-2, use_sparse_sdf=True,
                     grid_formula: str = "torch"):
    """Optimizer suite (training/optimizer.py:119-154)."""
    sdf_opt = (SparseGridAdam([model.sdf_grid.grid], lr=lr_sdf, betas=(0.9, 0.99), formula=grid_formula)
               if use_sparse_sdf
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
                 occupancy_update_interval: int = 16, occupancy_seed: int = 0, cuda_graph: bool = False,
                 grid_adam: str = "torch", tc_wait_polls: Optional[int] = None, tc_check_every: int = 8):
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
        self.optimizers = (create_optimizer(model, lr_sdf, lr_hash, lr_mlp, lr_variance, grid_formula=grid_adam)
                           if optimize else {})
        dev = model.sdf_grid.grid.device
        self.res = [int(r) for r in model.sdf_grid.res]
        eps = model.sdf_grid.voxel_size_host()
        # |f| < band * eps_x, threshold rounded to float32 like a float32 tensor comparison
        self.band = float(torch.tensor(band_voxels * eps[0], dtype=torch.float32)) if band_voxels else 0.0
        self.bitmap = ops.new_bitmap(self.res, dev)
        self.filtered = ops.new_filtered(self.res, dev)
        self.counts = torch.zeros(4, dtype=torch.int64, device=dev)
        self.reg_losses = torch.zeros(2, device=dev)
        self.n_active = torch.zeros((), dtype=torch.int64, device=dev)  # |V_R| after the filters
        self.amp_flag = torch.zeros(1, dtype=torch.int32, device=dev)
        # blocks of the MLP kernels that gave up waiting on the tensor core, accumulated over the
        # steps (also returned by every step as "tc_status"); copied to the host every
        # tc_check_every steps and read a step later without a synchronisation: a nonzero value
        # makes the next step raise
        self.tc_status = torch.zeros(1, dtype=torch.int32, device=dev)
        self.tc_wait_polls = tc_wait_polls
        self._tc_watch = ops.StatusWatch(self.tc_status, "training step", every=tc_check_every)
        # training/trainer.py:171-173: occupancy refresh every `occupancy_update_interval` steps
        # (0 disables). Data-parallel ranks draw the cells from one shared seed so that their
        # masks stay identical; a single process draws from the default generator.
        self.occupancy_update_interval = int(occupancy_update_interval)
        self.occ_generator = None
        if exchange is not None:
            self.occ_generator = torch.Generator(device=dev)
            self.occ_generator.manual_seed(int(occupancy_seed))
        self.cuda_graph = bool(cuda_graph)
        self._graphs: Dict[bool, _StepGraph] = {}
        self._eager_steps = 0
        self.replayed_launches = 0  # library kernel launches run by graph replays (not in the launch counter)

    def lr_factor(self, step: int) -> float:
        """Cosine decay to 0.05 of the base LR (training/trainer.py:378-385)."""
        return (math.cos(math.pi * step / max(self.total_steps, 1)) + 1.0) * 0.5 * (1.0 - 0.05) + 0.05

    def step(self, rays_o, rays_d, target, step: int = 0, randoms=None, z_vals=None) -> Dict[str, torch.Tensor]:
        """One training step. rays_o, rays_d, target may be device tensors or (pinned) host tensors,
        which are copied to the device on the current stream: in graph mode straight into the
        graph's input buffers. In graph mode the returned tensors are the graph's outputs,
        overwritten by the next step (copy them to keep them). randoms: the sampler's (t_rand, u)
        uniforms; z_vals: sample depths to train on instead of running the sampler (VoxNeuS.render);
        either makes the step eager."""
        m = self.model
        if [int(r) for r in m.sdf_grid.res] != self.res:
            raise RuntimeError("grid resolution changed; build a new FusedTrainer after scale_volume_grid")
        graphable = (self.cuda_graph and self.optimize and randoms is None and z_vals is None
                     and torch.is_grad_enabled())
        self._tc_watch.check()
        if graphable and self._eager_steps >= GRAPH_WARMUP_STEPS:
            out = self._graph_step(rays_o, rays_d, target, step)
            self._tc_watch.after_step()
            return out
        self._graphs.clear()  # an eager step owns fresh gradients; replays would no longer see them
        self._eager_steps += 1
        dev = self.bitmap.device
        rays_o, rays_d, target = (t if t.device == dev else t.to(dev, non_blocking=True)
                                  for t in (rays_o, rays_d, target))
        if z_vals is not None and z_vals.device != dev:
            z_vals = z_vals.to(dev, non_blocking=True)
        out = self._eager_step(rays_o, rays_d, target, step, randoms, z_vals)
        self._tc_watch.after_step()
        return out

    def _refresh_occupancy(self, step: int) -> None:
        if self.occupancy_update_interval > 0 and step % self.occupancy_update_interval == 0:
            self.model.update_occupancy_grid(subsample_ratio=0.25, generator=self.occ_generator)

    def _render_backward(self, rays_o, rays_d, target, amp_k: float, randoms=None, z_vals=None):
        """Render, loss and backward (the V_R bitmap marked on the way); returns (loss, rgb)."""
        m = self.model
        self.bitmap.zero_()
        self.counts.zero_()
        with ops.tc_guard(self.tc_status, self.tc_wait_polls):
            out = m.render(rays_o, rays_d, self.sampler, None, None, up_sample_steps=self.up_sample_steps,
                           sphere_radius=1.0, randoms=randoms, vr_bitmap=self.bitmap, extras=False,
                           amplify_k=0.0 if self.exchange is not None else amp_k, amp_flag=self.amp_flag,
                           z_vals=z_vals)
            # the loss kernel writes dL/drgb beside the loss: the backward starts from it directly
            # (the same values as loss.backward(), without the seed fill and the scale by 1)
            loss, d_rgb = ops.huber_loss(out["rgb"], target, self.huber_delta)
            out["rgb"].backward(d_rgb)
        return loss.detach(), out["rgb"].detach()

    def _exchange(self, amp_k: float) -> None:
        """Data-parallel ranks: the gradient exchange (reduce, bitmap union, amplification on the
        reduced sign), in place: the gradient and flag tensors keep their addresses."""
        m = self.model
        flag = self.exchange.exchange(list(m.parameters()), self.bitmap, m.variance_net.variance, amp_k)
        if flag is not None:
            self.amp_flag.copy_(flag.reshape(1).int())

    def _regularize(self, loss, rgb) -> Dict[str, torch.Tensor]:
        """V_R (counts and filters) and the regularizer stencil into the grid gradient."""
        m = self.model
        grid = m.sdf_grid.grid
        lo, hi = m.sdf_grid.bounds()
        ops.vr_count(self.bitmap, grid.detach(), self.res, lo, hi, self.relax_radius, self.band, self.counts,
                     self.filtered)
        ops.reg_stencil(grid.detach(), self.filtered, self.res, lo, hi, self.relax_radius, self.band, self.counts,
                        self.w_eik, self.w_curv, grid.grad, self.reg_losses, self.n_active)
        return {"loss_rgb": loss, "loss_eik": self.reg_losses[0], "loss_curv": self.reg_losses[1],
                "n_active": self.n_active, "rgb": rgb, "tc_status": self.tc_status}

    def _render_backward_regularize(self, rays_o, rays_d, target, amp_k: float, randoms=None, z_vals=None):
        """Render, loss, backward, gradient exchange, V_R and the regularizer stencil."""
        loss, rgb = self._render_backward(rays_o, rays_d, target, amp_k, randoms, z_vals)
        if self.exchange is not None:
            self._exchange(amp_k)
        return self._regularize(loss, rgb)

    def _eager_step(self, rays_o, rays_d, target, step: int, randoms, z_vals=None) -> Dict[str, torch.Tensor]:
        m = self.model
        for opt in self.optimizers.values():
            opt.zero_grad(set_to_none=True)
        if not self.optimize:
            for p in m.parameters():
                p.grad = None
        self._refresh_occupancy(step)
        amp_k = self.amplify_k if step >= self.s_warmup_steps else 0.0
        res = self._render_backward_regularize(rays_o, rays_d, target, amp_k, randoms, z_vals)
        if self.optimize:
            lr_factor = self.lr_factor(step)
            net = self.optimizers["net_optimizer"]
            net.param_groups[0]["lr"] = self.lr_hash * lr_factor
            net.param_groups[1]["lr"] = self.lr_mlp * lr_factor
            amplified = bool(self.amp_flag.item()) if amp_k > 0 else False
            net.param_groups[2]["lr"] = self.lr_variance * (self.amplify_k if amplified else 1.0)
            for opt in self.optimizers.values():
                opt.step()
        return res

    # ---------------------------------------------------------------- CUDA graph mode ------

    def _graph_step(self, rays_o, rays_d, target, step: int) -> Dict[str, torch.Tensor]:
        amplify = step >= self.s_warmup_steps
        g = self._graphs.get(amplify)
        if g is not None and (g.o.shape != rays_o.shape or g.d.shape != rays_d.shape or g.t.shape != target.shape
                              or g.io.dtype != rays_o.dtype):
            g = None  # a new batch shape: capture again
        if g is None:
            self._graphs.clear()  # one captured variant at a time (amplification switches on once)
            g = _StepGraph(self, rays_o, rays_d, target, amplify, self.bitmap.device)
            self._graphs[amplify] = g
        self._refresh_occupancy(step)
        g.run(rays_o, rays_d, target, step)
        self.replayed_launches += g.launches
        return g.outputs

    def graph(self) -> Optional["_StepGraph"]:
        """The captured step graph in use (None before the first graph step)."""
        return next(iter(self._graphs.values()), None)


GRAPH_WARMUP_STEPS = 2  # eager steps before the first capture (optimizer state, autograd, allocator)
_SCALAR_SLOTS = 4  # pinned host copies of the per-step optimizer scalars in flight


class _StepGraph:
    """One captured training step (render .. optimizer) of a FusedTrainer.

    Static inputs: rays_o, rays_d, target buffers (the caller's tensors are copied in) and a device
    table of optimizer scalars, three per parameter, the grid's first: {step size (lr/(1-b1^t) for
    the torch formula, lr*sqrt(1-b2^t)/(1-b1^t) for the extension's), 1/sqrt(1-b2^t), step size when
    the s gradient was amplified (the variance only)}. The sampler's uniforms come from torch's default
    CUDA generator inside the graph (torch advances its offset per replay, so the draws are the
    eager step's). Gradients live in the graph's memory pool and are rewritten by every replay.
    """

    def __init__(self, tr: FusedTrainer, rays_o, rays_d, target, amplify: bool, dev: torch.device):
        m = tr.model
        self.tr = tr
        self.amplify = amplify
        # the inputs as one (3, N, 3) buffer: a caller whose rays and targets are the three slices of
        # one host tensor is served with a single copy
        self.io = torch.empty((3,) + tuple(rays_o.shape), dtype=rays_o.dtype, device=dev)
        self.o, self.d, self.t = self.io[0], self.io[1], self.io[2]
        self.grid_opt = tr.optimizers["sdf_optimizer"]
        self.net_opt = tr.optimizers["net_optimizer"]
        if not isinstance(self.grid_opt, SparseGridAdam) or not isinstance(self.net_opt, FusedAdam):
            raise RuntimeError("graph mode needs the masked grid Adam and the fused network Adam")
        self.net_params = [(gi, p) for gi, grp in enumerate(self.net_opt.param_groups) for p in grp["params"]]
        for opt in (self.grid_opt, self.net_opt):
            for grp in opt.param_groups:
                for p in grp["params"]:
                    if not opt.state.get(p):
                        raise RuntimeError("graph mode starts after an eager step has created the optimizer state")
        n = 3 + 3 * len(self.net_params)
        self.scalars = torch.zeros(n, device=dev)
        self.host = torch.zeros(_SCALAR_SLOTS, n).pin_memory()
        self.slot_events = [None] * _SCALAR_SLOTS
        self.slot = 0
        for opt in (self.grid_opt, self.net_opt):
            opt.zero_grad(set_to_none=True)  # backward inside the capture allocates the gradients
        amp_k = tr.amplify_k if amplify else 0.0
        from . import _lib

        self.graph = torch.cuda.CUDAGraph(keep_graph=True)
        self.graph2 = None
        self.amp_k = amp_k
        l0 = _lib.launch_count()
        if tr.exchange is None:
            with torch.cuda.graph(self.graph):
                self.outputs = tr._render_backward_regularize(self.o, self.d, self.t, amp_k)
                self._optimizer_launches(m)
        else:
            # data-parallel ranks: two graphs, the collectives between them run eagerly (no NCCL
            # call inside a graph): render + backward, then V_R + regularizer + optimizers
            with torch.cuda.graph(self.graph):
                loss, rgb = tr._render_backward(self.o, self.d, self.t, amp_k)
            self.graph.instantiate()
            tr._exchange(amp_k)  # the gradients the capture allocated, as every replay leaves them
            self.graph2 = torch.cuda.CUDAGraph(keep_graph=True)
            with torch.cuda.graph(self.graph2):
                self.outputs = tr._regularize(loss, rgb)
                self._optimizer_launches(m)
            self.graph2.instantiate()
        self.launches = _lib.launch_count() - l0
        if self.graph2 is None:
            self.graph.instantiate()

    def _optimizer_launches(self, m) -> None:
        grid = m.sdf_grid.grid
        b1, b2 = self.grid_opt.param_groups[0]["betas"]
        st = self.grid_opt.state[grid]
        if self.grid_opt.formula == "torch":
            ops.adam_torch([(grid, grid.grad, st["exp_avg"], st["exp_avg_sq"], 0, 0.0, self.scalars[0:3], None)],
                           b1, b2, self.grid_opt.param_groups[0]["eps"], masked=True)
        else:
            ops.masked_adam_update_dev(grid, grid.grad, st["exp_avg"], st["exp_avg_sq"], self.scalars[0:1], b1, b2,
                                       self.grid_opt.param_groups[0]["eps"])
        flag = self.tr.amp_flag if self.amplify else None
        batches: Dict[tuple, list] = {}
        for k, (gi, p) in enumerate(self.net_params):
            grp = self.net_opt.param_groups[gi]
            if p.grad is None:
                raise RuntimeError("graph mode needs a gradient for every network parameter")
            st = self.net_opt.state[p]
            b1, b2 = grp["betas"]
            batches.setdefault((float(b1), float(b2), float(grp["eps"])), []).append(
                (p, p.grad, st["exp_avg"], st["exp_avg_sq"], 0, 0.0, self.scalars[3 + 3 * k:6 + 3 * k],
                 flag if gi == 2 else None))
        for (b1, b2, eps), segs in batches.items():
            ops.adam_torch(segs, b1, b2, eps)

    def _advance_scalars(self, step: int) -> torch.Tensor:
        """Advance the optimizer state's step counts as the eager optimizers do; return this
        step's scalar row (the values the eager kernels would compute on the host)."""
        tr = self.tr
        row = [0.0] * self.scalars.numel()
        grp = self.grid_opt.param_groups[0]
        st = self.grid_opt.state[tr.model.sdf_grid.grid]
        st["step"] += 1
        b1, b2 = grp["betas"]
        if self.grid_opt.formula == "torch":
            ss, inv = ops.adam_torch_step_scalars(st["step"], b1, b2, grp["lr"])
            row[0:3] = [ss, inv, ss]
        else:
            row[0] = ops.adam_reference_step_size(st["step"], b1, b2, grp["lr"])
        f = tr.lr_factor(step)
        lrs = [tr.lr_hash * f, tr.lr_mlp * f, tr.lr_variance]
        for gi, lr in enumerate(lrs):
            self.net_opt.param_groups[gi]["lr"] = lr
        for k, (gi, p) in enumerate(self.net_params):
            grp = self.net_opt.param_groups[gi]
            st = self.net_opt.state[p]
            st["step"] += 1
            b1, b2 = grp["betas"]
            ss, inv = ops.adam_torch_step_scalars(st["step"], b1, b2, lrs[gi])
            amp = ss
            if gi == 2 and self.amplify:
                amp = ops.adam_torch_step_scalars(st["step"], b1, b2, tr.lr_variance * tr.amplify_k)[0]
            row[3 + 3 * k:6 + 3 * k] = [ss, inv, amp]
        return torch.tensor(row, dtype=torch.float32)

    def run(self, rays_o, rays_d, target, step: int) -> None:
        b = rays_o._base
        if (b is not None and rays_d._base is b and target._base is b and b.shape == self.io.shape
                and b.dtype == self.io.dtype and b.is_contiguous() and rays_o.data_ptr() == b[0].data_ptr()
                and rays_d.data_ptr() == b[1].data_ptr() and target.data_ptr() == b[2].data_ptr()):
            self.io.copy_(b, non_blocking=True)
        else:
            self.o.copy_(rays_o, non_blocking=True)
            self.d.copy_(rays_d, non_blocking=True)
            self.t.copy_(target, non_blocking=True)
        s = self.slot
        self.slot = (s + 1) % _SCALAR_SLOTS
        if self.slot_events[s] is not None:
            self.slot_events[s].synchronize()  # the copy that last read this pinned slot has run
        self.host[s].copy_(self._advance_scalars(step))
        self.scalars.copy_(self.host[s], non_blocking=True)
        ev = self.slot_events[s] or torch.cuda.Event()
        ev.record()
        self.slot_events[s] = ev
        self.graph.replay()
        if self.graph2 is not None:  # data-parallel: the exchange between the two graphs
            self.tr._exchange(self.amp_k)
            self.graph2.replay()

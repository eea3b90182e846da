"""Data-parallel training over ranks (one process per GPU, torch.distributed / NCCL).

Rays are independent, so each rank renders its own ray batch against a full replica of the
scene. The one exchange per step (`GradExchange.exchange`), in this order:
1. the render gradients (grid, hash table, MLP, variance) are summed over the ranks and divided
   by the world size (each rank's loss is the mean over its equal share of the global batch, so
   this is the gradient of the global-batch mean): the tensors of at least `bucket_bytes` are
   reduced in place, the small ones packed into one flat bucket and reduced with one call, so a
   step issues at most a few collectives;
2. the V_R bitmaps are unioned (all-gather + OR), so every rank regularizes the same vertices;
3. the k-amplification of dL/dv is applied to the reduced gradient, on its global sign
   (training/scheduler.py:14-33 after the reduction).
The regularizer then runs on the union, identically on every rank, and each rank's optimizers
take identical steps.
"""

from __future__ import annotations

from typing import List, Optional

import torch
import torch.distributed as dist


class GradExchange:
    """The exchange FusedTrainer runs between backward and the regularizer when world_size > 1."""

    def __init__(self, group=None, bucket_bytes: int = 1 << 20):
        self.group = group
        self.world = dist.get_world_size(group)
        self.bucket_bytes = int(bucket_bytes)
        self.collectives = 0  # collectives issued (for tests and diagnostics)

    def reduce_grads(self, params: List[torch.Tensor]) -> None:
        """Sum every parameter's gradient over the ranks, then divide by the world size."""
        small: List[torch.Tensor] = []
        for p in params:
            if p.grad is None:
                p.grad = torch.zeros_like(p)
            g = p.grad
            if g.numel() * g.element_size() >= self.bucket_bytes or not g.is_contiguous():
                dist.all_reduce(g, op=dist.ReduceOp.SUM, group=self.group)
                self.collectives += 1
                g.div_(self.world)
            else:
                small.append(g)
        by_dtype = {}
        for g in small:
            by_dtype.setdefault(g.dtype, []).append(g)
        for grads in by_dtype.values():
            flat = torch.cat([g.reshape(-1) for g in grads])
            dist.all_reduce(flat, op=dist.ReduceOp.SUM, group=self.group)
            self.collectives += 1
            flat.div_(self.world)
            off = 0
            for g in grads:
                n = g.numel()
                g.copy_(flat[off:off + n].view_as(g))
                off += n

    def union_bitmap(self, bitmap: torch.Tensor) -> None:
        """OR of every rank's bitmap (any integer tensor), in place."""
        flat = bitmap.reshape(-1)
        if dist.get_backend(self.group) == "nccl":
            gathered = torch.empty(self.world, flat.numel(), dtype=flat.dtype, device=flat.device)
            dist.all_gather_into_tensor(gathered, flat, group=self.group)
            parts = list(gathered)
        else:
            parts = [torch.empty_like(flat) for _ in range(self.world)]
            dist.all_gather(parts, flat, group=self.group)
        self.collectives += 1
        out = parts[0].clone()
        for r in range(1, self.world):
            out.bitwise_or_(parts[r])
        bitmap.copy_(out.reshape(bitmap.shape))

    def exchange(self, params: List[torch.Tensor], bitmap: torch.Tensor, variance: Optional[torch.Tensor] = None,
                 amplify_k: float = 0.0) -> Optional[torch.Tensor]:
        """The step's exchange in order: reduce the gradients, union the V_R bitmaps, amplify the
        reduced variance gradient (when amplify_k > 0). Returns the amplification flag (a device
        bool) or None."""
        self.reduce_grads(params)
        self.union_bitmap(bitmap)
        if variance is not None and amplify_k > 0:
            return amplify_after_reduce(variance, amplify_k)
        return None


def amplify_after_reduce(variance: torch.nn.Parameter, k: float) -> torch.Tensor:
    """grad <- k * grad where the (reduced) grad is negative, in place (a captured optimizer
    launch holds the gradient's address); returns the device flag."""
    g = variance.grad
    neg = g < 0
    g.copy_(torch.where(neg, g * k, g))
    return neg

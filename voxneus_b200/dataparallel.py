"""Data-parallel training over ranks (one process per GPU, torch.distributed / NCCL).

Rays are independent, so each rank renders its own ray batch against a full replica of the
scene. The one exchange per step: the render gradients (grid, hash table, MLP, variance) are
all-reduced and averaged (the loss is a mean over the global batch), and the V_R bitmaps are
unioned (all-gather + OR) so every rank applies the identical regularizer gradient. The
k-amplification of dL/dv is applied after the reduction, on the global sign.
"""

from __future__ import annotations

from typing import List, Optional

import torch
import torch.distributed as dist


class GradExchange:
    """Hooks FusedTrainer calls between backward and the regularizer when world_size > 1."""

    def __init__(self, group=None):
        self.group = group
        self.world = dist.get_world_size(group)

    def reduce_grads(self, params: List[torch.Tensor]) -> None:
        for p in params:
            if p.grad is None:
                p.grad = torch.zeros_like(p)
            dist.all_reduce(p.grad, op=dist.ReduceOp.SUM, group=self.group)
            p.grad.div_(self.world)

    def union_bitmap(self, bitmap: torch.Tensor) -> None:
        flat = bitmap.reshape(-1)
        if dist.get_backend(self.group) == "nccl":
            gathered = torch.empty(self.world, flat.numel(), dtype=flat.dtype, device=flat.device)
            dist.all_gather_into_tensor(gathered, flat, group=self.group)
            parts = list(gathered)
        else:
            parts = [torch.empty_like(flat) for _ in range(self.world)]
            dist.all_gather(parts, flat, group=self.group)
        out = parts[0].clone()
        for r in range(1, self.world):
            out.bitwise_or_(parts[r])
        bitmap.copy_(out.reshape(bitmap.shape))


def amplify_after_reduce(variance: torch.nn.Parameter, k: float) -> torch.Tensor:
    """grad <- k * grad where the (reduced) grad is negative; returns the device flag."""
    g = variance.grad
    neg = g < 0
    variance.grad = torch.where(neg, g * k, g)
    return neg

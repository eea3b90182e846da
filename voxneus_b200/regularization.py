"""Active vertices and closed-form regularizers (reference voxneus/regularization/*)."""

from __future__ import annotations

from typing import Optional, Tuple

import torch

from . import ops


def _eps_host(voxel_size):
    if isinstance(voxel_size, torch.Tensor):
        return [float(v) for v in voxel_size.detach().float().cpu()]
    return [float(v) for v in voxel_size]


def extract_active_vertices(corner_indices: torch.Tensor, grid_res) -> Tuple[torch.Tensor, torch.Tensor]:
    """Unique, ascending vertices of all corners (regularization/active_vertices.py:12-50).

    Bitmap mark + count + ordered compaction; the output size needs one host read of the count.
    """
    res = [int(r) for r in grid_res]
    dev = corner_indices.device
    bm = ops.new_bitmap(res, dev)
    ops.vr_mark_corners(corner_indices, res, bm)
    zeros3 = (0.0, 0.0, 0.0)
    counts = ops.vr_count(bm, None, res, zeros3, (1.0, 1.0, 1.0))
    n = int(counts[0].item())
    verts, lin = ops.vr_compact(bm, None, res, zeros3, (1.0, 1.0, 1.0), 0.0, 0.0, counts, n)
    return verts, lin


def _grid_parts(grid_data):
    data = grid_data.squeeze(0).squeeze(0) if grid_data.dim() == 5 else grid_data
    return data.detach().contiguous()


def compute_eikonal_loss_and_gradient(grid_data, active_vertices, voxel_size, grid_res, eps: float = 1e-8,
                                      accumulate_grad: Optional[torch.Tensor] = None, weight: float = 1.0):
    """Closed-form eikonal loss and gradient (regularization/eikonal.py:13-171).

    accumulate_grad given: the weighted gradient is added in place and (loss, None) returned;
    otherwise (loss, gradient (1,1,X,Y,Z)) with weight 1 like the reference.
    """
    if eps != 1e-8:
        raise ValueError("the kernel uses eps = 1e-8")
    data = _grid_parts(grid_data)
    res = [int(r) for r in grid_res]
    verts = active_vertices.to(torch.int64).contiguous()
    if accumulate_grad is not None:
        target = accumulate_grad.squeeze(0).squeeze(0) if accumulate_grad.dim() == 5 else accumulate_grad
        losses = ops.reg_list("eikonal", data, verts, _eps_host(voxel_size), weight, target)
        return losses[0], None
    g = torch.zeros(res, device=data.device)
    losses = ops.reg_list("eikonal", data, verts, _eps_host(voxel_size), 1.0, g)
    return losses[0], g.reshape(1, 1, *res)


def compute_curvature_loss_and_gradient(grid_data, active_vertices, voxel_size, grid_res,
                                        accumulate_grad: Optional[torch.Tensor] = None, weight: float = 1.0):
    """Closed-form Laplacian curvature loss and gradient (regularization/curvature.py:13-165)."""
    data = _grid_parts(grid_data)
    res = [int(r) for r in grid_res]
    verts = active_vertices.to(torch.int64).contiguous()
    if accumulate_grad is not None:
        target = accumulate_grad.squeeze(0).squeeze(0) if accumulate_grad.dim() == 5 else accumulate_grad
        losses = ops.reg_list("curvature", data, verts, _eps_host(voxel_size), weight, target)
        return losses[1], None
    g = torch.zeros(res, device=data.device)
    losses = ops.reg_list("curvature", data, verts, _eps_host(voxel_size), 1.0, g)
    return losses[1], g.reshape(1, 1, *res)

"""The reference extension's Python seam (voxneus/cuda/__init__.py:25-106) on this library.

A maintainer drops these in with
    voxneus.geometry.gradients.cuda_gradient_interp = voxneus_b200.cuda.cuda_gradient_interp
    voxneus.regularization.eikonal.cuda_eikonal_grad = voxneus_b200.cuda.cuda_eikonal_grad
    voxneus.regularization.curvature.cuda_curvature_grad = voxneus_b200.cuda.cuda_curvature_grad
Unlike the reference seam, which returns None/False when its backend is missing, these raise
when the library or the device is missing (there is no fallback on this path).
"""

from __future__ import annotations

import torch

from . import _lib, ops

GradientInterpFunction = ops.GradientInterpFunction


def is_cuda_available() -> bool:
    return torch.cuda.is_available() and __import__("os").path.exists(_lib.library_path())


def cuda_gradient_interp(grid: torch.Tensor, coords: torch.Tensor, voxel_size: torch.Tensor):
    if not grid.is_cuda:
        return None
    return GradientInterpFunction.apply(grid, coords, voxel_size)


def _reg(kind, grid, active_verts, grad_grid, voxel_size, weight):
    if not grid.is_cuda:
        return False
    data = (grid.squeeze(0).squeeze(0) if grid.dim() == 5 else grid).detach().contiguous()
    target = grad_grid.squeeze(0).squeeze(0) if grad_grid.dim() == 5 else grad_grid
    eps = [float(v) for v in voxel_size.detach().float().cpu()]
    ops.reg_list(kind, data, active_verts.to(torch.int64).contiguous(), eps, weight, target)
    return True


def cuda_eikonal_grad(grid, active_verts, grad_grid, voxel_size, weight: float = 1.0) -> bool:
    return _reg("eikonal", grid, active_verts, grad_grid, voxel_size, weight)


def cuda_curvature_grad(grid, active_verts, grad_grid, voxel_size, weight: float = 1.0) -> bool:
    return _reg("curvature", grid, active_verts, grad_grid, voxel_size, weight)

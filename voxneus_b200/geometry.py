"""Geometry primitives of the hot path (reference voxneus/geometry/*), backed by the sm_100a library.

Same names, arguments and return shapes as the reference functions; every tensor must be on a
CUDA device.
"""

from __future__ import annotations

from typing import List, Tuple, Union

import torch

from . import ops


def world_to_grid_index(xyz, xyz_min, xyz_max, grid_res):
    """Continuous grid-index coordinates (geometry/coordinates.py:10-29); elementwise plumbing."""
    return (xyz - xyz_min) / (xyz_max - xyz_min + 1e-8) * (grid_res - 1.0)


def get_voxel_corners_and_weights(continuous_coords: torch.Tensor, grid_res) -> Tuple[torch.Tensor, torch.Tensor]:
    """8 corner indices (..., 8, 3) int64 and trilinear weights (..., 8) (coordinates.py:55-124)."""
    return ops.corners_weights(continuous_coords, grid_res)


def interpolate_gradients(grid, continuous_coords, voxel_size, grid_res):
    """Eq.7 at grid-index coordinates (geometry/gradients.py:103-139).

    Returns (grad_interp, normals, corner_indices, weights) like the reference.
    """
    lead = continuous_coords.shape[:-1]
    g = ops.GradientInterpFunction.apply(grid, continuous_coords.reshape(-1, 3), voxel_size).reshape(*lead, 3)
    normals = g / (torch.linalg.norm(g, dim=-1, keepdim=True) + 1e-8)
    corners, weights = get_voxel_corners_and_weights(continuous_coords, grid_res)
    return g, normals, corners, weights


def upsample_sdf_grid(grid_tensor: torch.Tensor, new_res: Union[List[int], Tuple[int, int, int], int]) -> torch.Tensor:
    """Trilinear align_corners upsampling (geometry/upsample.py:12-39) on the device."""
    with torch.no_grad():
        return ops.grid_upsample(grid_tensor, new_res)


def get_resolution_for_step(step: int, milestones=(10000, 30000), resolutions=(96, 160, 320)) -> int:
    """Paper resolution schedule (geometry/upsample.py:42-63); host logic."""
    if step < milestones[0]:
        return resolutions[0]
    if step < milestones[1]:
        return resolutions[1]
    return resolutions[2]

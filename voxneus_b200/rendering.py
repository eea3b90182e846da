"""Rendering API of the hot path (reference voxneus/rendering/*), backed by the sm_100a library."""

from __future__ import annotations

from typing import Any, Dict, Optional, Tuple

import torch
import torch.nn as nn

from . import ops


def near_far_from_sphere(rays_o, rays_d, radius: float = 1.0, default_near: float = 0.05, default_far: float = 4.0):
    """rendering/rays.py:102-128."""
    if default_near != 0.05:
        raise ValueError("the kernel uses default_near = 0.05 (rays.py:106)")
    return ops.near_far_from_sphere(rays_o, rays_d, radius)


def sample_pdf(bins, weights, n_samples: int, det: bool = False, eps: float = 1e-5, u=None):
    """Inverse-CDF sampling (rendering/sampler.py:11-66); `u` replaces the torch.rand draw."""
    if eps != 1e-5:
        raise ValueError("the kernel uses eps = 1e-5 (sampler.py:16)")
    return ops.sample_pdf(bins, weights, n_samples, det=det, u=u)


def up_sample(rays_o, rays_d, z_vals, sdf, n_importance: int, inv_s: float, det: bool = True,
              occupancy_grid: Optional[Any] = None, u=None):
    """One NeuS upsampling step (rendering/sampler.py:243-292)."""
    occ = None if occupancy_grid is None else occupancy_grid.occupancy_mask
    lo, hi = (None, None) if occupancy_grid is None else occupancy_grid.bounds()
    return ops.up_sample(rays_o, rays_d, z_vals, sdf, n_importance, inv_s, det=det, u=u, occupancy=occ, occ_min=lo,
                         occ_max=hi)


def cat_z_vals(rays_o, rays_d, z_vals, new_z_vals, sdf, sdf_fn, last: bool = False):
    """Concatenate, sort and query (rendering/sampler.py:295-320): the caller's sdf_fn evaluates the
    new points (unless last), one kernel sorts the depths and carries the SDF values along."""
    nr, ni = new_z_vals.shape
    if last:
        z, _ = ops.cat_z_vals(z_vals, new_z_vals)
        return z, sdf
    pts = rays_o[:, None, :] + rays_d[:, None, :] * new_z_vals[..., :, None]
    fnew = sdf_fn(pts.reshape(-1, 3)).reshape(nr, ni)
    return ops.cat_z_vals(z_vals, new_z_vals, sdf, fnew)


class RaySampler(nn.Module):
    """Stratified + multistep NeuS sampler (rendering/sampler.py:69-204)."""

    def __init__(self, n_samples: int = 64, n_importance: int = 64, perturb: bool = True):
        super().__init__()
        self.n_samples = n_samples
        self.n_importance = n_importance
        self.perturb = perturb

    def sample_multistep_sdf(self, rays_o, rays_d, near, far, sdf_fn, n_samples=None, n_importance=None,
                             up_sample_steps=4, perturb=None, occupancy_grid=None, randoms=None):
        """(z_vals, dists, mid_z_vals). sdf_fn must be DenseSDFGrid.sdf_fn() of this package (or a
        DenseSDFGrid): the kernel samples that grid directly."""
        grid_module = getattr(sdf_fn, "grid_module", None)
        if grid_module is None and hasattr(sdf_fn, "grid") and hasattr(sdf_fn, "bounds"):
            grid_module = sdf_fn
        if grid_module is None:
            raise TypeError("sdf_fn must be DenseSDFGrid.sdf_fn() (the fused sampler reads the grid itself)")
        n_samples = n_samples or self.n_samples
        n_importance = self.n_importance if n_importance is None else n_importance
        perturb = self.perturb if perturb is None else perturb
        t_rand = u = None
        if perturb:
            if randoms is None:
                per = max(n_importance // up_sample_steps, 1) if (n_importance > 0 and up_sample_steps > 0) else 0
                t_rand = torch.rand(rays_o.shape[0], n_samples, device=rays_o.device)
                u = torch.stack([torch.rand(rays_o.shape[0], per, device=rays_o.device)
                                 for _ in range(up_sample_steps)]) if per else None
            else:
                t_rand, u = randoms
        occ = None if occupancy_grid is None else occupancy_grid.occupancy_mask
        olo, ohi = (None, None) if occupancy_grid is None else occupancy_grid.bounds()
        lo, hi = grid_module.bounds()
        with torch.no_grad():
            return ops.sample_multistep(grid_module.grid.detach(), lo, hi, rays_o, rays_d, near, far, n_samples,
                                        n_importance, up_sample_steps, perturb, t_rand, u, occ, olo, ohi)


def compute_neus_alpha(sdf, normals, ray_dirs, dists, s, cos_anneal_ratio: float = 0.0,
                       use_iter_cos_annealing: bool = False, eps: float = 1e-5):
    """Eq.2 (rendering/neus_alpha.py:12-81) for any leading shape."""
    if eps != 1e-5:
        raise ValueError("the kernel uses eps = 1e-5")
    lead = normals.shape[:-1]
    p = normals.numel() // 3
    if not isinstance(s, torch.Tensor):
        s = torch.tensor(float(s), device=normals.device)
    dirs = ray_dirs.expand(*lead, 3).reshape(p, 3)
    a = ops.NeusAlphaFn.apply(sdf.reshape(p, 1), normals.reshape(p, 1, 3), dirs, dists.reshape(p, 1), s,
                              use_iter_cos_annealing, cos_anneal_ratio)
    return a.reshape(lead)


def composite_weights(alpha: torch.Tensor, eps: float = 1e-7) -> Tuple[torch.Tensor, torch.Tensor]:
    """(weights, transmittance) (rendering/volume_render.py:12-40)."""
    if eps != 1e-7:
        raise ValueError("the kernel uses eps = 1e-7")
    return ops.CompositeWeightsFn.apply(alpha)


def compute_huber_color_loss(pred_rgb, target_rgb, delta: float = 0.1):
    """NeuS2 Huber loss (rendering/volume_render.py:43-54): one fused loss + gradient kernel."""
    return ops.HuberLossFn.apply(pred_rgb, target_rgb, delta)


def volume_render_from_samples(colors, sdf, normals, ray_dirs, z_vals, dists, s, pts=None, sphere_radius=1.0,
                               background_rgb=None, cos_anneal_ratio: float = 0.0,
                               use_iter_cos_annealing: bool = False) -> Dict[str, torch.Tensor]:
    """Fused alpha + transmittance + compositing (rendering/volume_render.py:57-153)."""
    if not isinstance(s, torch.Tensor):
        s = torch.tensor(float(s), device=z_vals.device)
    radius = float(sphere_radius) if (pts is not None and sphere_radius is not None and sphere_radius > 0) else 0.0
    outs = ops.CompositeFn.apply(colors, sdf, normals, s, ray_dirs, z_vals.contiguous(), dists.contiguous(),
                                 pts if radius > 0 else None, None, False, 0.0, radius, background_rgb,
                                 use_iter_cos_annealing, cos_anneal_ratio, 0.0, None)
    keys = ("rgb", "depth", "normal", "opacity", "weights", "alpha", "transmittance")
    return dict(zip(keys, outs))

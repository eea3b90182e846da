"""Seeded synthetic inputs for the benchmark workloads (no datasets are involved).

* cameras on a radius-3 hemisphere aimed at the origin, OpenCV convention (x right, y down,
  z forward) as in the reference's DTU ray sampling (datasets/dtu.py:230-241), pixel centres
  at +0.5 (rendering/rays.py:41-46);
* SDF grids: a noisy sphere, a union of random spheres and boxes, a union of Gaussian-bump
  perturbed spheres.
"""

from __future__ import annotations

import math
from typing import List, Tuple

import torch


def hemisphere_cameras(n_cams: int, radius: float = 3.0) -> List[Tuple[torch.Tensor, torch.Tensor]]:
    """(position, rotation camera->world with columns right, down, forward) per camera."""
    cams = []
    for c in range(n_cams):
        el = math.radians(5.0 + 80.0 * (c + 0.5) / n_cams)
        az = 2.0 * math.pi * ((c * 0.618034) % 1.0)
        pos = torch.tensor([radius * math.cos(el) * math.cos(az), radius * math.cos(el) * math.sin(az),
                            radius * math.sin(el)], dtype=torch.float64)
        fwd = -pos / pos.norm()
        up = torch.tensor([0.0, 0.0, 1.0], dtype=torch.float64)
        right = torch.linalg.cross(fwd, up)
        right = right / right.norm()
        down = torch.linalg.cross(fwd, right)
        cams.append((pos, torch.stack([right, down, fwd], dim=1)))
    return cams


class RayPool:
    """Uniform (camera, pixel) ray batches from a fixed camera rig."""

    def __init__(self, n_cams: int = 64, width: int = 800, height: int = 600, focal: float = 700.0, seed: int = 0):
        self.cams = hemisphere_cameras(n_cams)
        self.pos = torch.stack([p for p, _ in self.cams]).float()
        self.rot = torch.stack([r for _, r in self.cams]).float()
        self.w, self.h, self.f = width, height, focal
        self.gen = torch.Generator().manual_seed(seed)

    def sample(self, n_rays: int) -> Tuple[torch.Tensor, torch.Tensor]:
        ci = torch.randint(0, len(self.cams), (n_rays,), generator=self.gen)
        px = torch.randint(0, self.w, (n_rays,), generator=self.gen).float() + 0.5
        py = torch.randint(0, self.h, (n_rays,), generator=self.gen).float() + 0.5
        return self.rays_for(ci, px, py)

    def rays_for(self, ci, px, py):
        v = torch.stack([(px - self.w / 2) / self.f, (py - self.h / 2) / self.f, torch.ones_like(px)], -1)
        d = torch.einsum("nij,nj->ni", self.rot[ci], v)
        d = d / d.norm(dim=-1, keepdim=True)
        return self.pos[ci].clone(), d.contiguous()

    def view(self, cam: int, stride: int = 1) -> Tuple[torch.Tensor, torch.Tensor]:
        """All pixel rays of one camera (every `stride`-th pixel)."""
        ys, xs = torch.meshgrid(torch.arange(0, self.h, stride), torch.arange(0, self.w, stride), indexing="ij")
        px = xs.reshape(-1).float() + 0.5
        py = ys.reshape(-1).float() + 0.5
        ci = torch.full_like(xs.reshape(-1), cam)
        return self.rays_for(ci, px, py)


def _lattice(res: int) -> torch.Tensor:
    ax = torch.linspace(-1.0, 1.0, res)
    gx, gy, gz = torch.meshgrid(ax, ax, ax, indexing="ij")
    return torch.stack([gx, gy, gz], -1)


def sphere_grid(res: int, radius: float = 0.5, noise: float = 0.01, seed: int = 0) -> torch.Tensor:
    """||x|| - r + N(0, noise) on a res^3 lattice over [-1,1]^3, shaped (1,1,R,R,R)."""
    g = torch.Generator().manual_seed(seed)
    f = _lattice(res).norm(dim=-1) - radius
    return (f + noise * torch.randn(f.shape, generator=g)).reshape(1, 1, res, res, res)


def shapes_grid(res: int, n_shapes: int = 8, noise: float = 0.005, seed: int = 0) -> torch.Tensor:
    """Union (min) of random spheres and axis-aligned boxes + N(0, noise), (1,1,R,R,R)."""
    g = torch.Generator().manual_seed(seed)
    p = _lattice(res)
    f = torch.full(p.shape[:-1], 1e9)
    for i in range(n_shapes):
        c = (torch.rand(3, generator=g) - 0.5) * 1.0
        if i % 2 == 0:
            r = 0.1 + 0.2 * float(torch.rand(1, generator=g))
            fi = (p - c).norm(dim=-1) - r
        else:
            h = 0.08 + 0.17 * torch.rand(3, generator=g)
            q = (p - c).abs() - h
            fi = q.clamp(min=0).norm(dim=-1) + q.max(dim=-1).values.clamp(max=0)
        f = torch.minimum(f, fi)
    return (f + noise * torch.randn(f.shape, generator=g)).reshape(1, 1, res, res, res)


def bumpy_spheres_grid(res: int, n_spheres: int = 32, seed: int = 0, device="cpu") -> torch.Tensor:
    """min_k ||x - c_k|| - r_k (1 + a_k exp(-||x - p_k||^2 / s_k^2)), (1,1,R,R,R).

    Shape parameters come from a CPU generator (seeded); the field is evaluated on `device`.
    """
    g = torch.Generator().manual_seed(seed)
    ax = torch.linspace(-1.0, 1.0, res, device=device)
    f = torch.full((res, res, res), 1e9, device=device)
    for _ in range(n_spheres):
        c = ((torch.rand(3, generator=g) - 0.5) * 1.2).tolist()
        r = 0.1 + 0.3 * float(torch.rand(1, generator=g))
        a = (float(torch.rand(1, generator=g)) - 0.5) * 0.2
        s = 0.05 + 0.15 * float(torch.rand(1, generator=g))
        pk = [c[i] + r * v for i, v in enumerate(torch.nn.functional.normalize(torch.randn(3, generator=g), dim=0).tolist())]
        for i0 in range(0, res, 64):  # slabs keep the temporaries small at 512^3
            x = ax[i0:i0 + 64].view(-1, 1, 1)
            y = ax.view(1, -1, 1)
            z = ax.view(1, 1, -1)
            dc = torch.sqrt((x - c[0]) ** 2 + (y - c[1]) ** 2 + (z - c[2]) ** 2)
            dp = (x - pk[0]) ** 2 + (y - pk[1]) ** 2 + (z - pk[2]) ** 2
            fi = dc - r * (1.0 + a * torch.exp(-dp / (s * s)))
            f[i0:i0 + 64] = torch.minimum(f[i0:i0 + 64], fi)
    return f.reshape(1, 1, res, res, res)


def throughput_scene(res: int, device, seed: int = 0, hash_log2_size: int = 19, occupancy_res: int = 128):
    """The training-throughput scene: a (res/2)^3 union of 8 random spheres/boxes + N(0, 0.005),
    upsampled on the device to res^3 by trilinear interpolation (geometry/upsample.py:12-39), a
    16-level hash table of 2^hash_log2_size entries initialised U(-1e-2, 1e-2), default MLP and s.

    Returns (model, milliseconds of the upsampling launch)."""
    from .models import VoxNeuS

    torch.manual_seed(seed)
    m = VoxNeuS(grid_res=res // 2, hash_log2_size=hash_log2_size, occupancy_res=occupancy_res).to(device)
    with torch.no_grad():
        m.sdf_grid.grid.copy_(shapes_grid(res // 2, seed=seed).to(device))
        m.radiance_hash.encoder.embeddings.uniform_(-1e-2, 1e-2)
    t0 = torch.cuda.Event(enable_timing=True)
    t1 = torch.cuda.Event(enable_timing=True)
    t0.record()
    m.sdf_grid.scale_volume_grid(res)
    t1.record()
    torch.cuda.synchronize()
    return m, t0.elapsed_time(t1)

"""VoxNeuS modules on the sm_100a path (reference voxneus/models/*).

Parameter and buffer names match the reference state_dict (sdf_grid.grid,
variance_net.variance, radiance_hash.encoder.embeddings, radiance_mlp.net.{0,2}.*,
occupancy_grid.*), so reference checkpoints load unchanged. Geometry, sampling,
compositing, the hash encoding and the 2-layer radiance MLP (on the tcgen05 tensor cores) run in
the library's kernels, each with its hand-written adjoint.
"""

from __future__ import annotations

from typing import Dict, List, Optional, Tuple

import torch
import torch.nn as nn

from . import ops


def _res_list(resolution) -> List[int]:
    return [int(resolution)] * 3 if isinstance(resolution, int) else [int(r) for r in resolution]


class GridSDF:
    """sdf_fn callable bound to a DenseSDFGrid: p (P,3) -> SDF (P,) (models/voxneus.py:211-212)."""

    def __init__(self, grid_module: "DenseSDFGrid"):
        self.grid_module = grid_module

    def __call__(self, p: torch.Tensor) -> torch.Tensor:
        return self.grid_module.query_sdf(p).squeeze(-1)


def _dense_grid_of(fn) -> Optional["DenseSDFGrid"]:
    """The DenseSDFGrid behind a query_sdf bound method or a GridSDF, else None."""
    if isinstance(fn, GridSDF):
        return fn.grid_module
    owner = getattr(fn, "__self__", None)
    if isinstance(owner, DenseSDFGrid) and getattr(fn, "__func__", None) is DenseSDFGrid.query_sdf:
        return owner
    return None


class DenseSDFGrid(nn.Module):
    """Dense FP32 SDF grid (models/sdf_grid.py:24-199)."""

    def __init__(self, resolution=96, xyz_min=(-1.0, -1.0, -1.0), xyz_max=(1.0, 1.0, 1.0), init_mode="sphere",
                 sphere_radius=0.5, feat_dim=0):
        super().__init__()
        if feat_dim:
            raise NotImplementedError("geometry feature grids (feat_dim > 0) are not on the fused path")
        self.res = torch.tensor(_res_list(resolution), dtype=torch.float32)
        self.register_buffer("xyz_min", torch.tensor(xyz_min, dtype=torch.float32))
        self.register_buffer("xyz_max", torch.tensor(xyz_max, dtype=torch.float32))
        self.init_mode = init_mode
        self.sphere_radius = sphere_radius
        self.feat_dim = 0
        self.feat_grid = None
        r = _res_list(resolution)
        self.grid = nn.Parameter(torch.zeros([1, 1, *r], dtype=torch.float32))
        self._bounds = (tuple(float(v) for v in xyz_min), tuple(float(v) for v in xyz_max))
        self.reset_parameters()

    def reset_parameters(self):
        """Sphere / zero / uniform initialisation (models/sdf_grid.py:59-81)."""
        r = [int(v) for v in self.res]
        lo, hi = self._bounds
        if self.init_mode == "sphere":
            axes = [torch.linspace(lo[a], hi[a], r[a]) for a in range(3)]
            gx, gy, gz = torch.meshgrid(*axes, indexing="ij")
            d = torch.linalg.norm(torch.stack([gx, gy, gz], -1), dim=-1) - self.sphere_radius
            with torch.no_grad():
                self.grid.data.copy_(d.reshape(self.grid.shape))
        elif self.init_mode == "zero":
            with torch.no_grad():
                self.grid.data.zero_()
        else:
            with torch.no_grad():
                self.grid.data.uniform_(-0.05, 0.05)

    def bounds(self) -> Tuple[Tuple[float, ...], Tuple[float, ...]]:
        return self._bounds

    def _load_from_state_dict(self, state_dict, prefix, *args, **kwargs):
        super()._load_from_state_dict(state_dict, prefix, *args, **kwargs)
        self._bounds = (tuple(float(v) for v in self.xyz_min.cpu()), tuple(float(v) for v in self.xyz_max.cpu()))

    @property
    def voxel_size(self) -> torch.Tensor:
        return (self.xyz_max - self.xyz_min) / (self.res.to(self.xyz_min.device) - 1.0)

    def voxel_size_host(self) -> List[float]:
        lo, hi = self._bounds
        r = [int(v) for v in self.res]
        return [float(torch.tensor(hi[a] - lo[a], dtype=torch.float32) / (torch.tensor(float(r[a])) - 1.0))
                for a in range(3)]

    def sdf_fn(self) -> GridSDF:
        return GridSDF(self)

    def query_sdf(self, xyz: torch.Tensor) -> torch.Tensor:
        """(..., 3) -> (..., 1), grid_sample semantics (models/sdf_grid.py:90-120)."""
        return ops.SdfQueryFn.apply(self.grid, xyz, *self._bounds)

    def query_normals(self, xyz: torch.Tensor, gradient_mode: str = "interpolated", return_corners: bool = True):
        """(grad, normal, corner_indices, weights) (models/sdf_grid.py:122-160)."""
        if gradient_mode.lower() != "interpolated":
            raise ValueError("the fused path implements the interpolated (Eq.7) gradient mode only")
        grad, normal = ops.NormalsFn.apply(self.grid, xyz, *self._bounds)
        corners = weights = None
        if return_corners:
            _, _, _, corners, weights = ops.field_query(self.grid.detach(), *self._bounds,
                                                        xyz.detach().reshape(-1, 3).contiguous(), sdf=False,
                                                        corners=True, weights=True)
            lead = xyz.shape[:-1]
            corners = corners.reshape(*lead, 8, 3)
            weights = weights.reshape(*lead, 8)
        return grad, normal, corners, weights

    def scale_volume_grid(self, new_resolution):
        """Trilinear super-resolution (models/sdf_grid.py:183-195)."""
        up = ops.grid_upsample(self.grid, new_resolution)
        self.grid = nn.Parameter(up)
        self.res = torch.tensor(_res_list(new_resolution), dtype=torch.float32)

    def get_numpy_grid(self):
        return self.grid.detach().squeeze().cpu().numpy()


class SingleVarianceNetwork(nn.Module):
    """s = clamp(exp(10 v), 1e-4, s_max) (models/variance.py:11-46)."""

    def __init__(self, init_val: float = 0.3, s_max: float = 300.0):
        super().__init__()
        self.variance = nn.Parameter(torch.tensor(init_val, dtype=torch.float32))
        self._s_max = float(s_max)

    @property
    def s(self) -> torch.Tensor:
        return torch.clamp(torch.exp(self.variance * 10.0), min=1e-4, max=self._s_max)

    @property
    def std(self) -> torch.Tensor:
        return 1.0 / self.s

    def forward(self, x=1):
        s = self.s
        if isinstance(x, torch.Tensor):
            return torch.ones_like(x[..., :1]) * s
        return s


class HashEncoder(nn.Module):
    """Parameter holder with the reference PyTorchHashGrid's names (radiance_hash.py:25-69)."""

    def __init__(self, n_levels=16, n_features_per_level=2, log2_hashmap_size=19, base_resolution=16,
                 max_resolution=2048):
        super().__init__()
        self.n_levels = n_levels
        self.n_features_per_level = n_features_per_level
        self.log2_hashmap_size = log2_hashmap_size
        self.out_dim = n_levels * n_features_per_level
        self.register_buffer("primes", torch.tensor([1, 2654435761, 805459861], dtype=torch.int64))
        self.embeddings = nn.Parameter(torch.empty(n_levels, 2 ** log2_hashmap_size, n_features_per_level))
        nn.init.uniform_(self.embeddings, -1e-4, 1e-4)
        self.cfg = ops.HashConfig(n_levels, n_features_per_level, log2_hashmap_size, base_resolution, max_resolution)


class RadianceHashGrid(nn.Module):
    """Multiresolution hash grid with NeuS2 lambda masking (radiance_hash.py:169-231)."""

    def __init__(self, n_levels=16, n_features_per_level=2, log2_hashmap_size=19, base_resolution=16,
                 max_resolution=2048, force_pytorch=False):
        super().__init__()
        self.n_levels = n_levels
        self.n_features_per_level = n_features_per_level
        self.out_dim = n_levels * n_features_per_level
        self.encoder = HashEncoder(n_levels, n_features_per_level, log2_hashmap_size, base_resolution, max_resolution)

    def forward(self, norm_xyz: torch.Tensor, active_levels: Optional[float] = None) -> torch.Tensor:
        return ops.HashEncodeFn.apply(self.encoder.embeddings, norm_xyz, self.encoder.cfg, active_levels)


class SphericalHarmonicsEmbedder(nn.Module):
    """Degree-4 SH (models/embedder.py:47-87)."""

    def __init__(self, degree: int = 4):
        super().__init__()
        if degree != 4:
            raise NotImplementedError("the kernel implements degree 4 (16 coefficients)")
        self.degree = degree
        self.out_dim = 16

    def forward(self, dirs: torch.Tensor) -> torch.Tensor:
        return ops.sh4(dirs)


class RadianceMLP(nn.Module):
    """[hash, SH, normal] -> 64 ReLU -> 3 Sigmoid (models/radiance_mlp.py:11-98)."""

    def __init__(self, hash_feature_dim=32, view_embed_dim=16, normal_dim=3, geom_feature_dim=0, hidden_dim=64,
                 num_layers=2, weight_norm=False, entangled=False):
        super().__init__()
        if geom_feature_dim or entangled or num_layers != 2 or weight_norm:
            raise NotImplementedError("the fused path implements the default 2-layer disentangled MLP")
        in_dim = hash_feature_dim + view_embed_dim + normal_dim
        self.net = nn.Sequential(nn.Linear(in_dim, hidden_dim), nn.ReLU(inplace=True), nn.Linear(hidden_dim, 3),
                                 nn.Sigmoid())
        for m in self.net.modules():
            if isinstance(m, nn.Linear):
                nn.init.kaiming_uniform_(m.weight, nonlinearity="relu")
                nn.init.zeros_(m.bias)

    def forward(self, hash_features, view_embeddings, normals, geom_features=None, sdf=None):
        """models/radiance_mlp.py:81-98 on the fused tensor-core MLP (forward and adjoint). The
        adjoint gives the gradients of the hash features, the normals and the weights; the view
        embedding (SH of the ray directions) takes none, as in the reference's training."""
        if view_embeddings.requires_grad:
            raise NotImplementedError("the fused MLP adjoint gives no gradient for the view embedding")
        x = torch.cat([hash_features, view_embeddings, normals], dim=-1)
        lead = x.shape[:-1]
        l0, l1 = self.net[0], self.net[2]
        out = ops.RadianceMLPFn.apply(x.reshape(-1, x.shape[-1]), l0.weight, l0.bias, l1.weight, l1.bias)
        return out.reshape(*lead, 3)


class OccupancyGrid(nn.Module):
    """NeuS2 occupancy bitmask (rendering/occupancy_grid.py:25-150); the lookup runs in the sampler."""

    def __init__(self, resolution=128, xyz_min=(-1.0, -1.0, -1.0), xyz_max=(1.0, 1.0, 1.0), decay=0.95,
                 threshold=0.01):
        super().__init__()
        self.resolution = resolution
        self.register_buffer("xyz_min", torch.tensor(xyz_min, dtype=torch.float32))
        self.register_buffer("xyz_max", torch.tensor(xyz_max, dtype=torch.float32))
        self.decay = decay
        self.threshold = threshold
        self.register_buffer("density_grid", torch.zeros((resolution,) * 3, dtype=torch.float32))
        self.register_buffer("occupancy_mask", torch.ones((resolution,) * 3, dtype=torch.bool))
        self.total_updates = 0
        self._bounds = (tuple(float(v) for v in xyz_min), tuple(float(v) for v in xyz_max))

    def _load_from_state_dict(self, state_dict, prefix, *args, **kwargs):
        super()._load_from_state_dict(state_dict, prefix, *args, **kwargs)
        self._bounds = (tuple(float(v) for v in self.xyz_min.cpu()), tuple(float(v) for v in self.xyz_max.cpu()))

    def bounds(self):
        return self._bounds

    @property
    def occupied_percentage(self) -> float:
        return float(self.occupancy_mask.float().mean().item() * 100.0)

    @torch.no_grad()
    def update_from_sdf(self, query_sdf_fn, s_val, subsample_ratio: float = 0.25, generator=None) -> None:
        """EMA update with the NeuS2 logistic density (rendering/occupancy_grid.py:62-119).

        Draws max(int(R^3 * subsample_ratio), 1024) cells with three torch.randint calls (x, y, z,
        the reference's order, from `generator` or the default generator of the grid's device).
        query_sdf_fn: a DenseSDFGrid's query_sdf (or its GridSDF) is evaluated inside the kernel;
        any other callable (N,3) -> (N,1) or (N,) is called on the cell centres. s_val: s as a
        tensor or number, or a SingleVarianceNetwork (s derived from its parameter on the device).
        """
        dev = self.density_grid.device
        res = self.resolution
        n = max(int(res * res * res * subsample_ratio), 1024)
        idx = [torch.randint(0, res, (n,), device=dev, generator=generator) for _ in range(3)]
        lo, hi = self._bounds
        if isinstance(s_val, SingleVarianceNetwork):
            s, is_var, s_max = s_val.variance.detach(), True, s_val._s_max
        else:
            s, is_var, s_max = torch.as_tensor(s_val).detach().to(device=dev, dtype=torch.float32), False, 0.0
        grid_mod = _dense_grid_of(query_sdf_fn)
        if grid_mod is not None:
            kw = dict(grid=grid_mod.grid.detach(), grid_bounds=grid_mod.bounds())
        else:
            pts = ops.occupancy_points(res, lo, hi, idx)
            kw = dict(sdf_values=query_sdf_fn(pts).detach().reshape(-1).float().contiguous())
        ops.occupancy_update(self.density_grid, self.occupancy_mask, idx, lo, hi, s, is_var, s_max,
                             self.total_updates == 0, self.decay, self.threshold, **kw)
        self.total_updates += 1

    @torch.no_grad()
    def is_occupied(self, pts_world: torch.Tensor) -> torch.Tensor:
        """(..., 3) world points -> (...) bool (rendering/occupancy_grid.py:121-147)."""
        lo, hi = self._bounds
        return ops.occupancy_query(self.occupancy_mask, lo, hi, pts_world)


class VoxNeuS(nn.Module):
    """Assembled model (models/voxneus.py:21-260) with the fused render."""

    def __init__(self, grid_res=96, xyz_min=(-1.0, -1.0, -1.0), xyz_max=(1.0, 1.0, 1.0), gradient_mode="interpolated",
                 init_s_val=0.3, s_max=300.0, hash_n_levels=16, hash_n_features=2, hash_log2_size=19,
                 geom_feature_dim=0, mlp_hidden_dim=64, view_embed_type="sh", entangled=False, occupancy_res=128,
                 force_pytorch=False):
        super().__init__()
        if gradient_mode != "interpolated" or view_embed_type != "sh" or geom_feature_dim or entangled:
            raise NotImplementedError("the fused path implements the default VoxNeuS configuration")
        self.gradient_mode = gradient_mode
        self.sdf_grid = DenseSDFGrid(grid_res, xyz_min, xyz_max, init_mode="sphere")
        self.variance_net = SingleVarianceNetwork(init_s_val, s_max)
        self.occupancy_grid = OccupancyGrid(occupancy_res, xyz_min, xyz_max)
        self.radiance_hash = RadianceHashGrid(hash_n_levels, hash_n_features, hash_log2_size)
        self.view_embedder = SphericalHarmonicsEmbedder(4)
        self.radiance_mlp = RadianceMLP(self.radiance_hash.out_dim, 16, 3, 0, mlp_hidden_dim)

    @property
    def s(self):
        return self.variance_net.s

    @property
    def std(self):
        return self.variance_net.std

    @torch.no_grad()
    def update_occupancy_grid(self, subsample_ratio: float = 0.25, generator=None) -> None:
        """Periodic occupancy refresh from the SDF grid and the current s (models/voxneus.py:104-113);
        s is derived from the variance parameter inside the kernel."""
        self.occupancy_grid.update_from_sdf(self.sdf_grid.query_sdf, self.variance_net, subsample_ratio,
                                            generator=generator)

    def draw_sampler_randoms(self, n_rays: int, n_samples: int, n_importance: int, steps: int, device,
                             generator=None):
        """The uniforms the reference sampler draws, in its order (sampler.py:117, then :44 per step)."""
        t_rand = torch.rand((n_rays, n_samples), device=device, generator=generator)
        per = max(n_importance // steps, 1) if (n_importance > 0 and steps > 0) else 0
        u = None
        if per:  # each step's draw written in place into its slice (the same values as separate tensors)
            u = torch.empty((steps, n_rays, per), device=device)
            for k in range(steps):
                torch.rand((n_rays, per), device=device, generator=generator, out=u[k])
        return t_rand, u

    def render(self, rays_o, rays_d, sampler, near=None, far=None, background_rgb=None, cos_anneal_ratio=0.0,
               use_iter_cos_annealing=False, active_levels=None, up_sample_steps=4, sphere_radius=1.0,
               *, randoms=None, vr_bitmap=None, extras=True, amplify_k=0.0, amp_flag=None,
               z_vals=None) -> Dict[str, torch.Tensor]:
        """Fused render (models/voxneus.py:169-260).

        near/far None: computed from the unit sphere inside the sampler kernel. randoms:
        (t_rand, u) uniforms for a perturbed sampler (drawn in the reference order when None).
        vr_bitmap: V_R bitmap receiving every sample's Eq.7 corners. extras: also return pts,
        sdf_samples, corner_indices, grad_samples, normal_samples like the reference; with
        extras=False the per-sample weights, alpha and transmittance are not written (None).
        z_vals: (N_rays, S) sorted sample depths to render instead of running the sampler (as the
        reference sampler returns them); their dists and midpoints are formed as in
        rendering/sampler.py:197-202.
        """
        dev = rays_o.device
        o = rays_o.contiguous()
        d = rays_d.contiguous()
        nr = o.shape[0]
        lo, hi = self.sdf_grid.bounds()
        ns, ni = sampler.n_samples, sampler.n_importance
        perturb = sampler.perturb
        t_rand = u = None
        if z_vals is not None:
            with torch.no_grad():
                z = z_vals.detach().to(torch.float32).contiguous()
                dists = torch.cat([z[:, 1:] - z[:, :-1], z[:, -1:] - z[:, -2:-1]], dim=-1)
                mid = z + dists * 0.5
        else:
            if perturb:
                t_rand, u = (randoms if randoms is not None
                             else self.draw_sampler_randoms(nr, ns, ni, up_sample_steps, dev))
            occ = self.occupancy_grid
            with torch.no_grad():
                _, dists, mid = ops.sample_multistep(self.sdf_grid.grid.detach(), lo, hi, o, d, near, far, ns, ni,
                                                     up_sample_steps, perturb, t_rand, u, occ.occupancy_mask,
                                                     *occ.bounds(), want_z=False)
        handoff = ops.NormalGradHandoff(torch.is_grad_enabled())
        sdf, normal, gsamp = ops.RenderGeometryFn.apply(self.sdf_grid.grid, o, d, mid, lo, hi, vr_bitmap, extras,
                                                        handoff)
        l0, l1 = self.radiance_mlp.net[0], self.radiance_mlp.net[2]
        colors = ops.AppearanceMLPFn.apply(self.radiance_hash.encoder.embeddings, normal, l0.weight, l0.bias, l1.weight,
                                           l1.bias, o, d, mid, lo, hi, self.radiance_hash.encoder.cfg, active_levels,
                                           torch.is_grad_enabled(), handoff)
        out_t = ops.CompositeFn.apply(colors, sdf, normal, self.variance_net.variance, d, mid, dists, None, o, True,
                                      self.variance_net._s_max, sphere_radius if sphere_radius else 0.0,
                                      background_rgb, use_iter_cos_annealing, cos_anneal_ratio, amplify_k, amp_flag,
                                      extras)
        keys = ("rgb", "depth", "normal", "opacity", "weights", "alpha", "transmittance")
        out = dict(zip(keys, out_t))
        out["dists"] = dists
        out["mid_z_vals"] = mid
        if extras:
            pts = o.unsqueeze(1) + d.unsqueeze(1) * mid.unsqueeze(-1)
            out["pts"] = pts
            out["sdf_samples"] = sdf.unsqueeze(-1)
            out["grad_samples"] = gsamp
            out["normal_samples"] = normal
            out["corner_indices"] = ops.field_query(self.sdf_grid.grid.detach(), lo, hi, pts.detach().reshape(-1, 3),
                                                    sdf=False, corners=True)[3].reshape(nr, mid.shape[1], 8, 3)
        return out

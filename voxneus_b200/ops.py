"""Tensor-level wrappers of the C ABI and the torch.autograd.Functions of the hot path.

Every function validates its tensors (CUDA, dtype, contiguity) the way the reference
extension's CHECK_INPUT does (voxneus/cuda/adam_upd.cpp:44-46) and launches on the current
torch stream. Nothing here falls back to another implementation.
"""

from __future__ import annotations

import math
import threading
from typing import Dict, Optional, Sequence, Tuple

import torch

from . import _lib as L
from ._lib import call, check_tensor, f3, i3, ptr, stream_ptr

# ------------------------------------------------------------------ scratch memory --------


class Scratch:
    """Per-(device, stream) scratch: block partials and zero-initialised completion counters."""

    _lock = threading.Lock()
    _pool: Dict[Tuple[int, int], "Scratch"] = {}

    def __init__(self, device: torch.device):
        self.device = device
        self.counters = torch.zeros(16, dtype=torch.int32, device=device)
        self.partials = torch.zeros(4096, dtype=torch.float64, device=device)
        self.blocks = torch.zeros(4096, dtype=torch.int32, device=device)

    @classmethod
    def get(cls, device: torch.device) -> "Scratch":
        dev = torch.device(device)
        idx = dev.index if dev.index is not None else torch.cuda.current_device()
        key = (idx, torch.cuda.current_stream(idx).cuda_stream)
        with cls._lock:
            s = cls._pool.get(key)
            if s is None:
                s = cls(torch.device("cuda", idx))
                cls._pool[key] = s
        return s

    def partials_for(self, n: int) -> torch.Tensor:
        if self.partials.numel() < n:
            self.partials = torch.zeros(max(n, 2 * self.partials.numel()), dtype=torch.float64, device=self.device)
        return self.partials

    def blocks_for(self, n: int) -> torch.Tensor:
        if self.blocks.numel() < n:
            self.blocks = torch.zeros(max(n, 2 * self.blocks.numel()), dtype=torch.int32, device=self.device)
        return self.blocks

    def counter(self, i: int):
        return self.counters[i:i + 1]


COUNTER_COMPOSITE, COUNTER_EIK, COUNTER_CURV, COUNTER_STENCIL = 0, 1, 2, 3


def _f(t):
    return check_tensor(t, "tensor")


def _grid3(grid: torch.Tensor):
    check_tensor(grid, "grid")
    res = list(grid.shape[-3:])
    if grid.dim() == 5 and (grid.shape[0] != 1 or grid.shape[1] != 1):
        raise RuntimeError("grid must be (1,1,X,Y,Z) or (X,Y,Z)")
    return res


# ------------------------------------------------------------------ field queries ---------


# Batches of scattered points against grids larger than the L2 cache are queried in Morton order
# (vx_field_query_sorted; bit-identical outputs): at least this many points, this many grid bytes.
SORTED_QUERY_MIN_POINTS = 1 << 20
SORTED_QUERY_MIN_GRID_BYTES = 128 << 20


def field_query_sorted(grid, xyz_min, xyz_max, xyz, sdf=True, grad=False, normal=False):
    """field_query's sdf/grad/normal through the spatially sorted path."""
    res = _grid3(grid)
    xyz = check_tensor(xyz, "xyz")
    n = xyz.numel() // 3
    dev = xyz.device
    need = int(L.query("vx_field_query_sorted_workspace", n, i3(res)))
    if need <= 0:
        raise RuntimeError("vx_field_query_sorted_workspace failed (needs a CUDA device, n < 2^31)")
    ws = torch.empty(need, dtype=torch.uint8, device=dev)
    o_sdf = torch.empty(n, device=dev) if sdf else None
    o_grad = torch.empty(n, 3, device=dev) if grad else None
    o_nrm = torch.empty(n, 3, device=dev) if normal else None
    call("vx_field_query_sorted", ptr(grid), i3(res), f3(xyz_min), f3(xyz_max), ptr(xyz), n, ptr(o_sdf), ptr(o_grad),
         ptr(o_nrm), ptr(ws), need, stream_ptr(dev))
    return o_sdf, o_grad, o_nrm, None, None


def field_query(grid, xyz_min, xyz_max, xyz, sdf=True, grad=False, normal=False, corners=False, weights=False):
    res = _grid3(grid)
    xyz = check_tensor(xyz, "xyz")
    n = xyz.numel() // 3
    if (not corners and not weights and n >= SORTED_QUERY_MIN_POINTS and n < (1 << 31)
            and grid.numel() * 4 >= SORTED_QUERY_MIN_GRID_BYTES):
        return field_query_sorted(grid, xyz_min, xyz_max, xyz, sdf=sdf, grad=grad, normal=normal)
    dev = xyz.device
    o_sdf = torch.empty(n, device=dev) if sdf else None
    o_grad = torch.empty(n, 3, device=dev) if grad else None
    o_nrm = torch.empty(n, 3, device=dev) if normal else None
    o_cor = torch.empty(n, 8, 3, dtype=torch.int64, device=dev) if corners else None
    o_w = torch.empty(n, 8, device=dev) if weights else None
    call("vx_field_query", ptr(grid), i3(res), f3(xyz_min), f3(xyz_max), ptr(xyz), n, ptr(o_sdf), ptr(o_grad),
         ptr(o_nrm), ptr(o_cor), ptr(o_w), stream_ptr(dev))
    return o_sdf, o_grad, o_nrm, o_cor, o_w


def field_query_backward(grid, xyz_min, xyz_max, xyz, d_sdf=None, d_grad=None, d_normal=None, out=None):
    res = _grid3(grid)
    n = xyz.numel() // 3
    if out is None:
        out = torch.zeros(res, device=grid.device)
    for t, nm in ((d_sdf, "d_sdf"), (d_grad, "d_grad"), (d_normal, "d_normal")):
        if t is not None:
            check_tensor(t, nm)
    call("vx_field_query_backward", ptr(grid), i3(res), f3(xyz_min), f3(xyz_max), ptr(xyz), n, ptr(d_sdf),
         ptr(d_grad), ptr(d_normal), ptr(out), stream_ptr(grid.device))
    return out


class SdfQueryFn(torch.autograd.Function):
    """Trilinear SDF (models/sdf_grid.py:90-120) with the grid_sample adjoint."""

    @staticmethod
    def forward(ctx, grid, xyz, xyz_min, xyz_max):
        xyz_c = xyz.detach().reshape(-1, 3).contiguous()
        sdf, _, _, _, _ = field_query(grid.detach(), xyz_min, xyz_max, xyz_c, sdf=True)
        ctx.save_for_backward(grid, xyz_c)
        ctx.bounds = (xyz_min, xyz_max)
        return sdf.reshape(*xyz.shape[:-1], 1)

    @staticmethod
    def backward(ctx, g):
        grid, xyz = ctx.saved_tensors
        gg = None
        if ctx.needs_input_grad[0]:
            gg = field_query_backward(grid.detach(), *ctx.bounds, xyz, d_sdf=g.reshape(-1).contiguous())
            gg = gg.reshape(grid.shape)
        return gg, None, None, None


class NormalsFn(torch.autograd.Function):
    """Eq.7 gradient and normal (models/sdf_grid.py:122-160) with the stencil adjoint."""

    @staticmethod
    def forward(ctx, grid, xyz, xyz_min, xyz_max):
        xyz_c = xyz.detach().reshape(-1, 3).contiguous()
        _, g, n, _, _ = field_query(grid.detach(), xyz_min, xyz_max, xyz_c, sdf=False, grad=True, normal=True)
        ctx.save_for_backward(grid, xyz_c)
        ctx.bounds = (xyz_min, xyz_max)
        lead = xyz.shape[:-1]
        return g.reshape(*lead, 3), n.reshape(*lead, 3)

    @staticmethod
    def backward(ctx, dg, dn):
        grid, xyz = ctx.saved_tensors
        gg = None
        if ctx.needs_input_grad[0]:
            gg = field_query_backward(grid.detach(), *ctx.bounds, xyz,
                                      d_grad=None if dg is None else dg.reshape(-1, 3).contiguous(),
                                      d_normal=None if dn is None else dn.reshape(-1, 3).contiguous())
            gg = gg.reshape(grid.shape)
        return gg, None, None, None


class GradientInterpFunction(torch.autograd.Function):
    """Eq.7 at grid-index coordinates (voxneus/cuda/__init__.py:29-59 interface)."""

    @staticmethod
    def forward(ctx, grid, coords, voxel_size):
        g3 = grid.detach()
        res = _grid3(g3)
        coords_c = check_tensor(coords.detach().contiguous(), "coords")
        eps = [float(v) for v in voxel_size.detach().cpu()] if isinstance(voxel_size, torch.Tensor) else list(voxel_size)
        n = coords_c.numel() // 3
        out = torch.empty(n, 3, device=coords.device)
        call("vx_gradient_interp_forward", ptr(g3), i3(res), ptr(coords_c), n, f3(eps), ptr(out),
             stream_ptr(coords.device))
        ctx.save_for_backward(coords_c)
        ctx.meta = (res, eps, grid.shape)
        return out

    @staticmethod
    def backward(ctx, g):
        (coords,) = ctx.saved_tensors
        res, eps, shape = ctx.meta
        gg = None
        if ctx.needs_input_grad[0]:
            gg = torch.zeros(res, device=g.device)
            gc = check_tensor(g.contiguous(), "grad_out")
            call("vx_gradient_interp_backward", ptr(gc), ptr(coords), coords.numel() // 3, ptr(gg), i3(res), f3(eps),
                 stream_ptr(g.device))
            gg = gg.reshape(shape)
        return gg, None, None


def gradient_interp_raw(grid3, coords, eps):
    res = _grid3(grid3)
    n = coords.numel() // 3
    out = torch.empty(n, 3, device=coords.device)
    call("vx_gradient_interp_forward", ptr(grid3), i3(res), ptr(coords), n, f3(eps), ptr(out),
         stream_ptr(coords.device))
    return out


def corners_weights(coords, grid_res):
    res = [int(r) for r in grid_res]
    lead = coords.shape[:-1]
    c = check_tensor(coords.detach().reshape(-1, 3).contiguous(), "continuous_coords")
    n = c.shape[0]
    corners = torch.empty(n, 8, 3, dtype=torch.int64, device=c.device)
    weights = torch.empty(n, 8, device=c.device)
    call("vx_corners_weights", ptr(c), n, i3(res), ptr(corners), ptr(weights), stream_ptr(c.device))
    return corners.reshape(*lead, 8, 3), weights.reshape(*lead, 8)


def field_query_lattice(grid, xyz_min, xyz_max, lattice, lat_min, lat_max, sdf=True, normal=True):
    res = _grid3(grid)
    n = int(lattice[0]) * int(lattice[1]) * int(lattice[2])
    o_sdf = torch.empty(n, device=grid.device) if sdf else None
    o_n = torch.empty(n, 3, device=grid.device) if normal else None
    call("vx_field_query_lattice", ptr(grid), i3(res), f3(xyz_min), f3(xyz_max), i3(lattice), f3(lat_min),
         f3(lat_max), ptr(o_sdf), ptr(o_n), stream_ptr(grid.device))
    return o_sdf, o_n


# ------------------------------------------------------------------ sampler ---------------

_TABLES: Dict[Tuple, torch.Tensor] = {}


def linspace_table(a: float, b: float, n: int, device) -> torch.Tensor:
    """torch.linspace values on the device (cached): the tables the sampler kernel reads."""
    key = (float(a), float(b), int(n), str(device))
    t = _TABLES.get(key)
    if t is None:
        t = torch.linspace(a, b, steps=n, device=device, dtype=torch.float32)
        _TABLES[key] = t
    return t


def near_far_from_sphere(rays_o, rays_d, radius=1.0):
    o = check_tensor(rays_o.contiguous(), "rays_o")
    d = check_tensor(rays_d.contiguous(), "rays_d")
    n = o.numel() // 3
    near = torch.empty(*o.shape[:-1], 1, device=o.device)
    far = torch.empty(*o.shape[:-1], 1, device=o.device)
    call("vx_near_far_from_sphere", ptr(o), ptr(d), n, float(radius), ptr(near), ptr(far), stream_ptr(o.device))
    return near, far


def sample_multistep(grid, xyz_min, xyz_max, rays_o, rays_d, near=None, far=None, n_samples=64, n_importance=64,
                     steps=4, perturb=False, t_rand=None, u=None, occupancy=None, occ_min=None, occ_max=None,
                     want_z=True):
    res = _grid3(grid)
    o = check_tensor(rays_o.contiguous(), "rays_o")
    d = check_tensor(rays_d.contiguous(), "rays_d")
    nr = o.shape[0]
    dev = o.device
    per = max(n_importance // steps, 1) if (n_importance > 0 and steps > 0) else 0
    total = n_samples + per * steps
    t_lin = linspace_table(0.0, 1.0, n_samples, dev)
    u_det = linspace_table(0.5 / per, 1.0 - 0.5 / per, per, dev) if per > 0 else None
    if near is not None:
        near = check_tensor(near.contiguous(), "near")
        far = check_tensor(far.contiguous(), "far")
    if perturb:
        t_rand = check_tensor(t_rand.contiguous(), "t_rand")
        if per > 0:
            u = check_tensor(u.contiguous(), "u")
    occ_ptr, occ_res = None, 0
    if occupancy is not None:
        occ = check_tensor(occupancy.contiguous(), "occupancy", dtype=torch.bool)
        occ_ptr, occ_res = ptr(occ), occ.shape[0]
    z = torch.empty(nr, total, device=dev) if want_z else None
    dists = torch.empty(nr, total, device=dev)
    mid = torch.empty(nr, total, device=dev)
    call("vx_sample_multistep", ptr(grid), i3(res), f3(xyz_min), f3(xyz_max), ptr(o), ptr(d), ptr(near), ptr(far), nr,
         n_samples, n_importance, steps, int(bool(perturb)), ptr(t_lin), ptr(t_rand if perturb else None),
         ptr(u if perturb else None), ptr(u_det), occ_ptr, occ_res, f3(occ_min if occ_min is not None else xyz_min),
         f3(occ_max if occ_max is not None else xyz_max), ptr(z), ptr(dists), ptr(mid), stream_ptr(dev))
    return z, dists, mid


def up_sample(rays_o, rays_d, z, sdf, n_importance, inv_s, det=True, u=None, occupancy=None, occ_min=None,
              occ_max=None):
    o = check_tensor(rays_o.contiguous(), "rays_o")
    d = check_tensor(rays_d.contiguous(), "rays_d")
    z = check_tensor(z.contiguous(), "z_vals")
    nr, n = z.shape
    sdf = check_tensor(sdf.reshape(nr, n).contiguous(), "sdf")
    dev = z.device
    u_det = linspace_table(0.5 / n_importance, 1.0 - 0.5 / n_importance, n_importance, dev) if det else None
    if not det:
        u = check_tensor(u.contiguous(), "u") if u is not None else torch.rand(nr, n_importance, device=dev)
    occ_ptr, occ_res = None, 0
    if occupancy is not None:
        occ = check_tensor(occupancy.contiguous(), "occupancy", dtype=torch.bool)
        occ_ptr, occ_res = ptr(occ), occ.shape[0]
    out = torch.empty(nr, n_importance, device=dev)
    lo = occ_min if occ_min is not None else (-1.0, -1.0, -1.0)
    hi = occ_max if occ_max is not None else (1.0, 1.0, 1.0)
    call("vx_up_sample", ptr(o), ptr(d), ptr(z), ptr(sdf), nr, n, n_importance, float(inv_s),
         ptr(None if det else u), ptr(u_det), occ_ptr, occ_res, f3(lo), f3(hi), ptr(out), stream_ptr(dev))
    return out


def sample_pdf(bins, weights, n_samples, det=False, u=None, cdf=None, return_indices=False):
    bins = check_tensor(bins.contiguous(), "bins")
    nr, nb = bins.shape
    dev = bins.device
    if cdf is None:
        weights = check_tensor(weights.contiguous(), "weights")
    else:
        cdf = check_tensor(cdf.contiguous(), "cdf")
    u_det = None
    if det:
        u_det = linspace_table(0.5 / n_samples, 1.0 - 0.5 / n_samples, n_samples, dev)
        u = None
    else:
        u = check_tensor(u.contiguous(), "u") if u is not None else torch.rand(nr, n_samples, device=dev)
    out = torch.empty(nr, n_samples, device=dev)
    idx = torch.empty(nr, n_samples, dtype=torch.int64, device=dev) if return_indices else None
    call("vx_sample_pdf", ptr(bins), ptr(weights if cdf is None else None), ptr(cdf), nr, nb, n_samples, ptr(u),
         ptr(u_det), ptr(out), ptr(idx), stream_ptr(dev))
    return (out, idx) if return_indices else out


def cat_z_vals(z_old, z_new, sdf_old=None, sdf_new=None):
    """Per ray: z_old (R, n) and z_new (R, m) concatenated and sorted as torch.sort orders them; the
    SDF values (when given) carried with their depths. Returns (z, sdf or None)."""
    zo = check_tensor(z_old.contiguous(), "z_vals")
    zn = check_tensor(z_new.contiguous(), "new_z_vals", device=zo.device)
    nr, n = zo.shape
    m = zn.shape[1]
    if zn.shape[0] != nr:
        raise RuntimeError(f"new_z_vals has {zn.shape[0]} rays, z_vals {nr}")
    carry = sdf_old is not None
    so = check_tensor(sdf_old.reshape(nr, n).contiguous(), "sdf", device=zo.device) if carry else None
    sn = check_tensor(sdf_new.reshape(nr, m).contiguous(), "new_sdf", device=zo.device) if carry else None
    z = torch.empty(nr, n + m, device=zo.device)
    sdf = torch.empty(nr, n + m, device=zo.device) if carry else None
    call("vx_cat_z_vals", ptr(zo), ptr(zn), ptr(so), ptr(sn), nr, n, m, ptr(z), ptr(sdf), stream_ptr(zo.device))
    return z, sdf


# ------------------------------------------------------------------ render geometry -------


class NormalGradHandoff:
    """dL/dnormal of the appearance branch, handed from AppearanceMLPFn's adjoint to
    RenderGeometryFn's, which adds it to the compositing branch's inside the geometry adjoint kernel
    (the same single addition autograd would make, without its (P, 3) sum kernel). The geometry
    adjoint runs after both consumers of the normals, so the hand-off is complete by then."""

    def __init__(self, training: bool = True):
        self.d_normal = None
        self.training = training  # the caller's grad mode (Function.forward itself runs without grad)


class RenderGeometryFn(torch.autograd.Function):
    """Pass-2 geometry (positions, SDF, Eq.7 normal) of (rays, midpoints); marks V_R corners."""

    @staticmethod
    def forward(ctx, grid, rays_o, rays_d, mid, xyz_min, xyz_max, bitmap, want_grad, handoff=None):
        g = grid.detach()
        res = _grid3(g)
        nr, ns = mid.shape
        dev = mid.device
        sdf = torch.empty(nr, ns, device=dev)
        nrm = torch.empty(nr, ns, 3, device=dev)
        gr = torch.empty(nr, ns, 3, device=dev) if want_grad else None
        # kept for the adjoint (its normalisation term) when the caller does not receive it; only in
        # training (needs_input_grad stays True under no_grad)
        keep = gr is None and ctx.needs_input_grad[0] and handoff is not None and handoff.training
        gkeep = torch.empty(nr, ns, 3, device=dev) if keep else None
        call("vx_render_geometry_forward", ptr(g), i3(res), f3(xyz_min), f3(xyz_max), ptr(rays_o), ptr(rays_d),
             ptr(mid), nr, ns, ptr(sdf), ptr(nrm), ptr(gr if gr is not None else gkeep), ptr(bitmap), stream_ptr(dev))
        ctx.gkeep = gkeep
        ctx.save_for_backward(grid, rays_o, rays_d, mid)
        ctx.bounds = (xyz_min, xyz_max)
        ctx.handoff = handoff
        if gr is not None:
            ctx.mark_non_differentiable(gr)
        return sdf, nrm, gr

    @staticmethod
    def backward(ctx, d_sdf, d_nrm, _d_gr):
        grid, rays_o, rays_d, mid = ctx.saved_tensors
        d_nrm2 = None
        if ctx.handoff is not None:
            d_nrm2, ctx.handoff.d_normal = ctx.handoff.d_normal, None
        if not ctx.needs_input_grad[0]:
            return (None,) * 9
        g = grid.detach()
        res = _grid3(g)
        nr, ns = mid.shape
        gg = torch.zeros(res, device=mid.device)
        d_sdf = None if d_sdf is None else d_sdf.contiguous()
        d_nrm = None if d_nrm is None else d_nrm.contiguous()
        gkeep, ctx.gkeep = ctx.gkeep, None
        geometry_backward(g, res, ctx.bounds, rays_o, rays_d, mid, d_sdf, d_nrm, gg, d_nrm2, gkeep)
        return gg.reshape(grid.shape), None, None, None, None, None, None, None, None


# ------------------------------------------------------------------ deterministic mode ------

_deterministic = False


def set_deterministic(flag: bool) -> None:
    """Route the geometry and hash-table adjoints through the sorted segmented reduction
    (bitwise reproducible) instead of float atomics."""
    global _deterministic
    _deterministic = bool(flag)


def is_deterministic() -> bool:
    return _deterministic


def _workspace(dev, nbytes: int) -> torch.Tensor:
    sc = Scratch.get(dev)
    ws = getattr(sc, "det_ws", None)
    if ws is None or ws.numel() < nbytes:
        sc.det_ws = ws = torch.empty(int(nbytes), dtype=torch.uint8, device=dev)
    return ws


def geometry_backward(g, res, bounds, rays_o, rays_d, mid, d_sdf, d_normal, out, d_normal2=None, grad_fwd=None):
    """d_normal2: a second dL/dnormal source, (P, 3) contiguous, added to d_normal in the kernel.
    grad_fwd: the forward's Eq.7 gradients (P, 3), read instead of recomputed (atomic path)."""
    nr, ns = mid.shape
    dev = mid.device
    if d_normal2 is not None:
        check_tensor(d_normal2, "d_normal2", device=dev)
        if d_normal2.numel() != nr * ns * 3:
            raise RuntimeError(f"d_normal2 has {d_normal2.numel()} elements, need {nr * ns * 3}")
    if _deterministic:
        need = int(L.query("vx_geometry_backward_det_workspace", nr, ns, i3(res)))
        if need == 0:
            raise RuntimeError("batch too large for one deterministic geometry pass")
        ws = _workspace(dev, need)
        call("vx_render_geometry_backward_det", ptr(g), i3(res), f3(bounds[0]), f3(bounds[1]), ptr(rays_o),
             ptr(rays_d), ptr(mid), nr, ns, ptr(d_sdf), ptr(d_normal), ptr(d_normal2), 3, ptr(out), ptr(ws),
             ws.numel(), stream_ptr(dev))
    else:
        call("vx_render_geometry_backward", ptr(g), i3(res), f3(bounds[0]), f3(bounds[1]), ptr(rays_o), ptr(rays_d),
             ptr(mid), nr, ns, ptr(d_sdf), ptr(d_normal), ptr(d_normal2), 3, None, ptr(grad_fwd), ptr(out),
             stream_ptr(dev))


def hash_backward(d_emb, cfg, active_levels, pts, rays_o, rays_d, mid, n_samples, xyz_min, xyz_max, n_points,
                  d_out, ld):
    dev = d_out.device
    lw = cfg.level_weights(active_levels)
    if _deterministic:
        need = int(L.query("vx_hash_backward_det_workspace", n_points, cfg.n_levels, cfg.log2_size))
        if need == 0:
            raise RuntimeError("batch too large for one deterministic hash pass")
        ws = _workspace(dev, need)
        res_d, lw_d = cfg.device_tables(dev, lw)
        call("vx_hash_encode_backward_det", ptr(d_emb), cfg.n_levels, cfg.log2_size, cfg.n_features, ptr(res_d),
             ptr(lw_d), ptr(pts), ptr(rays_o), ptr(rays_d), ptr(mid), n_samples,
             f3(xyz_min) if xyz_min is not None else None, f3(xyz_max) if xyz_max is not None else None, n_points,
             ptr(d_out), ld, ptr(ws), ws.numel(), stream_ptr(dev))
    else:
        call("vx_hash_encode_backward", ptr(d_emb), cfg.n_levels, cfg.log2_size, cfg.n_features, cfg._res_c, lw,
             ptr(pts), ptr(rays_o), ptr(rays_d), ptr(mid), n_samples,
             f3(xyz_min) if xyz_min is not None else None, f3(xyz_max) if xyz_max is not None else None, n_points,
             ptr(d_out), ld, stream_ptr(dev))


class HashConfig:
    """Static hash-grid description (models/radiance_hash.py:25-60)."""

    def __init__(self, n_levels=16, n_features=2, log2_size=19, base=16, finest=2048):
        self.n_levels = n_levels
        self.n_features = n_features
        self.log2_size = log2_size
        b = math.exp((math.log(finest) - math.log(base)) / max(n_levels - 1, 1))
        self.resolutions = [math.floor(base * (b ** lvl)) for lvl in range(n_levels)]
        self._res_c = L.iarr(self.resolutions)
        self._dev_tables: Dict[tuple, tuple] = {}

    def device_tables(self, dev, level_weights):
        """(resolutions int32, level weights float32) on `dev`, cached per weights. Uploaded from
        pinned host copies (kept alive here), so a first use inside CUDA graph capture is legal."""
        idx = torch.device(dev).index
        lw = tuple(float(w) for w in list(level_weights)[:self.n_levels])
        key = (idx, lw)
        t = self._dev_tables.get(key)
        if t is None:
            hr = torch.tensor(self.resolutions, dtype=torch.int32).pin_memory()
            hw = torch.tensor(lw, dtype=torch.float32).pin_memory()
            t = (hr.to(dev, non_blocking=True), hw.to(dev, non_blocking=True), hr, hw)
            self._dev_tables[key] = t
        return t[0], t[1]

    def level_weights(self, active_levels: Optional[float]):
        w = []
        for lvl in range(self.n_levels):
            if active_levels is None:
                w.append(1.0)
                continue
            li = lvl + 1.0
            if li <= active_levels:
                w.append(1.0)
            elif li - 1.0 < active_levels < li:
                w.append(active_levels - (li - 1.0))
            else:
                w.append(0.0)
        return L.farr(w)


MLP_LD = 52  # row stride of the radiance-MLP input buffer: [hash 32 | SH 16 | normal 3 | pad]
# Row stride of the fused appearance path's compact rows, [hash 32 | normal 3 | pad]: the 16 SH(d)
# columns depend on the ray only and the MLP kernels recompute them from the ray direction.
MLP_LD_COMPACT = 36
# Inference rows scratch: up to 4M compact rows (576 MiB) per call, whole rays at a time. The split
# gather + MLP kernels beat the fused in-shared-memory kernel by ~25% per sample, and chunks this
# large keep the per-chunk launch and tail cost small (a 65,536-ray render: 256K-row chunks
# 3.2 ms, 1M 2.66 ms, 4M 2.49 ms of appearance time).
INFER_CHUNK_ROWS = 1 << 22


def mlp_forward(rows: torch.Tensor, W0, b0, W1, b1) -> torch.Tensor:
    """Fused radiance MLP on input rows (P, >=51) with any row stride: colours (P, 3)."""
    p = rows.shape[0]
    if rows.stride(1) != 1:
        raise RuntimeError("MLP rows must have unit column stride")
    out = torch.empty(p, 3, device=rows.device)
    call("vx_radiance_mlp_forward", ptr(rows), rows.stride(0), p, rows.shape[1], W0.shape[0], W1.shape[0],
         ptr(W0.detach()), ptr(b0.detach()), ptr(W1.detach()), ptr(b1.detach()), ptr(out), stream_ptr(rows.device))
    return out


def mlp_backward(rows, W0, b0, W1, b1, d_colors, colors=None, rays_d=None, n_samples=0):
    """colors: the forward's (P, 3) outputs (the adjoint then skips recomputing the output layer),
    or None. rays_d given: rows are the compact rows of AppearanceMLPFn (P, 36) whose SH(d) the
    kernel recomputes from rays_d of row i's ray (i // n_samples)."""
    dev = rows.device
    p = rows.shape[0]
    if colors is not None:
        check_tensor(colors, "colors", device=dev)
        if colors.numel() != 3 * p:
            raise RuntimeError(f"colors has {colors.numel()} elements, need {3 * p}")
    nb = int(L.query("vx_mlp_blocks", p))
    nf = int(L.query("vx_mlp_partial_floats"))
    sc = Scratch.get(dev)
    if not hasattr(sc, "mlp_partials") or sc.mlp_partials.numel() < nb * nf:
        sc.mlp_partials = torch.empty(nb * nf, device=dev)
    d_hash = torch.empty(p, 32, device=dev)
    d_normal = torch.empty(p, 3, device=dev)
    dW0, db0, dW1, db1 = (torch.empty_like(t) for t in (W0, b0, W1, b1))
    weights = (ptr(W0.detach()), ptr(b0.detach()), ptr(W1.detach()), ptr(b1.detach()))
    outs = (ptr(check_tensor(d_colors.contiguous(), "d_colors")), ptr(colors), ptr(d_hash), ptr(d_normal), ptr(dW0),
            ptr(db0), ptr(dW1), ptr(db1), ptr(sc.mlp_partials), sc.mlp_partials.numel(), stream_ptr(dev))
    if rays_d is None:
        call("vx_radiance_mlp_backward", ptr(rows), rows.stride(0), p, rows.shape[1], W0.shape[0], W1.shape[0],
             *weights, *outs)
    else:
        if rows.shape[1] != MLP_LD_COMPACT or not rows.is_contiguous():
            raise RuntimeError(f"compact MLP rows must be contiguous ({MLP_LD_COMPACT} floats a row)")
        call("vx_appearance_mlp_backward", ptr(rows), ptr(check_tensor(rays_d, "rays_d")), n_samples, p, *weights,
             *outs)
    return d_hash, d_normal, dW0, db0, dW1, db1


class RadianceMLPFn(torch.autograd.Function):
    """The 51-64-3 radiance MLP on pre-assembled rows, fused forward and adjoint."""

    @staticmethod
    def forward(ctx, rows, W0, b0, W1, b1):
        ctx.save_for_backward(rows, W0, b0, W1, b1)
        return mlp_forward(rows.detach(), W0, b0, W1, b1)

    @staticmethod
    def backward(ctx, g):
        rows, W0, b0, W1, b1 = ctx.saved_tensors
        d_hash, d_normal, dW0, db0, dW1, db1 = mlp_backward(rows.detach(), W0, b0, W1, b1, g)
        d_rows = None
        if ctx.needs_input_grad[0]:
            d_rows = torch.zeros(rows.shape, device=rows.device)
            d_rows[:, :32] = d_hash
            d_rows[:, 48:51] = d_normal
        return d_rows, dW0, db0, dW1, db1


class AppearanceMLPFn(torch.autograd.Function):
    """Hash encoding + SH + normal rows -> fused MLP -> colours for (rays, midpoints).

    models/voxneus.py:147-157 without materialising the hidden layer: the compact rows
    [hash 32 | normal 3 | pad] are kept for the adjoint, which recomputes SH(d) from the ray
    direction and the hidden layer, and scatters into the hash table.
    """

    @staticmethod
    def forward(ctx, embeddings, normals, W0, b0, W1, b1, rays_o, rays_d, mid, xyz_min, xyz_max, cfg, active_levels,
                keep_rows=True, handoff=None):
        nr, ns = mid.shape
        p = nr * ns
        width = 2 * cfg.n_levels + 16 + 3
        if width != 51:
            raise RuntimeError("the fused appearance path needs 16 hash levels x 2 features")
        ld = MLP_LD_COMPACT
        # keep_rows: the caller's grad mode (forward itself always runs with grad disabled, and
        # needs_input_grad stays True under no_grad), so inference does not write the rows
        need_rows = bool(keep_rows) and any(ctx.needs_input_grad[:6])
        rows = torch.empty(p, ld, device=mid.device) if need_rows else None
        nrm = normals.detach().contiguous()
        colors = torch.empty(p, 3, device=mid.device)
        args = (ptr(embeddings.detach()), cfg.n_levels, cfg.log2_size, cfg.n_features, cfg._res_c,
                cfg.level_weights(active_levels), ptr(rays_o), ptr(rays_d), ptr(mid), ns, f3(xyz_min), f3(xyz_max), p,
                ptr(nrm), ptr(W0.detach()), ptr(b0.detach()), ptr(W1.detach()), ptr(b1.detach()), ptr(colors))
        if rows is not None:
            call("vx_appearance_mlp_forward", *args, ptr(rows), ld, stream_ptr(mid.device))
        else:  # inference: rows pass through an L2-sized scratch, whole rays at a time
            n_rows = max(ns, min(p, (INFER_CHUNK_ROWS // ns) * ns))
            scratch = torch.empty(n_rows, MLP_LD_COMPACT, device=mid.device)
            call("vx_appearance_mlp_forward_chunked", *args, ptr(scratch), n_rows, stream_ptr(mid.device))
        ctx.save_for_backward(rays_o, rays_d, mid, W0, b0, W1, b1)
        ctx.rows = rows
        ctx.colors = colors if rows is not None else None  # the adjoint's sigmoid derivative reads them
        ctx.handoff = handoff
        ctx.meta = (xyz_min, xyz_max, cfg, active_levels, embeddings.shape, normals.shape)
        return colors.reshape(nr, ns, 3)

    @staticmethod
    def backward(ctx, g):
        rays_o, rays_d, mid, W0, b0, W1, b1 = ctx.saved_tensors
        xyz_min, xyz_max, cfg, active_levels, eshape, nshape = ctx.meta
        nr, ns = mid.shape
        rows, colors = ctx.rows, ctx.colors
        ctx.rows = ctx.colors = None
        if rows is None:
            raise RuntimeError("AppearanceMLPFn: forward ran with keep_rows=False; no adjoint input kept")
        d_hash, d_normal, dW0, db0, dW1, db1 = mlp_backward(rows, W0, b0, W1, b1, g.reshape(-1, 3), colors, rays_d,
                                                            ns)
        d_emb = None
        if ctx.needs_input_grad[0]:
            d_emb = torch.zeros(eshape, device=g.device)
            hash_backward(d_emb, cfg, active_levels, None, rays_o, rays_d, mid, ns, xyz_min, xyz_max, nr * ns, d_hash,
                          32)
        d_nrm = d_normal.reshape(nshape)
        if ctx.handoff is not None and ctx.needs_input_grad[1]:
            ctx.handoff.d_normal, d_nrm = d_normal, None  # summed inside the geometry adjoint
        return (d_emb, d_nrm, dW0, db0, dW1, db1, None, None, None, None, None, None, None, None, None)


class HashEncodeFn(torch.autograd.Function):
    """Hash encoding of normalised points (RadianceHashGrid.forward, radiance_hash.py:211-231)."""

    @staticmethod
    def forward(ctx, embeddings, norm_xyz, cfg, active_levels):
        x = check_tensor(norm_xyz.detach().reshape(-1, 3).contiguous(), "norm_xyz")
        p = x.shape[0]
        out = torch.empty(p, 2 * cfg.n_levels, device=x.device)
        call("vx_appearance_forward", ptr(embeddings.detach()), cfg.n_levels, cfg.log2_size, cfg.n_features,
             cfg._res_c, cfg.level_weights(active_levels), ptr(x), None, None, None, 1, None, None, p, ptr(out),
             2 * cfg.n_levels, -1, None, 0, -1, None, -1, stream_ptr(x.device))
        ctx.save_for_backward(x)
        ctx.meta = (cfg, active_levels, embeddings.shape)
        return out.reshape(*norm_xyz.shape[:-1], 2 * cfg.n_levels)

    @staticmethod
    def backward(ctx, g):
        (x,) = ctx.saved_tensors
        cfg, active_levels, eshape = ctx.meta
        d_emb = None
        if ctx.needs_input_grad[0]:
            gc = g.reshape(-1, 2 * cfg.n_levels).contiguous()
            d_emb = torch.zeros(eshape, device=g.device)
            hash_backward(d_emb, cfg, active_levels, x, None, None, None, 1, None, None, x.shape[0], gc, gc.shape[1])
        return d_emb, None, None, None


def sh4(dirs: torch.Tensor) -> torch.Tensor:
    """Degree-4 SH of unit directions (models/embedder.py:55-87)."""
    d = check_tensor(dirs.detach().reshape(-1, 3).contiguous(), "dirs")
    out = torch.empty(d.shape[0], 16, device=d.device)
    call("vx_appearance_forward", None, 0, 0, 2, None, None, None, None, None, None, 1, None, None, d.shape[0],
         ptr(out), 16, 0, ptr(d), 3, -1, None, -1, stream_ptr(d.device))
    return out.reshape(*dirs.shape[:-1], 16)


# ------------------------------------------------------------------ compositing -----------


def _dir_strides(dirs: torch.Tensor, n_rays: int, n_samples: int):
    if dirs.dim() == 2:
        if dirs.stride(1) != 1:
            raise RuntimeError("ray_dirs must have unit stride in the last dimension")
        return dirs, dirs.stride(0), 0
    if dirs.dim() == 3:
        if dirs.stride(2) != 1:
            raise RuntimeError("ray_dirs must have unit stride in the last dimension")
        return dirs, dirs.stride(0), dirs.stride(1)
    raise RuntimeError("ray_dirs must be (N,3) or (N,S,3)")


def huber_loss(pred, target, delta, with_grad=True):
    """(loss, dloss/dpred or None): the NeuS2 Huber colour loss and its gradient from one kernel."""
    p = check_tensor(pred.detach().contiguous(), "pred")
    t = check_tensor(target.detach().contiguous(), "target")
    if p.shape != t.shape:
        raise RuntimeError(f"pred {tuple(p.shape)} and target {tuple(t.shape)} differ")
    n = p.numel()
    nb = int(L.query("vx_huber_loss_blocks", n))
    part = Scratch.get(p.device).partials_for(nb)
    loss = torch.empty((), device=p.device)
    grad = torch.empty_like(p) if with_grad else None
    call("vx_huber_loss", ptr(p), ptr(t), n, float(delta), ptr(loss), ptr(grad), ptr(part), part.numel(),
         stream_ptr(p.device))
    return loss, grad


class HuberLossFn(torch.autograd.Function):
    """NeuS2 Huber colour loss (rendering/volume_render.py:43-54): mean elementwise Huber of
    pred - target; the gradient is written by the same kernel and scaled in the backward."""

    @staticmethod
    def forward(ctx, pred, target, delta):
        loss, grad = huber_loss(pred, target, delta, ctx.needs_input_grad[0])
        ctx.grad = grad
        ctx.shape = pred.shape
        return loss

    @staticmethod
    def backward(ctx, g):
        grad, ctx.grad = ctx.grad, None
        return (grad * g).reshape(ctx.shape), None, None


class CompositeFn(torch.autograd.Function):
    """Fused Eq.2 alpha + inside-sphere mask + transmittance + compositing, hand-written adjoint.

    rendering/volume_render.py:57-153 with neus_alpha.py:12-81 and volume_render.py:12-40.
    `s_param` is s (s_is_variance False) or the variance parameter v (True).
    """

    @staticmethod
    def forward(ctx, colors, sdf, normals, s_param, dirs, z, dists, pts, rays_o, s_is_variance, s_max, radius,
                background, iter_cos, cos_anneal, amplify_k, amp_flag, per_sample=True):
        nr, ns = z.shape
        dev = z.device
        colors_c = check_tensor(colors.detach().reshape(nr, ns, 3).contiguous(), "colors")
        sdf_c = check_tensor(sdf.detach().reshape(nr, ns).contiguous(), "sdf")
        nrm_c = check_tensor(normals.detach().reshape(nr, ns, 3).contiguous(), "normals")
        d, drs, dss = _dir_strides(dirs.detach(), nr, ns)
        s_c = check_tensor(s_param.detach().reshape(1).contiguous(), "s")
        bg = None
        bg_per_ray = 0
        if background is not None:
            if not isinstance(background, torch.Tensor):
                background = torch.full((3,), float(background), device=dev)
            bg = check_tensor(background.detach().contiguous(), "background")
            bg_per_ray = 1 if bg.dim() == 2 else 0
        ptsc = None if pts is None else check_tensor(pts.detach().reshape(nr, ns, 3).contiguous(), "pts")
        # per_sample=False: the (N, S) weights, alpha and transmittance are neither written nor returned
        outs = [torch.empty(nr, 3, device=dev), torch.empty(nr, 1, device=dev), torch.empty(nr, 3, device=dev),
                torch.empty(nr, 1, device=dev)]
        outs += [torch.empty(nr, ns, device=dev) if per_sample else None for _ in range(3)]
        call("vx_composite_forward", ptr(colors_c), ptr(sdf_c), ptr(nrm_c), ptr(d), drs, dss, ptr(z), ptr(dists),
             ptr(ptsc), ptr(rays_o), ptr(s_c), int(s_is_variance), float(s_max), float(radius), ptr(bg), bg_per_ray,
             int(iter_cos), float(cos_anneal), nr, ns, *[ptr(t) for t in outs], stream_ptr(dev))
        ctx.save_for_backward(colors_c, sdf_c, nrm_c, s_c, d, z, dists, ptsc, rays_o, bg)
        # outputs the loss does not use (depth, weights, alpha, ...) reach the adjoint as None, which
        # the kernel reads as zero: no zero-filled (N, S) gradient tensors
        ctx.set_materialize_grads(False)
        ctx.meta = (drs, dss, int(s_is_variance), float(s_max), float(radius), bg_per_ray, int(iter_cos),
                    float(cos_anneal), float(amplify_k), amp_flag, sdf.shape, normals.shape, colors.shape,
                    s_param.shape)
        return tuple(outs)

    @staticmethod
    def backward(ctx, g_rgb, g_depth, g_normal, g_op, g_w, g_a, g_t):
        colors, sdf, nrm, s_c, d, z, dists, pts, rays_o, bg = ctx.saved_tensors
        (drs, dss, s_is_var, s_max, radius, bg_per_ray, iter_cos, cos_anneal, amp_k, amp_flag, sdf_shape, n_shape,
         c_shape, s_shape) = ctx.meta
        nr, ns = z.shape
        dev = z.device
        sc = Scratch.get(dev)
        nblk = L.query("vx_composite_workspace_blocks", nr)
        partials = sc.partials_for(nblk)
        d_colors = torch.empty(nr, ns, 3, device=dev)
        d_sdf = torch.empty(nr, ns, device=dev)
        d_n = torch.empty(nr, ns, 3, device=dev)
        d_s = torch.empty(1, device=dev)

        def c(t):
            return None if t is None else t.contiguous()

        call("vx_composite_backward", ptr(colors), ptr(sdf), ptr(nrm), ptr(d), drs, dss, ptr(z), ptr(dists), ptr(pts),
             ptr(rays_o), ptr(s_c), s_is_var, s_max, radius, ptr(bg), bg_per_ray, iter_cos, cos_anneal, nr, ns,
             ptr(c(g_rgb)), ptr(c(g_depth)), ptr(c(g_normal)), ptr(c(g_op)), ptr(c(g_w)), ptr(c(g_a)), ptr(c(g_t)),
             ptr(d_colors), ptr(d_sdf), ptr(d_n), ptr(partials), int(partials.numel()),
             ptr(sc.counter(COUNTER_COMPOSITE)), ptr(d_s), amp_k, ptr(amp_flag), stream_ptr(dev))
        return (d_colors.reshape(c_shape), d_sdf.reshape(sdf_shape), d_n.reshape(n_shape), d_s.reshape(s_shape),
                None, None, None, None, None, None, None, None, None, None, None, None, None, None)


class NeusAlphaFn(torch.autograd.Function):
    """compute_neus_alpha (rendering/neus_alpha.py:12-81) for (N,S) samples."""

    @staticmethod
    def forward(ctx, sdf, normals, dirs, dists, s, iter_cos, cos_anneal):
        nr, ns = dists.shape
        sdf_c = check_tensor(sdf.detach().reshape(nr, ns).contiguous(), "sdf")
        n_c = check_tensor(normals.detach().reshape(nr, ns, 3).contiguous(), "normals")
        d, drs, dss = _dir_strides(dirs.detach(), nr, ns)
        dist_c = check_tensor(dists.detach().contiguous(), "dists")
        s_c = check_tensor(s.detach().reshape(1).contiguous(), "s")
        alpha = torch.empty(nr, ns, device=dists.device)
        call("vx_neus_alpha", ptr(sdf_c), ptr(n_c), ptr(d), drs, dss, ptr(dist_c), ptr(s_c), int(iter_cos),
             float(cos_anneal), nr, ns, ptr(alpha), None, None, None, None, stream_ptr(dists.device))
        ctx.save_for_backward(sdf_c, n_c, d, dist_c, s_c)
        ctx.meta = (drs, dss, int(iter_cos), float(cos_anneal), sdf.shape, normals.shape, s.shape)
        return alpha

    @staticmethod
    def backward(ctx, g):
        sdf, n, d, dists, s = ctx.saved_tensors
        drs, dss, iter_cos, cos_anneal, sdf_shape, n_shape, s_shape = ctx.meta
        nr, ns = dists.shape
        dev = dists.device
        d_sdf = torch.empty(nr, ns, device=dev)
        d_n = torch.empty(nr, ns, 3, device=dev)
        d_se = torch.empty(nr, ns, device=dev)
        call("vx_neus_alpha", ptr(sdf), ptr(n), ptr(d), drs, dss, ptr(dists), ptr(s), iter_cos, cos_anneal, nr, ns,
             None, ptr(g.contiguous()), ptr(d_sdf), ptr(d_n), ptr(d_se), stream_ptr(dev))
        d_s = d_se.sum().reshape(s_shape) if ctx.needs_input_grad[4] else None
        return d_sdf.reshape(sdf_shape), d_n.reshape(n_shape), None, None, d_s, None, None


class CompositeWeightsFn(torch.autograd.Function):
    """composite_weights (rendering/volume_render.py:12-40)."""

    @staticmethod
    def forward(ctx, alpha):
        a = check_tensor(alpha.detach().contiguous(), "alpha")
        nr, ns = a.shape
        w = torch.empty_like(a)
        t = torch.empty_like(a)
        call("vx_composite_weights", ptr(a), nr, ns, ptr(w), ptr(t), None, None, None, stream_ptr(a.device))
        ctx.save_for_backward(a)
        return w, t

    @staticmethod
    def backward(ctx, gw, gt):
        (a,) = ctx.saved_tensors
        nr, ns = a.shape
        da = torch.empty_like(a)
        call("vx_composite_weights", ptr(a), nr, ns, None, None, ptr(None if gw is None else gw.contiguous()),
             ptr(None if gt is None else gt.contiguous()), ptr(da), stream_ptr(a.device))
        return da


# ------------------------------------------------------------------ V_R + regularizers -----


def bitmap_words(res) -> int:
    return int(L.query("vx_vr_bitmap_words", i3(res)))


def new_bitmap(res, device) -> torch.Tensor:
    return torch.zeros(bitmap_words(res), dtype=torch.int32, device=device)


def vr_mark_corners(corners: torch.Tensor, res, bitmap: torch.Tensor):
    c = check_tensor(corners.reshape(-1, 3).contiguous(), "corner_indices", dtype=torch.int64)
    call("vx_vr_mark_corners", ptr(c), c.shape[0], i3(res), ptr(bitmap), stream_ptr(c.device))
    return bitmap


def vr_count(bitmap, grid, res, xyz_min, xyz_max, relax_radius=0.0, band=0.0, counts=None, filtered=None):
    """Counts [all, relax, band, relax&band]; `filtered` (2 x words int32) receives the regularizer's
    input bitmaps (bits & band, bits & band & relax)."""
    if counts is None:
        counts = torch.zeros(4, dtype=torch.int64, device=bitmap.device)
    call("vx_vr_count", ptr(bitmap), ptr(grid), i3(res), f3(xyz_min), f3(xyz_max), float(relax_radius), float(band),
         ptr(counts), ptr(filtered), stream_ptr(bitmap.device))
    return counts


def new_filtered(res, device) -> torch.Tensor:
    return torch.zeros(2 * bitmap_words(res), dtype=torch.int32, device=device)


def final_count(counts: torch.Tensor, relax_radius: float, band: float) -> torch.Tensor:
    """|V_R| after the filters, as a device scalar (no host sync)."""
    relax_on = (counts[1] > 0) if relax_radius > 0 else torch.zeros((), dtype=torch.bool, device=counts.device)
    if band > 0:
        return torch.where(relax_on, counts[3], counts[2])
    return torch.where(relax_on, counts[1], counts[0])


def vr_compact(bitmap, grid, res, xyz_min, xyz_max, relax_radius, band, counts, capacity):
    dev = bitmap.device
    sc = Scratch.get(dev)
    nb = int(L.query("vx_vr_compact_blocks", i3(res)))
    blocks = sc.blocks_for(nb)
    verts = torch.empty(capacity, 3, dtype=torch.int64, device=dev)
    lin = torch.empty(capacity, dtype=torch.int64, device=dev)
    call("vx_vr_compact", ptr(bitmap), ptr(grid), i3(res), f3(xyz_min), f3(xyz_max), float(relax_radius), float(band),
         ptr(counts), ptr(blocks), blocks.numel(), ptr(verts), ptr(lin), capacity, stream_ptr(dev))
    return verts, lin


def occupancy_points(res: int, xyz_min, xyz_max, idx: Sequence[torch.Tensor]) -> torch.Tensor:
    """World-space centres (n,3) of the drawn cells of a res^3 occupancy grid."""
    ix, iy, iz = (check_tensor(t, "idx", dtype=torch.int64) for t in idx)
    n = ix.numel()
    if iy.numel() != n or iz.numel() != n:
        raise RuntimeError("idx_x, idx_y and idx_z must have the same length")
    pts = torch.empty(n, 3, dtype=torch.float32, device=ix.device)
    call("vx_occupancy_points", int(res), f3(xyz_min), f3(xyz_max), ptr(ix), ptr(iy), ptr(iz), n, ptr(pts),
         stream_ptr(ix.device))
    return pts


def occupancy_query(mask: torch.Tensor, xyz_min, xyz_max, pts: torch.Tensor) -> torch.Tensor:
    """OccupancyGrid.is_occupied: (..., 3) world points -> (...) bool."""
    check_tensor(mask, "occupancy_mask", dtype=torch.bool)
    lead = pts.shape[:-1]
    p = check_tensor(pts.reshape(-1, 3).float().contiguous(), "pts")
    out = torch.empty(p.shape[0], dtype=torch.bool, device=p.device)
    call("vx_occupancy_query", ptr(mask), int(mask.shape[0]), f3(xyz_min), f3(xyz_max), ptr(p), p.shape[0], ptr(out),
         stream_ptr(p.device))
    return out.reshape(lead)


def occupancy_update(density: torch.Tensor, mask: torch.Tensor, idx: Sequence[torch.Tensor], xyz_min, xyz_max,
                     s: torch.Tensor, s_is_variance: bool, s_max: float, first: bool, decay: float, threshold: float,
                     grid: Optional[torch.Tensor] = None, grid_bounds=None, sdf_values: Optional[torch.Tensor] = None):
    """EMA update of density (R,R,R) float32 and mask (R,R,R) bool at the drawn cells, in place."""
    res = int(density.shape[0])
    check_tensor(density, "density_grid")
    check_tensor(mask, "occupancy_mask", dtype=torch.bool)
    if list(density.shape) != [res] * 3 or list(mask.shape) != [res] * 3:
        raise RuntimeError("density_grid and occupancy_mask must both be (R, R, R)")
    ix, iy, iz = (check_tensor(t, "idx", dtype=torch.int64) for t in idx)
    n = ix.numel()
    if iy.numel() != n or iz.numel() != n:
        raise RuntimeError("idx_x, idx_y and idx_z must have the same length")
    s = check_tensor(s.reshape(1), "s")
    dev = density.device
    if grid is not None:
        gres = _grid3(grid)
        glo, ghi = grid_bounds
        gargs = (ptr(grid), i3(gres), f3(glo), f3(ghi), None)
    else:
        sdf_values = check_tensor(sdf_values.reshape(-1), "sdf_values")
        if sdf_values.numel() != n:
            raise RuntimeError(f"query_sdf_fn returned {sdf_values.numel()} values for {n} points")
        gargs = (None, None, None, None, ptr(sdf_values))
    need = int(L.query("vx_occupancy_workspace", n))
    sc = Scratch.get(dev)
    ws = getattr(sc, "occ_ws", None)
    if ws is None or ws.numel() < need:
        sc.occ_ws = ws = torch.empty(max(need, 16), dtype=torch.uint8, device=dev)
    call("vx_occupancy_update", *gargs, res, f3(xyz_min), f3(xyz_max), ptr(ix), ptr(iy), ptr(iz), n, ptr(s),
         int(bool(s_is_variance)), float(s_max), int(bool(first)), float(decay), float(threshold), ptr(density),
         ptr(mask), ptr(ws), ws.numel(), None, stream_ptr(dev))


def reg_list(kind: str, grid3, verts, eps, weight, grad_out):
    """List-form eikonal / curvature (the reference kernels' interface); returns the loss tensor."""
    res = _grid3(grid3)
    v = check_tensor(verts.contiguous(), "active_vertices", dtype=torch.int64)
    nv = v.shape[0]
    dev = v.device
    losses = torch.zeros(2, device=dev)
    if nv == 0:
        return losses
    sc = Scratch.get(dev)
    nblk = int(L.query("vx_reg_list_blocks", nv))
    partials = sc.partials_for(3 * nblk)
    name, ci = ("vx_eikonal_grad", COUNTER_EIK) if kind == "eikonal" else ("vx_curvature_grad", COUNTER_CURV)
    call(name, ptr(grid3), i3(res), ptr(v), nv, ptr(grad_out), f3(eps), float(weight), ptr(partials),
         int(partials.numel()), ptr(sc.counter(ci)), ptr(losses), stream_ptr(dev))
    return losses


def reg_stencil(grid, filtered, res, xyz_min, xyz_max, relax_radius, band, counts, w_eik, w_curv, grad_out,
                losses=None, n_active=None):
    """Fused eikonal + curvature into grad_out; `filtered` and `counts` come from vr_count.
    n_active: an int64 device scalar receiving |V_R| after the filters (final_count's value)."""
    if n_active is not None:
        check_tensor(n_active, "n_active", dtype=torch.int64, device=grid.device)
    dev = grid.device
    bitmap = filtered
    sc = Scratch.get(dev)
    partials = sc.partials_for(int(L.query("vx_reg_stencil_workspace", i3(res))))
    if losses is None:
        losses = torch.zeros(2, device=dev)
    call("vx_reg_stencil", ptr(grid), ptr(bitmap), i3(res), f3(xyz_min), f3(xyz_max), float(relax_radius),
         float(band), ptr(counts), float(w_eik), float(w_curv), ptr(grad_out), ptr(partials), partials.numel(),
         ptr(sc.counter(COUNTER_STENCIL)), ptr(losses), ptr(n_active), stream_ptr(dev))
    return losses


# ------------------------------------------------------------------ grid upsample / Adam ---


def grid_upsample(grid: torch.Tensor, new_res) -> torch.Tensor:
    src = check_tensor(grid.detach().contiguous(), "grid")
    res_in = list(src.shape[-3:])
    res_out = [new_res] * 3 if isinstance(new_res, int) else [int(r) for r in new_res]
    lead = list(src.shape[:-3])
    dst = torch.empty(*lead, *res_out, device=src.device)
    call("vx_grid_upsample", ptr(src), i3(res_in), ptr(dst), i3(res_out), stream_ptr(src.device))
    return dst


def adam_torch(segments, beta1: float, beta2: float, eps: float, masked: bool = False):
    """torch.optim.Adam's update over [(param, grad, exp_avg, exp_avg_sq, step, lr), ...] in place;
    masked=True skips the elements whose gradient is exactly 0 (SparseGridAdam's torch path,
    training/optimizer.py:86-113).

    A segment may carry two more items, (..., scalars, flag): a float32 device tensor of 3 values
    {lr / (1 - b1^t), 1 / sqrt(1 - b2^t), the step size used when flag is nonzero} read by the
    kernel in place of (step, lr) — for launches replayed from a CUDA graph — and an int32 device
    flag or None.
    """
    import ctypes

    if not segments:
        return
    arr = (L.AdamSegment * len(segments))()
    dev = segments[0][0].device
    for k, seg in enumerate(segments):
        p, g, m, v, step, lr = seg[:6]
        scal, flag = (seg[6], seg[7]) if len(seg) > 6 else (None, None)
        for t, nm in ((p, "param"), (g, "grad"), (m, "exp_avg"), (v, "exp_avg_sq")):
            check_tensor(t, nm, device=dev)
            if t.numel() != p.numel():
                raise RuntimeError(f"{nm} has {t.numel()} elements, param has {p.numel()}")
        if scal is not None:
            check_tensor(scal, "scalars", device=dev)
            if scal.numel() < 3:
                raise RuntimeError("scalars holds fewer than 3 values")
        if flag is not None:
            check_tensor(flag, "flag", dtype=torch.int32, device=dev)
        arr[k] = L.AdamSegment(p.data_ptr(), g.data_ptr(), m.data_ptr(), v.data_ptr(), p.numel(), int(step), float(lr),
                               None if scal is None else scal.data_ptr(), None if flag is None else flag.data_ptr())
    call("vx_masked_adam_torch" if masked else "vx_adam_torch", ctypes.cast(arr, ctypes.c_void_p), len(segments),
         float(beta1), float(beta2), float(eps), stream_ptr(dev))


def adam_update(param, grad, exp_avg, exp_avg_sq, step, beta1, beta2, lr, eps, masked):
    for t, nm in ((param, "param"), (grad, "grad"), (exp_avg, "exp_avg"), (exp_avg_sq, "exp_avg_sq")):
        check_tensor(t, nm)
    call("vx_masked_adam_upd" if masked else "vx_adam_upd", ptr(param), ptr(grad), ptr(exp_avg), ptr(exp_avg_sq),
         param.numel(), int(step), float(beta1), float(beta2), float(lr), float(eps), stream_ptr(param.device))


def masked_adam_update_dev(param, grad, exp_avg, exp_avg_sq, step_size, beta1, beta2, eps):
    """The masked (reference-formula) update with its step size read from device memory
    (`step_size`: a float32 device tensor, from `adam_reference_step_size`)."""
    for t, nm in ((param, "param"), (grad, "grad"), (exp_avg, "exp_avg"), (exp_avg_sq, "exp_avg_sq"),
                  (step_size, "step_size")):
        check_tensor(t, nm, device=param.device)
    call("vx_masked_adam_upd_dev", ptr(param), ptr(grad), ptr(exp_avg), ptr(exp_avg_sq), param.numel(),
         ptr(step_size), float(beta1), float(beta2), float(eps), stream_ptr(param.device))


def adam_reference_step_size(step: int, beta1: float, beta2: float, lr: float) -> float:
    """The reference formula's step size, exactly as the masked update computes it from (step, lr)."""
    return float(L.query("vx_adam_reference_step_size", int(step), float(beta1), float(beta2), float(lr)))


def adam_torch_step_scalars(step: int, beta1: float, beta2: float, lr: float):
    """(lr / (1 - b1^t), 1 / sqrt(1 - b2^t)) exactly as `adam_torch` computes them from (step, lr)."""
    import ctypes

    out = (ctypes.c_float * 2)()
    L.query("vx_adam_torch_step_scalars", int(step), float(beta1), float(beta2), float(lr), out)
    return float(out[0]), float(out[1])


# ------------------------------------------------------------------ tensor-core wait policy ------


class tc_guard:
    """Context manager: MLP launches of this thread inside it poll the tensor core's mbarriers at
    most `wait_polls` times per wait (None: the library default) and increment the int32 device
    tensor `status` (or nothing, when None) for every block that gave up. Restores the previous
    policy on exit. Launches captured into a CUDA graph keep the policy they were captured with."""

    _local = threading.local()

    def __init__(self, status: Optional[torch.Tensor], wait_polls: Optional[int] = None):
        if status is not None:
            check_tensor(status, "status", dtype=torch.int32)
        self.status = status
        self.polls = -1 if wait_polls is None else int(wait_polls)

    def __enter__(self):
        stack = getattr(self._local, "stack", None)
        if stack is None:
            stack = self._local.stack = []
        stack.append((self.status, self.polls))
        call("vx_tc_guard", ptr(self.status), self.polls)
        return self

    def __exit__(self, *exc):
        stack = self._local.stack
        stack.pop()
        status, polls = stack[-1] if stack else (None, -1)
        call("vx_tc_guard", ptr(status), polls)
        return False


class StatusWatch:
    """Reads a device int32 status word without synchronising: every `every`-th `after_step()`
    queues its copy to pinned host memory on the current stream; `check()` raises if a copy that
    has landed holds a nonzero value (an earlier step's tensor-core wait gave up). A copy costs the
    stream a device-to-host round trip (~10 us in a step of graph replays), hence the interval."""

    def __init__(self, status: torch.Tensor, what: str, slots: int = 4, every: int = 1):
        self.status = status
        self.what = what
        self.every = max(int(every), 1)
        self.calls = 0
        self.host = torch.zeros(slots, dtype=torch.int32).pin_memory()
        self.events = [None] * slots
        self.slot = 0

    def after_step(self) -> None:
        self.calls += 1
        if self.calls % self.every:
            return
        s = self.slot
        if self.events[s] is not None:
            self.events[s].synchronize()  # the copy queued `slots` steps ago
            self._test(s)
        self.host[s:s + 1].copy_(self.status, non_blocking=True)
        ev = self.events[s] or torch.cuda.Event()
        ev.record()
        self.events[s] = ev
        self.slot = (s + 1) % len(self.events)

    def check(self) -> None:
        for s, ev in enumerate(self.events):
            if ev is not None and ev.query():
                self._test(s)

    def _test(self, s: int) -> None:
        v = int(self.host[s])
        if v:
            raise RuntimeError(f"{self.what}: {v} block(s) gave up waiting on the tensor core; the gradients "
                               f"and colours of that step are invalid")

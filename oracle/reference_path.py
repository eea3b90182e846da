"""Test infrastructure (the oracle): a CPU restatement of the VoxNeuS hot path.

Plain PyTorch tensor ops, run on CPU (float32 for parity, float64 for the error budget).
Each function names the reference file:line (paths inside ``Code/`` of rishidevde/VoxNeus)
whose algorithm it restates. This module is the checker: only ``tests/``,
``__graft_entry__.smoke()`` and the CPU-baseline legs of ``bench.py`` use it.

Pinned by ``tests/test_oracle_golden.py`` against vectors that the reference itself
produced (``tests/golden/make_golden.py``).
"""

from __future__ import annotations

import math
from typing import Dict, List, Optional, Sequence

import numpy as np
import torch
import torch.nn.functional as F

# ---------------------------------------------------------------------------------------
# S3 / S2 / S8: coordinates, trilinear SDF query, Eq.6/Eq.7 interpolated gradients
# ---------------------------------------------------------------------------------------


def voxel_size(xyz_min: torch.Tensor, xyz_max: torch.Tensor, res: torch.Tensor) -> torch.Tensor:
    """epsilon = (max - min) / (res - 1).  models/sdf_grid.py:83-88."""
    return (xyz_max - xyz_min) / (res.to(xyz_min.dtype) - 1.0)


def world_to_grid(xyz, xyz_min, xyz_max, res):
    """Continuous grid-index coordinates.  geometry/coordinates.py:10-29."""
    n = (xyz - xyz_min) / (xyz_max - xyz_min + 1e-8)
    return n * (res.to(xyz.dtype) - 1.0)


def corners_and_weights(coords: torch.Tensor, res: Sequence[int]):
    """8 corner indices (binary order 000..111, z fastest) and trilinear weights.

    geometry/coordinates.py:55-124: clamp to [0, R-1.0001], floor, clamp corners to
    [0, R-1], weights as products of (1-d) and d in the order (x*y)*z.
    """
    rx, ry, rz = (int(r) for r in res)
    hi = torch.tensor([rx - 1.0001, ry - 1.0001, rz - 1.0001], device=coords.device)
    hi = hi.to(coords.dtype) if coords.dtype == torch.float64 else hi
    cc = torch.clamp(coords, min=torch.zeros_like(hi), max=hi)
    lo = torch.floor(cc).to(torch.int64)
    up = lo + 1
    lim = torch.tensor([rx - 1, ry - 1, rz - 1], device=coords.device)
    lo = torch.minimum(torch.clamp(lo, min=0), lim)
    up = torch.minimum(torch.clamp(up, min=0), lim)
    d = cc - lo.to(cc.dtype)
    dx, dy, dz = d[..., 0:1], d[..., 1:2], d[..., 2:3]
    ox, oy, oz = 1.0 - dx, 1.0 - dy, 1.0 - dz
    sel = [(a, b, c) for a in (0, 1) for b in (0, 1) for c in (0, 1)]
    pick = (lo, up)
    corners = torch.stack(
        [torch.stack([pick[a][..., 0], pick[b][..., 1], pick[c][..., 2]], dim=-1) for a, b, c in sel],
        dim=-2,
    )
    wx, wy, wz = (ox, dx), (oy, dy), (oz, dz)
    weights = torch.cat([wx[a] * wy[b] * wz[c] for a, b, c in sel], dim=-1)
    return corners, weights


def query_sdf(grid5: torch.Tensor, xyz: torch.Tensor, xyz_min, xyz_max) -> torch.Tensor:
    """Trilinear SDF through grid_sample (border padding, align_corners=True).

    models/sdf_grid.py:90-120 (world -> [-1,1], coordinate flip to (z,y,x)).
    """
    lead = xyz.shape[:-1]
    p = xyz.reshape(1, 1, 1, -1, 3)
    n = (p - xyz_min) / (xyz_max - xyz_min + 1e-8)
    n = n * 2.0 - 1.0
    out = F.grid_sample(grid5, n.flip(-1), mode="bilinear", padding_mode="border", align_corners=True)
    return out.reshape(1, -1).T.reshape(*lead, 1)


def corner_normals(grid5: torch.Tensor, corners: torch.Tensor, eps: torch.Tensor) -> torch.Tensor:
    """Eq.6 central differences at corners, one-sided at the border.  geometry/gradients.py:59-100."""
    f = grid5.reshape(grid5.shape[-3:])
    rx, ry, rz = f.shape
    i, j, k = corners[..., 0], corners[..., 1], corners[..., 2]
    out = []
    for axis, (r, e) in enumerate(zip((rx, ry, rz), (eps[0], eps[1], eps[2]))):
        c = (i, j, k)[axis]
        cp = torch.clamp(c + 1, max=r - 1)
        cm = torch.clamp(c - 1, min=0)
        den = torch.clamp((cp - cm).to(f.dtype) * e, min=e)
        ip = [i, j, k]
        im = [i, j, k]
        ip[axis] = cp
        im[axis] = cm
        out.append((f[ip[0], ip[1], ip[2]] - f[im[0], im[1], im[2]]) / den)
    return torch.stack(out, dim=-1)


def interpolate_gradients(grid5, coords, eps, res):
    """Eq.7: g = sum_k w_k n[c_k]; normal = g/(|g|+1e-8).  geometry/gradients.py:103-139."""
    corners, weights = corners_and_weights(coords, res)
    n = corner_normals(grid5, corners, eps)
    g = torch.sum(weights.unsqueeze(-1) * n, dim=-2)
    normal = g / (torch.linalg.norm(g, dim=-1, keepdim=True) + 1e-8)
    return g, normal, corners, weights


def query_normals(grid5, xyz, xyz_min, xyz_max):
    """models/sdf_grid.py:122-160 (interpolated mode)."""
    res = torch.tensor(grid5.shape[-3:], dtype=torch.float32, device=grid5.device)
    coords = world_to_grid(xyz, xyz_min, xyz_max, res)
    eps = voxel_size(xyz_min, xyz_max, res)
    return interpolate_gradients(grid5, coords, eps, [int(r) for r in res])


# ---------------------------------------------------------------------------------------
# S1 / S0 / S4-S7 / S20: ray bounds and the multistep NeuS sampler
# ---------------------------------------------------------------------------------------


def near_far_from_sphere(o, d, radius: float = 1.0):
    """rendering/rays.py:102-128."""
    a = torch.sum(d ** 2, dim=-1, keepdim=True)
    b = 2.0 * torch.sum(o * d, dim=-1, keepdim=True)
    mid = 0.5 * (-b) / a
    near = torch.clamp(mid - radius, min=0.05)
    far = torch.clamp(mid + radius, min=near + 0.1)
    return near, far


def sample_pdf(bins, weights, n_samples: int, det: bool, u=None, eps: float = 1e-5, return_detail=False):
    """Inverse-CDF sampling.  rendering/sampler.py:11-66.

    ``u`` replaces the ``torch.rand`` draw of the stochastic branch (sampler.py:44) so that
    a caller can feed identical uniforms to two implementations.
    """
    w = weights + eps
    pdf = w / torch.sum(w, dim=-1, keepdim=True)
    cdf = torch.cumsum(pdf, dim=-1)
    cdf = torch.cat([torch.zeros_like(cdf[..., :1]), cdf], dim=-1)
    lead = list(cdf.shape[:-1])
    if det:
        u = torch.linspace(0.5 / n_samples, 1.0 - 0.5 / n_samples, steps=n_samples, dtype=cdf.dtype,
                           device=cdf.device)
        u = u.expand(lead + [n_samples]).contiguous()
    else:
        if u is None:
            u = torch.rand(lead + [n_samples], dtype=cdf.dtype, device=cdf.device)
        u = u.to(cdf.dtype).contiguous()
    idx = torch.searchsorted(cdf, u, right=True)
    below = torch.clamp(idx - 1, min=0)
    above = torch.clamp(idx, max=cdf.shape[-1] - 1)
    c0 = torch.gather(cdf, -1, below)
    c1 = torch.gather(cdf, -1, above)
    b0 = torch.gather(bins, -1, below)
    b1 = torch.gather(bins, -1, above)
    den = c1 - c0
    den = torch.where(den < eps, torch.ones_like(den), den)
    t = (u - c0) / den
    out = b0 + t * (b1 - b0)
    if return_detail:
        return out, {"cdf": cdf, "u": u, "indices": idx}
    return out


def sample_stratified(near, far, n_samples: int, perturb: bool, t_rand=None):
    """rendering/sampler.py:85-125.  ``t_rand`` replaces the rand_like draw (sampler.py:117)."""
    t = torch.linspace(0.0, 1.0, steps=n_samples, dtype=near.dtype, device=near.device)
    z = near * (1.0 - t) + far * t
    if perturb:
        mids = 0.5 * (z[..., 1:] + z[..., :-1])
        upper = torch.cat([mids, z[..., -1:]], dim=-1)
        lower = torch.cat([z[..., :1], mids], dim=-1)
        if t_rand is None:
            t_rand = torch.rand_like(z)
        z = lower + (upper - lower) * t_rand.to(z.dtype)
    dists = z[..., 1:] - z[..., :-1]
    dists = torch.cat([dists, dists[..., -1:]], dim=-1)
    return z, dists


def is_occupied(mask: torch.Tensor, pts: torch.Tensor, xyz_min, xyz_max) -> torch.Tensor:
    """rendering/occupancy_grid.py:122-147."""
    r = mask.shape[0]
    lead = pts.shape[:-1]
    p = pts.reshape(-1, 3)
    n = (p - xyz_min) / (xyz_max - xyz_min + 1e-8)
    inb = ((n >= 0.0) & (n <= 1.0)).all(dim=-1)
    c = torch.clamp(n * float(r), 0.0, float(r - 1.0001)).to(torch.int64)
    occ = mask[c[:, 0], c[:, 1], c[:, 2]] & inb
    return occ.reshape(lead)


def occupancy_update(density: torch.Tensor, mask: torch.Tensor, idx: torch.Tensor, sdf_fn, s, first: bool,
                     xyz_min, xyz_max, decay: float = 0.95, threshold: float = 0.01) -> None:
    """One EMA update of the occupancy grid at the drawn cells idx (3, n), in place.

    rendering/occupancy_grid.py:62-119: cell centres -> world points, SDF query, logistic density
    s*sig*(1-sig) with sig = sigmoid(s*sdf) (:15-22), near-surface floor 2*threshold where
    |sdf| < 2*|voxel step|, max with decay*previous after the first update, mask = density > threshold.
    Cells drawn more than once all read the previous value and write the same result.
    """
    r = density.shape[0]
    lo = torch.as_tensor(xyz_min, dtype=torch.float32)
    hi = torch.as_tensor(xyz_max, dtype=torch.float32)
    ix, iy, iz = idx[0], idx[1], idx[2]
    step = (hi - lo) / float(r)
    pts = torch.stack([lo[a] + ((i.float() + 0.5) / float(r)) * (hi[a] - lo[a]) for a, i in enumerate((ix, iy, iz))],
                      dim=-1)
    sdf = sdf_fn(pts).reshape(-1)
    s = torch.as_tensor(s, dtype=torch.float32)
    sig = torch.sigmoid(s * sdf)
    dens = s * sig * (1.0 - sig)
    near = (torch.abs(sdf) < 2.0 * torch.linalg.norm(step).item()).float()
    eff = torch.maximum(dens, near * (threshold * 2.0))
    upd = eff if first else torch.maximum(density[ix, iy, iz] * decay, eff)
    density[ix, iy, iz] = upd
    mask[ix, iy, iz] = upd > threshold


def up_sample(o, d, z, sdf, n_importance: int, inv_s: float, det: bool, occ_fn=None, u=None,
              return_detail=False):
    """One NeuS upsampling step.  rendering/sampler.py:243-292."""
    nr, ns = z.shape
    pts = o[:, None, :] + d[:, None, :] * z[..., :, None]
    radius = torch.linalg.norm(pts, ord=2, dim=-1, keepdim=False)
    inside = ((radius[:, :-1] < 1.0) | (radius[:, 1:] < 1.0)).to(z.dtype)
    sdf = sdf.reshape(nr, ns)
    f0, f1 = sdf[:, :-1], sdf[:, 1:]
    z0, z1 = z[:, :-1], z[:, 1:]
    fm = (f0 + f1) * 0.5
    cos = (f1 - f0) / (z1 - z0 + 1e-5)
    prev = torch.cat([torch.zeros([nr, 1], dtype=z.dtype, device=z.device), cos[:, :-1]], dim=-1)
    cos = torch.min(torch.stack([prev, cos], dim=-1), dim=-1)[0]
    cos = cos.clip(-1e3, 0.0) * inside
    dist = z1 - z0
    e0 = fm - cos * dist * 0.5
    e1 = fm + cos * dist * 0.5
    c0 = torch.sigmoid(e0 * inv_s)
    c1 = torch.sigmoid(e1 * inv_s)
    alpha = (c0 - c1 + 1e-5) / (c0 + 1e-5)
    trans = torch.cumprod(torch.cat([torch.ones([nr, 1], dtype=z.dtype, device=z.device), 1.0 - alpha + 1e-7], -1),
                          -1)[:, :-1]
    w = alpha * trans
    if occ_fn is not None:
        zm = (z0 + z1) * 0.5
        pm = o[:, None, :] + d[:, None, :] * zm[..., :, None]
        w = w * (occ_fn(pm).to(z.dtype) * 0.90 + 0.10)
    out = sample_pdf(z, w, n_importance, det=det, u=u, return_detail=return_detail)
    if return_detail:
        out[1]["weights"] = w
        return out
    return out


def cat_z_vals(o, d, z, new_z, sdf, sdf_fn, last: bool):
    """rendering/sampler.py:295-320 (concatenate, sort, query new SDF, reorder)."""
    nr, ns = z.shape
    ni = new_z.shape[1]
    zc, order = torch.sort(torch.cat([z, new_z], dim=-1), dim=-1)
    if not last:
        pts = o[:, None, :] + d[:, None, :] * new_z[..., :, None]
        fnew = sdf_fn(pts.reshape(-1, 3)).reshape(nr, ni)
        sdf = torch.gather(torch.cat([sdf, fnew], dim=-1), -1, order)
    return zc, sdf


def sampler_draws(n_rays: int, n_samples: int, n_importance: int, steps: int, perturb: bool,
                  device="cpu", dtype=torch.float32, generator=None):
    """The uniforms the reference sampler draws, in its order (sampler.py:117 then :44 per step)."""
    if not perturb:
        return None, [None] * steps
    t_rand = torch.rand((n_rays, n_samples), device=device, dtype=dtype, generator=generator)
    per = max(n_importance // steps, 1)
    us = [torch.rand((n_rays, per), device=device, dtype=dtype, generator=generator) for _ in range(steps)]
    return t_rand, us


def sample_multistep_sdf(o, d, near, far, sdf_fn, n_samples=64, n_importance=64, steps=4, perturb=False,
                         occ_fn=None, t_rand=None, us=None):
    """rendering/sampler.py:127-204.  Returns (z, dists, mid_z)."""
    z, dists = sample_stratified(near, far, n_samples, perturb, t_rand=t_rand)
    nr = z.shape[0]
    if n_importance > 0 and steps > 0:
        with torch.no_grad():
            pts = o[:, None, :] + d[:, None, :] * z[..., :, None]
            sdf = sdf_fn(pts.reshape(-1, 3)).reshape(nr, n_samples)
            per = max(n_importance // steps, 1)
            for i in range(steps):
                u = None if us is None else us[i]
                nz = up_sample(o, d, z, sdf, per, 64.0 * (2.0 ** i), det=not perturb, occ_fn=occ_fn, u=u)
                z, sdf = cat_z_vals(o, d, z, nz, sdf, sdf_fn, last=(i + 1 == steps))
    dists = z[..., 1:] - z[..., :-1]
    dists = torch.cat([dists, dists[..., -1:]], dim=-1)
    mid = z + dists * 0.5
    return z, dists, mid


# ---------------------------------------------------------------------------------------
# S9-S13, S18: variance, NeuS alpha, transmittance, compositing, s-gradient amplification
# ---------------------------------------------------------------------------------------


def variance_s(v: torch.Tensor, s_max: float = 300.0) -> torch.Tensor:
    """s = clamp(exp(10 v), 1e-4, s_max).  models/variance.py:38-41."""
    return torch.clamp(torch.exp(v * 10.0), min=1e-4, max=s_max)


def neus_alpha(sdf, normals, dirs, dists, s, cos_anneal_ratio=0.0, use_iter_cos=False, eps=1e-5):
    """Eq.2.  rendering/neus_alpha.py:12-81.  sdf (...,1), normals/dirs (...,3), dists (...)."""
    if sdf.ndim < normals.ndim:
        sdf = sdf.unsqueeze(-1)
    if dists.ndim < normals.ndim:
        dists = dists.unsqueeze(-1)
    cos = torch.sum(normals * dirs, dim=-1, keepdim=True)
    if use_iter_cos:
        cos = -(F.relu(-cos * 0.5 + 0.5) * (1.0 - cos_anneal_ratio) + F.relu(-cos) * cos_anneal_ratio)
    off = 0.5 * dists * cos
    p0 = torch.sigmoid(s * (sdf - off))
    p1 = torch.sigmoid(s * (sdf + off))
    a = (p0 - p1) / torch.clamp(p0, min=eps)
    a = torch.clamp(a, min=0.0, max=1.0)
    if a.shape[-1] == 1 and sdf.ndim == normals.ndim:
        a = a.squeeze(-1)
    return a


def composite_weights(alpha, eps: float = 1e-7):
    """T = exclusive cumprod of clamp(1-a+eps,0,1); w = a T, zeroed where T<1e-4.

    rendering/volume_render.py:12-40.
    """
    n = alpha.shape[0]
    q = torch.clamp(1.0 - alpha + eps, min=0.0, max=1.0)
    t = torch.cumprod(torch.cat([torch.ones([n, 1], dtype=alpha.dtype, device=alpha.device), q], dim=-1),
                      dim=-1)[:, :-1]
    w = alpha * t
    w = torch.where(t < 1e-4, torch.zeros_like(w), w)
    return w, t


def volume_render(colors, sdf, normals, dirs, z, dists, s, pts=None, radius=1.0, background=None,
                  cos_anneal_ratio=0.0, use_iter_cos=False) -> Dict[str, torch.Tensor]:
    """rendering/volume_render.py:57-153."""
    if dirs.ndim == 2:
        dirs = dirs.unsqueeze(1).expand(-1, colors.shape[1], -1)
    a = neus_alpha(sdf, normals, dirs, dists, s, cos_anneal_ratio, use_iter_cos)
    if pts is not None and radius is not None and radius > 0:
        a = a * (torch.linalg.norm(pts, ord=2, dim=-1) < radius).to(a.dtype).detach()
    w, t = composite_weights(a)
    rgb = torch.sum(w.unsqueeze(-1) * colors, dim=1)
    depth = torch.sum(w * z, dim=-1, keepdim=True)
    nrm = torch.sum(w.unsqueeze(-1) * normals, dim=1)
    nrm = nrm / (torch.linalg.norm(nrm, dim=-1, keepdim=True) + 1e-8)
    opacity = torch.sum(w, dim=-1, keepdim=True)
    if background is not None:
        bg = background.unsqueeze(0).expand_as(rgb) if background.ndim == 1 else background
        rgb = rgb + (1.0 - opacity) * bg
    return {"rgb": rgb, "depth": depth, "normal": nrm, "opacity": opacity, "weights": w, "alpha": a,
            "transmittance": t}


def huber(pred, target, delta: float = 0.1):
    """rendering/volume_render.py:43-54."""
    diff = torch.abs(pred - target)
    return torch.mean(torch.where(diff < delta, 0.5 * diff ** 2 / delta, diff - 0.5 * delta))


def amplify_s_gradient(param: torch.Tensor, k: float = 5.0) -> bool:
    """training/scheduler.py:14-33: grad *= k when grad < 0."""
    if param.grad is None:
        return False
    with torch.no_grad():
        if param.grad.item() < 0.0:
            param.grad.mul_(k)
            return True
    return False


# ---------------------------------------------------------------------------------------
# A1: appearance branch (hash grid, SH-4 view embedding, 2-layer MLP)
# ---------------------------------------------------------------------------------------

HASH_PRIMES = (1, 2654435761, 805459861)


def hash_level_resolutions(n_levels=16, base=16, finest=2048) -> List[int]:
    """N_l = floor(N_min b^l), b = exp((ln N_max - ln N_min)/(L-1)).  models/radiance_hash.py:45-47,103."""
    b = math.exp((math.log(finest) - math.log(base)) / max(n_levels - 1, 1))
    return [math.floor(base * (b ** lvl)) for lvl in range(n_levels)]


def level_weight(level: int, active_levels: Optional[float]) -> float:
    """NeuS2 lambda mask.  models/radiance_hash.py:91-100."""
    if active_levels is None:
        return 1.0
    li = level + 1.0
    if li <= active_levels:
        return 1.0
    if li - 1.0 < active_levels < li:
        return active_levels - (li - 1.0)
    return 0.0


def hash_index_np(c: np.ndarray, log2_size: int = 19) -> np.ndarray:
    """Spatial hash in uint32 arithmetic (low bits of the int64 hash of radiance_hash.py:65-69)."""
    c = c.astype(np.uint64)
    h = (c[..., 0] * np.uint64(HASH_PRIMES[0])) ^ (c[..., 1] * np.uint64(HASH_PRIMES[1])) ^ \
        (c[..., 2] * np.uint64(HASH_PRIMES[2]))
    return (h & np.uint64((1 << log2_size) - 1)).astype(np.int64)


def hash_encode(norm_xyz, embeddings, resolutions: Sequence[int], active_levels=None):
    """Multiresolution hash encoding.  models/radiance_hash.py:71-166 with the clamp of :211-231."""
    x = torch.clamp(norm_xyz, min=0.0, max=1.0)
    lead = x.shape[:-1]
    xf = x.reshape(-1, 3)
    n_levels, tsize, nf = embeddings.shape
    primes = torch.tensor(HASH_PRIMES, dtype=torch.int64, device=xf.device)
    outs = []
    sel = [(a, b, c) for a in (0, 1) for b in (0, 1) for c in (0, 1)]
    for lvl in range(n_levels):
        lw = level_weight(lvl, active_levels)
        if lw == 0.0:
            outs.append(torch.zeros((xf.shape[0], nf), dtype=embeddings.dtype, device=xf.device))
            continue
        sx = xf * torch.tensor(resolutions[lvl], dtype=torch.float32, device=xf.device).to(xf.dtype)
        lo = torch.floor(sx).to(torch.int64)
        up = lo + 1
        dd = sx - lo.to(sx.dtype)
        wx = (1.0 - dd[:, 0:1], dd[:, 0:1])
        wy = (1.0 - dd[:, 1:2], dd[:, 1:2])
        wz = (1.0 - dd[:, 2:3], dd[:, 2:3])
        pick = (lo, up)
        emb = embeddings[lvl]
        feat = None
        for a, b, c in sel:
            cc = torch.stack([pick[a][:, 0], pick[b][:, 1], pick[c][:, 2]], dim=-1)
            h = torch.remainder((cc[:, 0] * primes[0]) ^ (cc[:, 1] * primes[1]) ^ (cc[:, 2] * primes[2]), tsize)
            term = (wx[a] * wy[b] * wz[c]) * emb[h]
            feat = term if feat is None else feat + term
        if lw < 1.0:
            feat = feat * lw
        outs.append(feat)
    return torch.cat(outs, dim=-1).reshape(*lead, n_levels * nf)


SH_C = (0.28209479177387814, 0.4886025119029199, 1.0925484305920792, 0.31539156525252005,
        0.5462742152960396, 0.5900435899266435, 2.890611442640554, 0.4570457994644658,
        0.3731763325901154, 1.445305721320277)


def sh4(dirs):
    """Degree-4 (16 coefficient) real spherical harmonics.  models/embedder.py:55-87."""
    x, y, z = dirs[..., 0:1], dirs[..., 1:2], dirs[..., 2:3]
    c = SH_C
    r = [torch.full_like(x, c[0]),
         -c[1] * y, c[1] * z, -c[1] * x,
         c[2] * x * y, -c[2] * y * z, c[3] * (2.0 * z * z - x * x - y * y), -c[2] * x * z,
         c[4] * (x * x - y * y),
         -c[5] * y * (3.0 * x * x - y * y), c[6] * x * y * z, -c[7] * y * (4.0 * z * z - x * x - y * y),
         c[8] * z * (2.0 * z * z - 3.0 * x * x - 3.0 * y * y), -c[7] * x * (4.0 * z * z - x * x - y * y),
         c[9] * z * (x * x - y * y), -c[5] * x * (x * x - 3.0 * y * y)]
    return torch.cat(r, dim=-1)


def radiance_mlp(hash_feats, view_embed, normals, w0, b0, w1, b1):
    """[hash, SH, n] -> Linear -> ReLU -> Linear -> Sigmoid.  models/radiance_mlp.py:42-53,81-98."""
    h = torch.cat([hash_feats, view_embed, normals], dim=-1)
    return torch.sigmoid(F.linear(F.relu(F.linear(h, w0, b0)), w1, b1))


# ---------------------------------------------------------------------------------------
# S15-S17, S19: active vertices, closed-form regularizers, grid upsampling
# ---------------------------------------------------------------------------------------


def extract_active_vertices(corners: torch.Tensor, res: Sequence[int]):
    """Unique sorted linear indices of all corners.  regularization/active_vertices.py:12-50."""
    rx, ry, rz = (int(r) for r in res)
    c = corners.reshape(-1, 3).to(torch.int64).clone()
    c[:, 0] = c[:, 0].clamp(0, rx - 1)
    c[:, 1] = c[:, 1].clamp(0, ry - 1)
    c[:, 2] = c[:, 2].clamp(0, rz - 1)
    lin = c[:, 0] * (ry * rz) + c[:, 1] * rz + c[:, 2]
    u = torch.unique(lin)
    iz = u % rz
    rem = u // rz
    return torch.stack([rem // ry, rem % ry, iz], dim=-1), u


def relax_filter(verts: torch.Tensor, xyz_min: torch.Tensor, eps: torch.Tensor, radius: float = 1.2):
    """Keep vertices with |min + idx*eps| < 1.2 when at least one qualifies.  training/trainer.py:262-266."""
    wc = xyz_min + verts.to(torch.float32) * eps
    keep = torch.linalg.norm(wc, dim=-1) < radius
    return verts[keep] if keep.sum() > 0 else verts


def band_filter(verts: torch.Tensor, grid3: torch.Tensor, eps_x: float, band_voxels: float = 3.0):
    """Narrow-band restriction |f(v)| < band*eps of the throughput workload (applied after relax)."""
    f = grid3[verts[:, 0], verts[:, 1], verts[:, 2]]
    return verts[torch.abs(f) < band_voxels * eps_x]


def _interior(verts, res):
    rx, ry, rz = res
    i, j, k = verts[:, 0], verts[:, 1], verts[:, 2]
    return (i > 0) & (i < rx - 1) & (j > 0) & (j < ry - 1) & (k > 0) & (k < rz - 1)


def eikonal(grid, verts, eps, res, weight: float = 1.0, eps_norm: float = 1e-8):
    """Closed-form eikonal loss and gradient (Eq.10-11).  regularization/eikonal.py:100-171.

    Returns (loss, grad (X,Y,Z)) with the gradient scaled by ``weight`` and 2/|V_R|.
    """
    f = grid.reshape(grid.shape[-3:])
    res = tuple(int(r) for r in res)
    g = torch.zeros(res, dtype=f.dtype, device=f.device)
    nv = verts.shape[0]
    if nv == 0:
        return torch.tensor(0.0, dtype=f.dtype, device=f.device), g
    v = verts[_interior(verts, res)]
    if v.shape[0] == 0:
        return torch.tensor(0.0, dtype=f.dtype, device=f.device), g
    i, j, k = v[:, 0], v[:, 1], v[:, 2]
    dx, dy, dz = 2.0 * eps[0], 2.0 * eps[1], 2.0 * eps[2]
    nx = (f[i + 1, j, k] - f[i - 1, j, k]) / dx
    ny = (f[i, j + 1, k] - f[i, j - 1, k]) / dy
    nz = (f[i, j, k + 1] - f[i, j, k - 1]) / dz
    nvec = torch.stack([nx, ny, nz], dim=-1)
    nn_ = torch.linalg.norm(nvec, dim=-1, keepdim=True)
    loss = torch.mean((nn_ - 1.0) ** 2)
    dl = (2.0 / nv) * (1.0 - 1.0 / (nn_ + eps_norm)) * nvec * weight
    for axis, den in enumerate((dx, dy, dz)):
        ip = [i, j, k]
        im = [i, j, k]
        ip[axis] = ip[axis] + 1
        im[axis] = im[axis] - 1
        g.index_put_(tuple(ip), dl[:, axis] / den, accumulate=True)
        g.index_put_(tuple(im), -dl[:, axis] / den, accumulate=True)
    return loss, g


def curvature(grid, verts, eps, res, weight: float = 1.0):
    """Closed-form Laplacian curvature loss and gradient (Eq.12-14).  regularization/curvature.py:100-165."""
    f = grid.reshape(grid.shape[-3:])
    res = tuple(int(r) for r in res)
    g = torch.zeros(res, dtype=f.dtype, device=f.device)
    nv = verts.shape[0]
    if nv == 0:
        return torch.tensor(0.0, dtype=f.dtype, device=f.device), g
    v = verts[_interior(verts, res)]
    if v.shape[0] == 0:
        return torch.tensor(0.0, dtype=f.dtype, device=f.device), g
    i, j, k = v[:, 0], v[:, 1], v[:, 2]
    e2 = (eps[0] * eps[0], eps[1] * eps[1], eps[2] * eps[2])
    fc = f[i, j, k]
    lap = [(f[i + 1, j, k] + f[i - 1, j, k] - 2.0 * fc) / e2[0],
           (f[i, j + 1, k] + f[i, j - 1, k] - 2.0 * fc) / e2[1],
           (f[i, j, k + 1] + f[i, j, k - 1] - 2.0 * fc) / e2[2]]
    loss = torch.mean(lap[0] ** 2 + lap[1] ** 2 + lap[2] ** 2)
    sc = 2.0 / nv * weight
    g.index_put_((i, j, k), sc * (-2.0 * lap[0] / e2[0] - 2.0 * lap[1] / e2[1] - 2.0 * lap[2] / e2[2]),
                 accumulate=True)
    for axis in range(3):
        ip = [i, j, k]
        im = [i, j, k]
        ip[axis] = ip[axis] + 1
        im[axis] = im[axis] - 1
        g.index_put_(tuple(ip), sc * (lap[axis] / e2[axis]), accumulate=True)
        g.index_put_(tuple(im), sc * (lap[axis] / e2[axis]), accumulate=True)
    return loss, g


def upsample_grid(grid5: torch.Tensor, new_res) -> torch.Tensor:
    """Trilinear, align_corners=True.  geometry/upsample.py:12-39."""
    shape = (new_res,) * 3 if isinstance(new_res, int) else tuple(new_res)
    with torch.no_grad():
        return F.interpolate(grid5, size=shape, mode="trilinear", align_corners=True)


# ---------------------------------------------------------------------------------------
# S14 + trainer math: the whole render and the timed training step
# ---------------------------------------------------------------------------------------


def sparse_adam_step(p, grad, state, lr, betas=(0.9, 0.99), eps=1e-8, formula: str = "torch"):
    """SparseGridAdam (training/optimizer.py:32-116): update only the grad != 0 entries.

    formula="torch": the vectorised torch path (optimizer.py:86-113),
        p -= lr/(1-b1^t) * m / (sqrt(v)/sqrt(1-b2^t) + eps).
    formula="cuda": the extension kernel the reference's optimizer dispatches to on a GPU
        (optimizer.py:64-77 -> cuda/adam_upd_kernel.cu:23-38 with the step size of
        cuda/adam_upd.cpp), p -= lr*sqrt(1-b2^t)/(1-b1^t) * m / (sqrt(v) + eps).
    The two differ only in where eps enters (by sqrt(1-b2^t)).
    """
    b1, b2 = betas
    if not state:
        state["step"] = 0
        state["exp_avg"] = torch.zeros_like(p)
        state["exp_avg_sq"] = torch.zeros_like(p)
    state["step"] += 1
    t = state["step"]
    with torch.no_grad():
        mask = grad != 0.0
        if not bool(mask.any()):
            return
        g = grad[mask]
        m = state["exp_avg"][mask] * b1 + (1.0 - b1) * g
        v = state["exp_avg_sq"][mask] * b2 + (1.0 - b2) * (g * g)
        state["exp_avg"][mask] = m
        state["exp_avg_sq"][mask] = v
        if formula == "cuda":
            step_size = lr * math.sqrt(1.0 - b2 ** t) / (1.0 - b1 ** t)
            den = torch.sqrt(v) + eps
        else:
            step_size = lr / (1.0 - b1 ** t)
            den = torch.sqrt(v) / math.sqrt(1.0 - b2 ** t) + eps
        p[mask] -= step_size * (m / den)


def lr_factor(step: int, total_steps: int) -> float:
    """Cosine decay of the hash and MLP learning rates to 0.05 (training/trainer.py:333)."""
    return (math.cos(math.pi * step / max(total_steps, 1)) + 1.0) * 0.5 * (1.0 - 0.05) + 0.05


class OracleScene:
    """Parameters of one scene with the reference's state_dict naming (models/voxneus.py:21-92).

    The tensors may live on any device: the oracle's ops follow the device of the grid.
    """

    def __init__(self, grid5, variance, embeddings, w0, b0, w1, b1, occupancy=None,
                 xyz_min=(-1.0, -1.0, -1.0), xyz_max=(1.0, 1.0, 1.0), s_max=300.0):
        self.grid = grid5
        self.variance = variance
        self.embeddings = embeddings
        self.w0, self.b0, self.w1, self.b1 = w0, b0, w1, b1
        self.occupancy = occupancy
        self.device = grid5.device
        self.xyz_min = torch.tensor(xyz_min, dtype=grid5.dtype, device=self.device)
        self.xyz_max = torch.tensor(xyz_max, dtype=grid5.dtype, device=self.device)
        self.s_max = s_max
        self.resolutions = hash_level_resolutions(embeddings.shape[0])

    def params(self):
        return [self.grid, self.variance, self.embeddings, self.w0, self.b0, self.w1, self.b1]

    def res(self):
        return [int(r) for r in self.grid.shape[-3:]]

    def eps(self):
        return voxel_size(self.xyz_min, self.xyz_max, torch.tensor(self.res(), dtype=torch.float32,
                                                                   device=self.device))

    def sdf_fn(self, p):
        return query_sdf(self.grid, p, self.xyz_min, self.xyz_max).squeeze(-1)

    def occ_fn(self, p):
        return is_occupied(self.occupancy, p, self.xyz_min, self.xyz_max)

    def render(self, o, d, near, far, n_samples=64, n_importance=64, steps=4, perturb=False,
               t_rand=None, us=None, active_levels=None, background=None, z_vals=None):
        """models/voxneus.py:169-260 (pass 1 sampler, pass 2 midpoints, pass 3 compositing).

        z_vals: the sampler's output for these rays, given instead of running the sampler (its
        dists and midpoints are then formed as in rendering/sampler.py:197-202)."""
        if z_vals is None:
            z, dists, mid = sample_multistep_sdf(o, d, near, far, self.sdf_fn, n_samples, n_importance, steps,
                                                 perturb, self.occ_fn if self.occupancy is not None else None,
                                                 t_rand=t_rand, us=us)
        else:
            z = z_vals
            dists = torch.cat([z[..., 1:] - z[..., :-1], z[..., -1:] - z[..., -2:-1]], dim=-1)
            mid = z + dists * 0.5
        pts = o.unsqueeze(1) + d.unsqueeze(1) * mid.unsqueeze(-1)
        dirs = d.unsqueeze(1).expand_as(pts)
        sdf = query_sdf(self.grid, pts, self.xyz_min, self.xyz_max)
        g, nrm, corners, _ = query_normals(self.grid, pts, self.xyz_min, self.xyz_max)
        nx = (pts - self.xyz_min) / (self.xyz_max - self.xyz_min + 1e-8)
        hf = hash_encode(nx, self.embeddings, self.resolutions, active_levels)
        rgb = radiance_mlp(hf, sh4(dirs), nrm, self.w0, self.b0, self.w1, self.b1)
        s = variance_s(self.variance, self.s_max)
        out = volume_render(rgb, sdf, nrm, dirs, mid, dists, s, pts=pts, radius=1.0, background=background)
        out.update({"pts": pts, "sdf_samples": sdf, "corner_indices": corners, "grad_samples": g,
                    "normal_samples": nrm, "z_vals": z, "dists": dists, "mid_z_vals": mid, "colors": rgb})
        return out

    def train_step(self, o, d, target, w_eik=0.1, w_curv=5e-4, band_voxels=None, amplify_k=None,
                   huber_delta=0.1, optimize=False, step=None, total_steps=40000, s_warmup_steps=5000,
                   lr_sdf=0.1, lr_hash=0.01, lr_mlp=0.001, lr_variance=0.0005, grid_adam="torch", **render_kw):
        """The timed unit: training/trainer.py:166-393 (render, Huber loss, backward, V_R with the
        relax filter, eikonal + curvature into grid.grad, s amplification, optimizer steps).

        step=None: the amplification runs when amplify_k is given and the learning rates are the
        base ones. step=k: the trainer's rules at step k: amplification (k = amplify_k or 5) only
        when step >= s_warmup_steps (:311-315), the hash and MLP learning rates scaled by the
        cosine factor and the variance learning rate multiplied by k when the gradient was
        amplified (:317-329). optimize=True runs SparseGridAdam(0.9, 0.99) on the grid (formula
        `grid_adam`, see sparse_adam_step) and torch.optim.Adam(0.9, 0.999) on the rest
        (training/optimizer.py:119-154); the state persists across calls on this scene.
        Returns the losses, |V_R|, the V_R linear indices, the amplification flag and the
        gradients of every parameter (after the amplification).
        """
        for p in self.params():
            p.grad = None
        near, far = near_far_from_sphere(o, d, radius=1.0)
        out = self.render(o, d, near, far, **render_kw)
        loss = huber(out["rgb"], target, huber_delta)
        loss.backward()
        verts, _ = extract_active_vertices(out["corner_indices"], self.res())
        verts = relax_filter(verts, self.xyz_min.float(), self.eps().float())
        if band_voxels is not None:
            verts = band_filter(verts, self.grid.detach().reshape(self.res()), float(self.eps()[0]), band_voxels)
        g3 = self.grid.detach().reshape(self.res())
        le, ge = eikonal(g3, verts, self.eps(), self.res(), weight=w_eik)
        lc, gc = curvature(g3, verts, self.eps(), self.res(), weight=w_curv)
        with torch.no_grad():
            self.grid.grad.add_(ge.reshape(self.grid.shape))
            self.grid.grad.add_(gc.reshape(self.grid.shape))
        amplified = False
        k = 5.0 if amplify_k is None else float(amplify_k)
        if step is None:
            if amplify_k is not None:
                amplified = amplify_s_gradient(self.variance, k)
            lrs = (lr_hash, lr_mlp, lr_variance)
        else:
            if step >= s_warmup_steps:
                amplified = amplify_s_gradient(self.variance, k)
            f = lr_factor(step, total_steps)
            lrs = (lr_hash * f, lr_mlp * f, lr_variance * (k if amplified else 1.0))
        grads = {"grid": self.grid.grad.clone(), "variance": self.variance.grad.clone(),
                 "embeddings": self.embeddings.grad.clone(), "w0": self.w0.grad.clone(),
                 "b0": self.b0.grad.clone(), "w1": self.w1.grad.clone(), "b1": self.b1.grad.clone()}
        if optimize:
            if not hasattr(self, "_opt_state"):
                self._opt_state = {}
                self._net_opt = torch.optim.Adam([{"params": [self.embeddings], "lr": lr_hash},
                                                  {"params": [self.w0, self.b0, self.w1, self.b1], "lr": lr_mlp},
                                                  {"params": [self.variance], "lr": lr_variance}],
                                                 betas=(0.9, 0.999), eps=1e-8)
            for grp, lr in zip(self._net_opt.param_groups, lrs):
                grp["lr"] = lr
            sparse_adam_step(self.grid, self.grid.grad, self._opt_state, lr=lr_sdf, formula=grid_adam)
            self._net_opt.step()
        r1, r2 = self.res()[1], self.res()[2]
        lin = verts[:, 0] * (r1 * r2) + verts[:, 1] * r2 + verts[:, 2]
        return {"loss_rgb": loss.detach(), "loss_eik": le, "loss_curv": lc, "n_active": verts.shape[0],
                "vr_linear": lin, "amplified": amplified, "render": out, "grads": grads}

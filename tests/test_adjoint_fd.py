"""Adjoint check: hand-written gradients vs FP64 autograd and FP64 central finite differences.

Workload: 96^3 grid (sphere SDF + N(0, 0.02)), 512 random rays, 64 stratified samples per ray
(n_importance = 0, so sample positions do not depend on the grid), colours from a fixed random
head c = W tanh(B [n; SH16(d)]) (3x64, 64x19), V_R = all sample corners in the relax sphere.
Objective J = <rgb, C> + (1/|V_R|) sum_valid (|n|-1)^2 + (1/|V_R|) sum_valid sum_a L_a^2 — the
function whose exact gradient is the render adjoint plus the closed-form eikonal and curvature
gradients (Eq.11, Eq.14). Checks:
  1. every grid value and dL/dv: the sm_100a adjoints (FP32) against the oracle's FP64
     autograd gradient, within 1e-4 of the largest magnitude;
  2. spot checks: the FP64 autograd gradient against FP64 central finite differences (h=1e-3)
     on the largest-gradient entries and random support entries, within 1e-3 relative where the
     function is smooth there (FD at h and h/2 agree to 1e-4; the others sit on a clamp/cutoff
     kink and are counted, not compared).
"""


import pytest
import torch

from oracle import reference_path as O

pytestmark = pytest.mark.gpu


def _setup(dtype=torch.float32):
    from voxneus_b200 import synthetic

    grid = synthetic.sphere_grid(96, 0.5, 0.02, seed=4)
    pool = synthetic.RayPool(n_cams=16, width=200, height=150, focal=180.0, seed=9)
    o, d = pool.sample(512)
    g = torch.Generator().manual_seed(10)
    Wc = torch.randn(3, 64, generator=g) * 0.3
    Bc = torch.randn(64, 19, generator=g) * 0.5
    C = torch.randn(512, 3, generator=g)
    return grid, o, d, Wc, Bc, C


def _objective_oracle(grid, v, o, d, Wc, Bc, C, verts):
    """J in the oracle's torch ops (any dtype)."""
    dt = grid.dtype
    lo = torch.tensor([-1.0] * 3, dtype=dt)
    hi = torch.tensor([1.0] * 3, dtype=dt)
    o, d = o.to(dt), d.to(dt)
    near, far = O.near_far_from_sphere(o, d)
    z, dists, mid = O.sample_multistep_sdf(o, d, near, far, None, 64, 0, 4, False)
    pts = o.unsqueeze(1) + d.unsqueeze(1) * mid.unsqueeze(-1)
    sdf = O.query_sdf(grid, pts, lo, hi)
    _, nrm, _, _ = O.query_normals(grid, pts, lo, hi)
    dirs = d.unsqueeze(1).expand_as(pts)
    feat = torch.cat([nrm, O.sh4(dirs)], -1)
    col = torch.tanh(feat @ Bc.to(dt).T) @ Wc.to(dt).T
    s = O.variance_s(v)
    out = O.volume_render(col, sdf, nrm, dirs, mid, dists, s, pts=pts, radius=1.0)
    J = (out["rgb"] * C.to(dt)).sum()
    f = grid.reshape(96, 96, 96)
    res = (96, 96, 96)
    eps = O.voxel_size(lo, hi, torch.tensor(res, dtype=dt))
    inner = O._interior(verts, res)
    vi = verts[inner]
    i, j, k = vi[:, 0], vi[:, 1], vi[:, 2]
    nx = (f[i + 1, j, k] - f[i - 1, j, k]) / (2 * eps[0])
    ny = (f[i, j + 1, k] - f[i, j - 1, k]) / (2 * eps[1])
    nz = (f[i, j, k + 1] - f[i, j, k - 1]) / (2 * eps[2])
    nn = torch.sqrt(nx ** 2 + ny ** 2 + nz ** 2)
    nv = verts.shape[0]
    fc = f[i, j, k]
    lap = [(f[i + 1, j, k] + f[i - 1, j, k] - 2 * fc) / eps[0] ** 2, (f[i, j + 1, k] + f[i, j - 1, k] - 2 * fc) / eps[1] ** 2,
           (f[i, j, k + 1] + f[i, j, k - 1] - 2 * fc) / eps[2] ** 2]
    J = J + ((nn - 1) ** 2).sum() / nv + (lap[0] ** 2 + lap[1] ** 2 + lap[2] ** 2).sum() / nv
    return J, mid


def test_adjoint_against_fp64_autograd_and_central_fd():
    from voxneus_b200 import ops
    from voxneus_b200.models import DenseSDFGrid, SingleVarianceNetwork

    grid, o, d, Wc, Bc, C = _setup()
    # V_R: every sample corner in the relax sphere (positions are grid independent here)
    with torch.no_grad():
        near, far = O.near_far_from_sphere(o, d)
        _, _, mid = O.sample_multistep_sdf(o, d, near, far, None, 64, 0, 4, False)
        pts = o.unsqueeze(1) + d.unsqueeze(1) * mid.unsqueeze(-1)
        _, _, corners, _ = O.query_normals(grid, pts, torch.tensor([-1.0] * 3), torch.tensor([1.0] * 3))
        verts, _ = O.extract_active_vertices(corners, (96, 96, 96))
        lo = torch.tensor([-1.0] * 3)
        verts = O.relax_filter(verts, lo, O.voxel_size(lo, -lo, torch.tensor([96.0] * 3)))

    # FP64 oracle gradient
    g64 = grid.double().clone().requires_grad_(True)
    v64 = torch.tensor(0.3, dtype=torch.float64, requires_grad=True)
    J64, _ = _objective_oracle(g64, v64, o, d, Wc, Bc, C, verts)
    J64.backward()

    # sm_100a path: geometry + colour head (torch) + fused composite + fused regularizer stencil
    dev = torch.device("cuda")
    sg = DenseSDFGrid(96).to(dev)
    with torch.no_grad():
        sg.grid.copy_(grid.to(dev))
    var = SingleVarianceNetwork(0.3).to(dev)
    od, dd = o.to(dev).contiguous(), d.to(dev).contiguous()
    lo3, hi3 = sg.bounds()
    _, dists, midd = ops.sample_multistep(sg.grid.detach(), lo3, hi3, od, dd, None, None, 64, 0, 4, False)
    assert torch.allclose(midd.cpu(), mid.float(), rtol=1e-6, atol=1e-6)
    bm = ops.new_bitmap([96] * 3, dev)
    sdf, nrm, _ = ops.RenderGeometryFn.apply(sg.grid, od, dd, midd, lo3, hi3, bm, False)
    dirs = dd.unsqueeze(1).expand(-1, 64, -1)
    feat = torch.cat([nrm, ops.sh4(dirs.contiguous())], -1)
    col = torch.tanh(feat @ Bc.to(dev).T) @ Wc.to(dev).T
    outs = ops.CompositeFn.apply(col, sdf, nrm, var.variance, dd, midd, dists, None, od, True, 300.0, 1.0, None,
                                 False, 0.0, 0.0, None)
    (outs[0] * C.to(dev)).sum().backward()
    fb = ops.new_filtered([96] * 3, dev)
    counts = ops.vr_count(bm, sg.grid.detach(), [96] * 3, lo3, hi3, 1.2, 0.0, filtered=fb)
    assert int(ops.final_count(counts, 1.2, 0.0)) == verts.shape[0]
    ops.reg_stencil(sg.grid.detach(), fb, [96] * 3, lo3, hi3, 1.2, 0.0, counts, 1.0, 1.0, sg.grid.grad)
    ours = sg.grid.grad.detach().cpu().double().reshape(96, 96, 96)
    ref = g64.grad.reshape(96, 96, 96)
    scale = float(ref.abs().max())
    err = float((ours - ref).abs().max())
    assert err <= 1e-4 * scale, f"grid gradient vs FP64 autograd: {err:.3e} of scale {scale:.3e}"
    dv = float(var.variance.grad)
    assert abs(dv - float(v64.grad)) <= 1e-4 * abs(float(v64.grad)) + 1e-7, (dv, float(v64.grad))

    # FP64 autograd vs FP64 central finite differences on spot-checked entries
    flat = ref.reshape(-1)
    top = torch.topk(flat.abs(), 12).indices
    support = torch.nonzero(flat.abs() > 1e-3 * scale).reshape(-1)
    gen = torch.Generator().manual_seed(3)
    rnd = support[torch.randperm(support.numel(), generator=gen)[:12]]
    idx = torch.unique(torch.cat([top, rnd]))
    base = grid.double().reshape(-1).clone()
    vd = torch.tensor(0.3, dtype=torch.float64)

    def J_at(vec, v=vd):
        with torch.no_grad():
            return float(_objective_oracle(vec.reshape(1, 1, 96, 96, 96), v, o, d, Wc, Bc, C, verts)[0])

    def fd(i, h):
        e = base.clone()
        e[i] += h
        jp = J_at(e)
        e[i] -= 2 * h
        jm = J_at(e)
        return (jp - jm) / (2 * h)

    compared, kinks = 0, 0
    for i in idx.tolist():
        a, b = fd(i, 1e-3), fd(i, 5e-4)
        if abs(a - b) > 1e-4 * max(abs(b), 1e-3 * scale):
            kinks += 1
            continue
        g = float(flat[i])
        assert abs(b - g) <= 1e-3 * max(abs(g), 1e-3 * scale), (i, b, g)
        assert abs(float(ours.reshape(-1)[i]) - b) <= 2e-3 * max(abs(b), 1e-3 * scale), (i, b)
        compared += 1
    assert compared >= len(idx) // 2, (compared, kinks)
    # dL/dv by central differences
    jp, jm = J_at(base, vd + 1e-4), J_at(base, vd - 1e-4)
    fdv = (jp - jm) / 2e-4
    assert abs(fdv - float(v64.grad)) <= 1e-3 * abs(fdv) + 1e-6, (fdv, float(v64.grad))

"""GPU parity of the sm_100a path against the oracle (and the reference's golden vectors).

Tolerances: values within 1e-5 relative, |a - b| <= 1e-5 * (|b| + scale), where scale is the
quantity's natural scale: 1 for colours, opacities, alphas, weights, transmittance and unit
normals (quantities in [0, 1] or of unit length, whose FP32 error is absolute: alpha =
(phi- - phi+)/phi- cancels to ~1e-7 absolute whatever its size), and the tensor's largest
magnitude otherwise. Gradients within 1e-4 relative to their largest magnitude (atomic
accumulation order differs). Integer outputs (corner indices, V_R, searchsorted indices)
bit-exact.
"""

import math

import numpy as np
import pytest
import torch

from oracle import reference_path as O

pytestmark = pytest.mark.gpu

DEV = "cuda"
VAL_TOL = 1e-5
GRAD_TOL = 1e-4


def rel_err(a, b):
    a = torch.as_tensor(a).double().cpu()
    b = torch.as_tensor(b).double().cpu()
    scale = max(float(b.abs().max()), 1e-30) if b.numel() else 1.0
    return float((a - b).abs().max() / scale) if b.numel() else 0.0


UNIT_SCALE = {"rgb", "opacity", "weights", "alpha", "transmittance", "normal", "normal_samples", "w", "T",
              "lattice normal"}


def assert_close(a, b, tol, what="", scale=None):
    a = torch.as_tensor(a).detach().double().cpu()
    b = torch.as_tensor(b).detach().double().cpu()
    assert a.shape == b.shape, (what, a.shape, b.shape)
    if scale is None:
        scale = float(b.abs().max()) if b.numel() else 0.0
        if what in UNIT_SCALE:
            scale = max(scale, 1.0)
    err = (a - b).abs()
    bound = tol * (b.abs() + max(scale, 1e-12))
    bad = err > bound
    assert not bool(bad.any()), f"{what}: max err {float(err.max()):.3e} vs scale {scale:.3e} ({int(bad.sum())} bad)"


@pytest.fixture(autouse=True)
def _lib_loaded():
    from voxneus_b200 import _lib

    _lib.load()


def to(t):
    return t.to(DEV)


# ------------------------------------------------------------------ field query (S2/S3/S8)


def test_field_query_matches_golden(golden):
    from voxneus_b200.models import DenseSDFGrid

    g = golden("field_query.npz")
    m = DenseSDFGrid([12, 10, 9]).to(DEV)
    with torch.no_grad():
        m.grid.copy_(to(g["grid"]))
    pts = to(g["pts"])
    sdf = m.query_sdf(pts)
    grad, normal, corners, weights = m.query_normals(pts)
    assert torch.equal(corners.cpu(), g["corners"])
    assert_close(sdf, g["sdf"], VAL_TOL, "sdf")
    assert_close(grad, g["grad"], VAL_TOL, "grad")
    assert_close(normal, g["normal"], VAL_TOL, "normal")
    assert_close(weights, g["weights"], VAL_TOL, "weights")
    loss = (grad * to(g["c1"])).sum() + (sdf * to(g["c2"])).sum() + (normal * to(g["c3"])).sum()
    loss.backward()
    assert_close(m.grid.grad, g["grid_grad"], GRAD_TOL, "grid grad")


def test_gradient_interp_reference_interface():
    """tests/test_cuda_parity.py:31-70 pattern: Eq.7 at grid coords, forward 1e-5, backward 1e-4."""
    from voxneus_b200.cuda import cuda_gradient_interp

    torch.manual_seed(42)
    res = 32
    vs = torch.tensor([2.0 / (res - 1)] * 3)
    grid = torch.randn(1, 1, res, res, res)
    coords = torch.rand(256, 3) * (res - 1.001)
    coords[:8] = torch.tensor([[0, 0, 0], [31, 31, 31], [30.9999, 0, 15], [0.5, 31, 0], [15, 15, 15],
                               [31, 0, 0], [0, 31, 31], [1e-7, 30.99, 2]], dtype=torch.float32)
    gref = grid.clone().requires_grad_(True)
    c, w = O.corners_and_weights(coords, [res] * 3)
    ref = torch.sum(w.unsqueeze(-1) * O.corner_normals(gref, c, vs), dim=-2)
    (ref ** 2).sum().backward()
    gd = to(grid).requires_grad_(True)
    out = cuda_gradient_interp(gd, to(coords), to(vs))
    assert_close(out, ref.detach(), VAL_TOL, "gradient_interp forward")
    (out ** 2).sum().backward()
    assert_close(gd.grad, gref.grad, GRAD_TOL, "gradient_interp backward")


def test_corners_weights_bit_exact():
    from voxneus_b200.geometry import get_voxel_corners_and_weights

    torch.manual_seed(0)
    res = [17, 9, 33]
    coords = torch.rand(5000, 3) * torch.tensor([17.5, 9.5, 33.5]) - 0.25
    coords[:3] = torch.tensor([[16.0, 8.0, 32.0], [15.9999, 7.99995, 0.0], [0.0, 3.0, 31.0]])
    c_ref, w_ref = O.corners_and_weights(coords, res)
    c, w = get_voxel_corners_and_weights(to(coords), res)
    assert torch.equal(c.cpu(), c_ref)
    assert_close(w, w_ref, VAL_TOL, "weights")


def test_lattice_query():
    from voxneus_b200 import ops

    torch.manual_seed(3)
    grid = torch.randn(1, 1, 20, 18, 22)
    lat = [11, 7, 13]
    sdf, nrm = ops.field_query_lattice(to(grid), (-1, -1, -1), (1, 1, 1), lat, (-1, -1, -1), (1, 1, 1))

    def lin(n):
        step = np.float32(2.0) / np.float32(n - 1)
        v = [np.float32(-1) + step * np.float32(i) if i < n // 2 else np.float32(1) - step * np.float32(n - 1 - i)
             for i in range(n)]
        return torch.tensor(np.array(v, dtype=np.float32))

    gx, gy, gz = torch.meshgrid(lin(11), lin(7), lin(13), indexing="ij")
    pts = torch.stack([gx, gy, gz], -1).reshape(-1, 3)
    lo, hi = torch.tensor([-1.0] * 3), torch.tensor([1.0] * 3)
    assert_close(sdf, O.query_sdf(grid, pts, lo, hi).reshape(-1), VAL_TOL, "lattice sdf")
    assert_close(nrm, O.query_normals(grid, pts, lo, hi)[1], VAL_TOL, "lattice normal")


# ------------------------------------------------------------------ sampler (S0-S7, S20)


def _scene_from(g):
    from voxneus_b200.models import VoxNeuS

    m = VoxNeuS(grid_res=list(g["grid"].shape[-3:]), hash_n_levels=16,
                hash_log2_size=int(g["embeddings"].shape[1]).bit_length() - 1, occupancy_res=8).to(DEV)
    sd = m.state_dict()
    sd["sdf_grid.grid"] = to(g["grid"])
    sd["variance_net.variance"] = to(g["variance"])
    sd["radiance_hash.encoder.embeddings"] = to(g["embeddings"])
    sd["radiance_mlp.net.0.weight"] = to(g["w0"])
    sd["radiance_mlp.net.0.bias"] = to(g["b0"])
    sd["radiance_mlp.net.2.weight"] = to(g["w1"])
    sd["radiance_mlp.net.2.bias"] = to(g["b1"])
    sd["occupancy_grid.occupancy_mask"] = to(g["occupancy"])
    m.load_state_dict(sd)
    return m


@pytest.mark.parametrize("name,perturb", [("render_det.npz", False), ("render_perturb.npz", True)])
def test_sampler_matches_golden(golden, name, perturb):
    from voxneus_b200.rendering import RaySampler

    g = golden(name)
    m = _scene_from(g)
    s = RaySampler(16, 16, perturb=perturb)
    randoms = (to(g["t_rand"]), to(g["us"])) if perturb else None
    z, dists, mid = s.sample_multistep_sdf(to(g["rays_o"]), to(g["rays_d"]), to(g["near"]), to(g["far"]),
                                           m.sdf_grid.sdf_fn(), up_sample_steps=4, occupancy_grid=m.occupancy_grid,
                                           randoms=randoms)
    assert_close(z, g["z"], VAL_TOL, "z")
    assert_close(mid, g["mid"], VAL_TOL, "mid")
    assert_close(dists, g["dists"], 1e-4, "dists")


def test_sample_pdf_indices_bit_exact_given_cdf():
    from voxneus_b200 import ops

    torch.manual_seed(11)
    bins = torch.sort(torch.rand(300, 40) * 4 + 1, dim=-1)[0]
    w = torch.rand(300, 39) ** 4
    w[:5] = 0
    u = torch.rand(300, 16)
    u[0, :4] = torch.tensor([0.0, 1.0, 0.5, 0.999999])
    ref, det = O.sample_pdf(bins, w, 16, det=False, u=u, return_detail=True)
    out, idx = ops.sample_pdf(to(bins), None, 16, det=False, u=to(u), cdf=to(det["cdf"]), return_indices=True)
    assert torch.equal(idx.cpu(), det["indices"])
    assert_close(out, ref, VAL_TOL, "samples given cdf")
    # full path (cdf rebuilt on the device), deterministic and stochastic
    out2 = ops.sample_pdf(to(bins), to(w), 16, det=False, u=to(u))
    assert_close(out2, ref, VAL_TOL, "samples")
    ref3 = O.sample_pdf(bins, w, 16, det=True)
    assert_close(ops.sample_pdf(to(bins), to(w), 16, det=True), ref3, VAL_TOL, "det samples")


def test_sample_pdf_golden(golden):
    from voxneus_b200.rendering import sample_pdf

    g = golden("sampler.npz")
    assert_close(sample_pdf(to(g["bins"]), to(g["weights"]), 16, det=True), g["det"], VAL_TOL, "det")
    assert_close(sample_pdf(to(g["bins"]), to(g["weights"]), 16, det=False, u=to(g["u"])), g["sto"], VAL_TOL, "sto")


def test_near_far_known_answer(golden):
    from voxneus_b200.rendering import near_far_from_sphere

    g = golden("sampler.npz")
    n, f = near_far_from_sphere(to(g["rays_o"]), to(g["rays_d"]))
    assert_close(n, g["near"], VAL_TOL, "near")
    assert_close(f, g["far"], VAL_TOL, "far")
    n, f = near_far_from_sphere(torch.tensor([[0.0, 0.0, 3.0]], device=DEV), torch.tensor([[0.0, 0.0, -1.0]], device=DEV))
    assert abs(n.item() - 2.0) < 1e-3 and abs(f.item() - 4.0) < 1e-3


def test_up_sample_single_step():
    from voxneus_b200.rendering import up_sample

    torch.manual_seed(5)
    nr, n = 50, 40
    o = torch.randn(nr, 3)
    o = 3.0 * o / o.norm(dim=-1, keepdim=True)
    d = -o / o.norm(dim=-1, keepdim=True) + 0.1 * torch.randn(nr, 3)
    d = d / d.norm(dim=-1, keepdim=True)
    z = torch.sort(torch.rand(nr, n) * 4 + 1, dim=-1)[0]
    sdf = torch.randn(nr, n) * 0.3
    u = torch.rand(nr, 16)
    ref = O.up_sample(o, d, z, sdf, 16, 128.0, det=False, u=u)
    out = up_sample(to(o), to(d), to(z), to(sdf), 16, 128.0, det=False, u=to(u))
    assert_close(out, ref, VAL_TOL, "up_sample")


@pytest.mark.parametrize("nr,n,ni", [(50, 64, 16), (7, 112, 16), (3, 1, 1), (5, 0, 9), (4, 300, 200)])
def test_cat_z_vals_matches_oracle(nr, n, ni):
    """rendering.cat_z_vals against the oracle's torch.sort + gather (rendering/sampler.py:295-320):
    the depths and the carried SDF values bit for bit, the new depths unsorted (sample_pdf with
    random draws), depths present in both lists, NaN depths (sorted last), an empty old list, and
    `last` (no query, SDF passed through)."""
    from voxneus_b200.models import DenseSDFGrid
    from voxneus_b200.rendering import cat_z_vals

    torch.manual_seed(31 + n)
    o = torch.randn(nr, 3)
    o = 2.5 * o / o.norm(dim=-1, keepdim=True)
    d = -o / o.norm(dim=-1, keepdim=True)
    z = torch.sort(torch.rand(nr, n) * 3 + 0.5, dim=-1)[0]
    nz = torch.rand(nr, ni) * 3 + 0.5
    if n > 2 and ni > 2:
        nz[:, 0] = z[:, 1]  # a depth in both lists
        nz[0, 1] = float("nan")
    grid = DenseSDFGrid(24).to(DEV)
    with torch.no_grad():
        grid.grid.normal_(0.0, 0.3)
    fn = grid.sdf_fn()
    with torch.no_grad():
        sdf = fn((to(o)[:, None, :] + to(d)[:, None, :] * to(z)[..., None]).reshape(-1, 3)).reshape(nr, n)
        ref_fn = lambda p: fn(to(p)).cpu()
        zr, sr = O.cat_z_vals(o, d, z, nz, sdf.cpu(), ref_fn, last=False)
        zg, sg = cat_z_vals(to(o), to(d), to(z), to(nz), sdf, fn, last=False)
        zl, sl = cat_z_vals(to(o), to(d), to(z), to(nz), sdf, fn, last=True)
    assert torch.equal(torch.nan_to_num(zg.cpu(), nan=7.0), torch.nan_to_num(zr, nan=7.0))
    assert torch.equal(torch.nan_to_num(sg.cpu(), nan=7.0), torch.nan_to_num(sr, nan=7.0))
    assert torch.equal(torch.nan_to_num(zl.cpu(), nan=7.0), torch.nan_to_num(zr, nan=7.0)) and sl is sdf
    assert bool(torch.isnan(zg[0]).any()) == (n > 2 and ni > 2) and (n < 3 or not bool(torch.isnan(zg[0, :-1]).any()))


@pytest.mark.parametrize("n", [40, 300])
def test_up_sample_with_occupancy_grid(n):
    """up_sample with an occupancy grid (rendering/sampler.py:243-292 with the occupancy factor
    0.9 occ + 0.1 of rendering/occupancy_grid.py:122-147 on each interval's midpoint) against the
    oracle, on a random 32^3 mask; 300 samples a ray takes more than eight 32-interval chunks."""
    from voxneus_b200.models import OccupancyGrid
    from voxneus_b200.rendering import up_sample

    torch.manual_seed(6 + n)
    nr = 50
    o = torch.randn(nr, 3)
    o = 3.0 * o / o.norm(dim=-1, keepdim=True)
    d = -o / o.norm(dim=-1, keepdim=True) + 0.1 * torch.randn(nr, 3)
    d = d / d.norm(dim=-1, keepdim=True)
    z = torch.sort(torch.rand(nr, n) * 4 + 1, dim=-1)[0]
    sdf = torch.randn(nr, n) * 0.3
    u = torch.rand(nr, 16)
    occ = OccupancyGrid(32).to(DEV)
    mask = torch.rand(32, 32, 32) < 0.5
    with torch.no_grad():
        occ.occupancy_mask.copy_(to(mask))
    lo, hi = torch.tensor((-1.0,) * 3), torch.tensor((1.0,) * 3)
    ref = O.up_sample(o, d, z, sdf, 16, 128.0, det=False, u=u, occ_fn=lambda p: O.is_occupied(mask, p, lo, hi))
    out = up_sample(to(o), to(d), to(z), to(sdf), 16, 128.0, det=False, occupancy_grid=occ, u=to(u))
    assert_close(out, ref, VAL_TOL, "up_sample with occupancy")


# ------------------------------------------------------------------ render forward / backward


@pytest.mark.parametrize("name,perturb,ns", [("render_det.npz", False, 16), ("render_perturb.npz", True, 16),
                                             ("render_128.npz", True, 64)])
def test_render_matches_golden(golden, name, perturb, ns):
    """The whole render and its gradients against the reference's; render_128 is the throughput
    workload's sampler (64 stratified + 4 x 16 upsampled samples per ray)."""
    from voxneus_b200.rendering import RaySampler, compute_huber_color_loss

    g = golden(name)
    m = _scene_from(g)
    s = RaySampler(ns, ns, perturb=perturb)
    randoms = (to(g["t_rand"]), to(g["us"])) if perturb else None
    z_vals = None
    if ns > 16:
        # 128 samples: the sampler alone first. A ray whose reference samples sit within a few ulps
        # of a discontinuity (occupancy cell, unit sphere, flat CDF stretch) may move by up to an
        # interval: at most one ray outside 1e-5, every ray within 1e-2. The render and its
        # gradients are then compared on the reference's own samples.
        z, _, _ = s.sample_multistep_sdf(to(g["rays_o"]), to(g["rays_d"]), to(g["near"]), to(g["far"]),
                                         m.sdf_grid.sdf_fn(), up_sample_steps=4, occupancy_grid=m.occupancy_grid,
                                         randoms=randoms)
        zr = g["z"].double()
        err = (z.cpu().double() - zr).abs()
        bad = (err > VAL_TOL * (zr.abs() + float(zr.abs().max()))).any(dim=1)
        assert int(bad.sum()) <= 1 and float(err.max()) < 1e-2, (int(bad.sum()), float(err.max()))
        z_vals = to(g["z"])
    out = m.render(to(g["rays_o"]), to(g["rays_d"]), s, to(g["near"]), to(g["far"]), randoms=randoms, z_vals=z_vals)
    # depth = sum w t: its FP32 error is that of the weights (absolute, alpha cancels) times the
    # sample depth, so its scale is the largest sample depth
    zmax = float(g["z"].abs().max())
    for k in ("rgb", "depth", "normal", "opacity", "weights", "alpha", "transmittance", "pts", "sdf_samples",
              "normal_samples", "grad_samples"):
        assert_close(out[k], g[k], VAL_TOL, k, scale=zmax if k == "depth" else None)
    loss = compute_huber_color_loss(out["rgb"], to(g["target"]), 0.1)
    assert_close(loss, g["loss"], VAL_TOL, "loss")
    loss.backward()
    grads = {"grid": m.sdf_grid.grid.grad, "variance": m.variance_net.variance.grad,
             "embeddings": m.radiance_hash.encoder.embeddings.grad, "w0": m.radiance_mlp.net[0].weight.grad,
             "b0": m.radiance_mlp.net[0].bias.grad, "w1": m.radiance_mlp.net[2].weight.grad,
             "b1": m.radiance_mlp.net[2].bias.grad}
    for k, v in grads.items():
        assert_close(v, g[k + "_grad"], GRAD_TOL, k + " grad")
    from voxneus_b200.regularization import extract_active_vertices

    verts, lin = extract_active_vertices(out["corner_indices"], list(g["grid"].shape[-3:]))
    assert torch.equal(verts.cpu(), g["vr_verts"]) and torch.equal(lin.cpu(), g["vr_linear"])


def test_vr_bitmap_from_render_equals_unique(golden):
    from voxneus_b200 import ops
    from voxneus_b200.rendering import RaySampler

    g = golden("render_det.npz")
    m = _scene_from(g)
    bm = ops.new_bitmap([24] * 3, DEV)
    out = m.render(to(g["rays_o"]), to(g["rays_d"]), RaySampler(16, 16, perturb=False), to(g["near"]), to(g["far"]),
                   vr_bitmap=bm)
    counts = ops.vr_count(bm, None, [24] * 3, (0, 0, 0), (1, 1, 1))
    verts, lin = ops.vr_compact(bm, None, [24] * 3, (0, 0, 0), (1, 1, 1), 0.0, 0.0, counts, int(counts[0]))
    assert torch.equal(verts.cpu(), g["vr_verts"]) and torch.equal(lin.cpu(), g["vr_linear"])


def test_volume_render_api_and_alpha():
    from voxneus_b200.rendering import compute_neus_alpha, composite_weights, volume_render_from_samples

    torch.manual_seed(8)
    nr, ns = 37, 70
    col = torch.rand(nr, ns, 3)
    sdf = torch.randn(nr, ns, 1) * 0.05
    nrm = torch.nn.functional.normalize(torch.randn(nr, ns, 3), dim=-1)
    dirs = torch.nn.functional.normalize(torch.randn(nr, 3), dim=-1)
    z = torch.sort(torch.rand(nr, ns) * 2 + 1, dim=-1)[0]
    dists = torch.rand(nr, ns) * 0.05
    pts = torch.randn(nr, ns, 3) * 0.7
    s = torch.tensor(40.0)
    bg = torch.rand(3)
    leaves = [t.clone().requires_grad_(True) for t in (col, sdf, nrm, s)]
    ref = O.volume_render(leaves[0], leaves[1], leaves[2], dirs.unsqueeze(1).expand(-1, ns, -1), z, dists, leaves[3],
                          pts=pts, radius=1.0, background=bg)
    gl = [t.clone().requires_grad_(True) for t in (to(col), to(sdf), to(nrm), to(s))]
    out = volume_render_from_samples(gl[0], gl[1], gl[2], to(dirs), to(z), to(dists), gl[3], pts=to(pts),
                                     background_rgb=to(bg))
    for k in ("rgb", "depth", "normal", "opacity", "weights", "alpha", "transmittance"):
        assert_close(out[k], ref[k].detach(), VAL_TOL, k)
    cot = {k: torch.randn_like(ref[k]) for k in ("rgb", "depth", "normal", "opacity", "weights")}
    sum(((ref[k] * cot[k]).sum() for k in cot)).backward()
    sum(((out[k] * to(cot[k])).sum() for k in cot)).backward()
    for a, b, nm in zip(gl, leaves, ("colors", "sdf", "normals", "s")):
        assert_close(a.grad, b.grad, GRAD_TOL, nm + " grad")
    # standalone alpha and composite_weights
    a_ref = O.neus_alpha(sdf, nrm, dirs.unsqueeze(1).expand(-1, ns, -1), dists, s)
    assert_close(compute_neus_alpha(to(sdf), to(nrm), to(dirs).unsqueeze(1), to(dists), to(s)), a_ref, VAL_TOL, "alpha")
    acut = torch.zeros(2, 10)
    acut[0, :2] = 0.999
    acut[1] = torch.rand(10)
    w, t = composite_weights(to(acut))
    wr, tr = O.composite_weights(acut)
    assert w[0, 3].item() == 0.0 and t[0, 3].item() < 1e-4
    assert_close(w, wr, VAL_TOL, "w")
    assert_close(t, tr, VAL_TOL, "T")


@pytest.mark.parametrize("ratio", [0.0, 0.35, 1.0])
def test_iter_cos_annealing(ratio):
    """NeuS's iter_cos annealing (rendering/neus_alpha.py:46-53: cos = -(relu(-cos/2 + 1/2)(1 - r) +
    relu(-cos) r)) through compute_neus_alpha and volume_render_from_samples against the oracle:
    values, and the gradients of colours, SDF, normals and s."""
    from voxneus_b200.rendering import compute_neus_alpha, volume_render_from_samples

    torch.manual_seed(9)
    nr, ns = 29, 48
    col = torch.rand(nr, ns, 3)
    sdf = torch.randn(nr, ns, 1) * 0.05
    nrm = torch.nn.functional.normalize(torch.randn(nr, ns, 3), dim=-1)
    dirs = torch.nn.functional.normalize(torch.randn(nr, 3), dim=-1)
    z = torch.sort(torch.rand(nr, ns) * 2 + 1, dim=-1)[0]
    dists = torch.rand(nr, ns) * 0.05
    s = torch.tensor(30.0)
    leaves = [t.clone().requires_grad_(True) for t in (col, sdf, nrm, s)]
    ref = O.volume_render(leaves[0], leaves[1], leaves[2], dirs.unsqueeze(1).expand(-1, ns, -1), z, dists, leaves[3],
                          cos_anneal_ratio=ratio, use_iter_cos=True)
    gl = [t.clone().requires_grad_(True) for t in (to(col), to(sdf), to(nrm), to(s))]
    out = volume_render_from_samples(gl[0], gl[1], gl[2], to(dirs), to(z), to(dists), gl[3],
                                     cos_anneal_ratio=ratio, use_iter_cos_annealing=True)
    for k in ("rgb", "depth", "normal", "opacity", "weights", "alpha"):
        assert_close(out[k], ref[k].detach(), VAL_TOL, k)
    cot = {k: torch.randn_like(ref[k]) for k in ("rgb", "depth", "normal", "opacity")}
    sum(((ref[k] * cot[k]).sum() for k in cot)).backward()
    sum(((out[k] * to(cot[k])).sum() for k in cot)).backward()
    for a, b, nm in zip(gl, leaves, ("colors", "sdf", "normals", "s")):
        assert_close(a.grad, b.grad, GRAD_TOL, nm + " grad")
    # the standalone alpha and its adjoint
    al = [t.clone().requires_grad_(True) for t in (sdf, nrm, s)]
    a_ref = O.neus_alpha(al[0], al[1], dirs.unsqueeze(1).expand(-1, ns, -1), dists, al[2], ratio, True)
    ag = [t.clone().requires_grad_(True) for t in (to(sdf), to(nrm), to(s))]
    a_out = compute_neus_alpha(ag[0], ag[1], to(dirs).unsqueeze(1), to(dists), ag[2], cos_anneal_ratio=ratio,
                               use_iter_cos_annealing=True)
    assert_close(a_out, a_ref.detach(), VAL_TOL, "alpha")
    ca = torch.randn_like(a_ref)
    (a_ref * ca).sum().backward()
    (a_out * to(ca)).sum().backward()
    for a, b, nm in zip(ag, al, ("sdf", "normals", "s")):
        assert_close(a.grad, b.grad, GRAD_TOL, "alpha " + nm + " grad")


# ------------------------------------------------------------------ regularizers, V_R, upsample, hash


def test_regularizers_list_golden(golden):
    from voxneus_b200.regularization import compute_curvature_loss_and_gradient, compute_eikonal_loss_and_gradient

    g = golden("regularizers.npz")
    res = torch.tensor([16.0, 14.0, 12.0])
    le, ge = compute_eikonal_loss_and_gradient(to(g["grid"]), to(g["verts"]), g["voxel_size"], res)
    lc, gc = compute_curvature_loss_and_gradient(to(g["grid"]), to(g["verts"]), g["voxel_size"], res)
    assert_close(ge, g["grad_eik"], GRAD_TOL, "eik grad")
    assert_close(gc, g["grad_curv"], GRAD_TOL, "curv grad")
    assert abs(le.item() - g["loss_eik"].item()) <= 1e-5 * abs(g["loss_eik"].item())
    assert abs(lc.item() - g["loss_curv"].item()) <= 1e-5 * abs(g["loss_curv"].item())
    # in-place accumulation equals the separate gradient (tests/test_cuda_parity.py:72-126)
    acc = torch.zeros(1, 1, 16, 14, 12, device=DEV)
    compute_eikonal_loss_and_gradient(to(g["grid"]), to(g["verts"]), g["voxel_size"], res, accumulate_grad=acc)
    assert_close(acc, ge, 1e-5, "in-place eik")
    from voxneus_b200.regularization import extract_active_vertices

    v, lin = extract_active_vertices(to(g["corners"]), (16, 14, 12))
    assert torch.equal(v.cpu(), g["vr_verts"]) and torch.equal(lin.cpu(), g["vr_linear"])


@pytest.mark.parametrize("band", [None, 3.0])
@pytest.mark.parametrize("res", [[40, 36, 44], [40, 36, 64]])
def test_fused_stencil_matches_oracle(band, res):
    """Gather-form eikonal + curvature over a V_R bitmap == oracle list form after relax/band filters
    (Z = 64: whole-row bitmap words, the vectorised count path; Z = 44: words spanning rows)."""
    from voxneus_b200 import ops

    torch.manual_seed(12)
    lo, hi = (-1.0, -1.0, -1.0), (1.0, 1.0, 1.0)
    axes = [torch.linspace(-1, 1, r) for r in res]
    gx, gy, gz = torch.meshgrid(*axes, indexing="ij")
    grid = (torch.sqrt(gx ** 2 + gy ** 2 + gz ** 2) - 0.6 + 0.01 * torch.randn(*res)).reshape(1, 1, *res)
    corners = torch.stack([torch.randint(0, r, (6000,)) for r in res], -1)
    verts, _ = O.extract_active_vertices(corners, res)
    eps = O.voxel_size(torch.tensor(lo), torch.tensor(hi), torch.tensor(res, dtype=torch.float32))
    v = O.relax_filter(verts, torch.tensor(lo), eps)
    bnd = 0.0
    if band:
        bnd = float(torch.tensor(band * float(eps[0]), dtype=torch.float32))
        v = O.band_filter(v, grid.reshape(res), float(eps[0]), band)
    le, ge = O.eikonal(grid.reshape(res), v, eps, res, weight=0.1)
    lc, gc = O.curvature(grid.reshape(res), v, eps, res, weight=5e-4)
    bm = ops.new_bitmap(res, DEV)
    ops.vr_mark_corners(to(corners), res, bm)
    gd = to(grid)
    fb = ops.new_filtered(res, DEV)
    counts = ops.vr_count(bm, gd, res, lo, hi, 1.2, bnd, filtered=fb)
    assert int(ops.final_count(counts, 1.2, bnd)) == v.shape[0]
    out = torch.zeros(res, device=DEV)
    n_active = torch.zeros((), dtype=torch.int64, device=DEV)
    losses = ops.reg_stencil(gd, fb, res, lo, hi, 1.2, bnd, counts, 0.1, 5e-4, out, n_active=n_active)
    assert int(n_active) == int(ops.final_count(counts, 1.2, bnd)) == v.shape[0]
    assert_close(out, ge + gc, GRAD_TOL, "fused stencil grad")
    assert abs(losses[0].item() - le.item()) <= 1e-5 * max(le.item(), 1e-12)
    assert abs(losses[1].item() - lc.item()) <= 1e-5 * max(lc.item(), 1e-12)
    vl, ll = ops.vr_compact(bm, gd, res, lo, hi, 1.2, bnd, counts, v.shape[0])
    assert torch.equal(vl.cpu(), v)


def _bitmap_voxels(words: torch.Tensor, nvox: int) -> torch.Tensor:
    w = words.cpu().numpy().view(np.uint32)
    bits = np.unpackbits(w.view(np.uint8), bitorder="little")[:nvox]
    return torch.from_numpy(np.nonzero(bits)[0].astype(np.int64))


@pytest.mark.parametrize("res", [[24, 20, 96], [24, 20, 90]])
def test_vr_count_and_filtered_bitmaps(res):
    """|V_R| under each filter and the two filtered bitmaps, bit for bit against the oracle's
    relax and band filters, on a dense random bitmap (whole-row words and row-spanning words)."""
    from voxneus_b200 import ops

    torch.manual_seed(13)
    lo, hi = (-1.0, -1.0, -1.0), (1.0, 1.0, 1.0)
    axes = [torch.linspace(-1, 1, r) for r in res]
    gx, gy, gz = torch.meshgrid(*axes, indexing="ij")
    grid = (torch.sqrt(gx ** 2 + gy ** 2 + gz ** 2) - 0.7 + 0.02 * torch.randn(*res)).contiguous()
    nvox = res[0] * res[1] * res[2]
    lin = torch.unique(torch.randint(0, nvox, (nvox // 3,)))
    verts = torch.stack([lin // (res[1] * res[2]), (lin // res[2]) % res[1], lin % res[2]], -1)
    eps = O.voxel_size(torch.tensor(lo), torch.tensor(hi), torch.tensor(res, dtype=torch.float32))
    bnd = float(torch.tensor(3.0 * float(eps[0]), dtype=torch.float32))

    def lin_of(v):
        return (v[:, 0] * res[1] + v[:, 1]) * res[2] + v[:, 2]

    relax = lin_of(O.relax_filter(verts, torch.tensor(lo), eps))
    band = lin_of(O.band_filter(verts, grid, float(eps[0]), 3.0))
    both = lin_of(O.band_filter(O.relax_filter(verts, torch.tensor(lo), eps), grid, float(eps[0]), 3.0))
    bm = ops.new_bitmap(res, DEV)
    ops.vr_mark_corners(to(verts), res, bm)
    fb = ops.new_filtered(res, DEV)
    counts = ops.vr_count(bm, to(grid), res, lo, hi, 1.2, bnd, filtered=fb)
    assert counts.cpu().tolist() == [lin.numel(), relax.numel(), band.numel(), both.numel()]
    nw = ops.bitmap_words(res)
    assert torch.equal(_bitmap_voxels(fb[:nw], nvox), band)
    assert torch.equal(_bitmap_voxels(fb[nw:], nvox), both)


def test_upsample_golden(golden):
    from voxneus_b200.geometry import upsample_sdf_grid

    g = golden("upsample.npz")
    assert_close(upsample_sdf_grid(to(g["grid"]), [17, 13, 11]), g["out_a"], VAL_TOL, "upsample a")
    assert_close(upsample_sdf_grid(to(g["grid"]), 12), g["out_b"], VAL_TOL, "upsample b")
    src = torch.randn(1, 1, 33, 32, 31)
    assert_close(upsample_sdf_grid(to(src), [64, 64, 64]), O.upsample_grid(src, 64), VAL_TOL, "upsample 64")


def test_hash_and_sh_golden(golden):
    from voxneus_b200.models import RadianceHashGrid, SphericalHarmonicsEmbedder

    g = golden("hash.npz")
    enc = RadianceHashGrid(16, 2, 8).to(DEV)
    with torch.no_grad():
        enc.encoder.embeddings.copy_(to(g["embeddings"]))
    assert_close(enc(to(g["x"])), g["feats"], VAL_TOL, "hash")
    assert_close(enc(to(g["x"]), active_levels=5.5), g["feats_l55"], VAL_TOL, "hash lambda")
    assert_close(SphericalHarmonicsEmbedder(4)(to(g["dirs"])), g["sh"], VAL_TOL, "sh")
    # SH products rounded one by one in the reference's order: the reference's own bits
    assert torch.equal(SphericalHarmonicsEmbedder(4)(to(g["dirs"])).cpu(), torch.as_tensor(g["sh"]))
    # adjoint vs autograd of the oracle
    emb = g["embeddings"].clone().requires_grad_(True)
    cot = torch.randn(200, 32)
    (O.hash_encode(g["x"], emb, O.hash_level_resolutions(16), 5.5) * cot).sum().backward()
    enc.encoder.embeddings.grad = None
    (enc(to(g["x"]), active_levels=5.5) * to(cot)).sum().backward()
    assert_close(enc.encoder.embeddings.grad, emb.grad, GRAD_TOL, "hash grad")


@pytest.mark.parametrize("ld", [52, 56])
@pytest.mark.parametrize("p", [3000, 50000])
def test_fused_mlp_matches_oracle(p, ld):
    """51-64-3 MLP forward (1e-5) and adjoint (input and weight gradients, 1e-4) vs torch fp32 autograd.

    3000 rows: one partial tile per block; 50000 rows: blocks accumulate several tiles of the
    weight gradient in tensor memory. Neither is a multiple of the 128-sample tile. Row stride 52
    (contiguous rows: the adjoint brings each tile's rows in with one bulk copy) and 56 (strided
    rows: prefetched through registers).

    Rows with a hidden pre-activation within 1e-6 of the largest |z| of zero (FP64) sit on a ReLU
    kink, where any two FP32 evaluation orders can disagree on the unit's sign (and move that
    sample's input gradient and its share of dW0 by ~|dz x|); they are dropped from the inputs
    (a handful: at most one in 2000) so every output is compared in full."""
    from voxneus_b200 import _lib, ops

    torch.manual_seed(13)
    rows = torch.randn(p, 52)
    l0, l1 = torch.nn.Linear(51, 64), torch.nn.Linear(64, 3)
    with torch.no_grad():
        z64 = rows[:, :51].double() @ l0.weight.double().T + l0.bias.double()
        smooth = (z64.abs() > 1e-6 * float(z64.abs().max())).all(dim=1)
    assert int((~smooth).sum()) <= max(2, p // 2000), int((~smooth).sum())
    rows = rows[smooth].contiguous()
    p = rows.shape[0]
    x = rows[:, :51].clone().requires_grad_(True)
    ws = [t.detach().clone().requires_grad_(True) for t in (l0.weight, l0.bias, l1.weight, l1.bias)]
    ref = O.radiance_mlp(x[:, :32], x[:, 32:48], x[:, 48:51], *ws)
    cot = torch.randn(p, 3)
    (ref * cot).sum().backward()
    wide = torch.zeros(p, ld)
    wide[:, :52] = rows
    rd = to(wide)
    wd = [to(t.detach()).requires_grad_(True) for t in ws]
    xd = rd[:, :51].requires_grad_(True)
    out = ops.RadianceMLPFn.apply(xd, *wd)
    assert_close(out, ref.detach(), VAL_TOL, "rgb")
    (out * to(cot)).sum().backward()
    assert_close(xd.grad[:, :32], x.grad[:, :32], GRAD_TOL, "d hash")
    assert_close(xd.grad[:, 48:51], x.grad[:, 48:51], GRAD_TOL, "d normal")
    for a, b, nm in zip(wd, ws, ("W0", "b0", "W1", "b1")):
        assert_close(a.grad, b.grad, GRAD_TOL, nm)
    assert _lib.query("vx_tensor_core_timeouts") == 0


@pytest.mark.parametrize("ld", [52, 56])
def test_mlp_adjoint_with_forward_colours_is_bitwise_the_recompute(ld):
    """The adjoint reading the forward's colours (for the sigmoid's derivative) instead of
    recomputing the output layer gives the same bits: same MMAs, same partial sums (52-float rows
    take the bulk-copy kernels, other strides the register-prefetch ones)."""
    from voxneus_b200 import ops

    torch.manual_seed(5)
    p = 3001  # a partial last tile
    rows = torch.randn(p, ld, device=DEV)[:, :51]  # 51 features in ld-float rows
    W0 = 0.2 * torch.randn(64, 51, device=DEV)
    b0 = 0.1 * torch.randn(64, device=DEV)
    W1 = 0.2 * torch.randn(3, 64, device=DEV)
    b1 = 0.1 * torch.randn(3, device=DEV)
    colors = ops.mlp_forward(rows, W0, b0, W1, b1)
    g = torch.randn(p, 3, device=DEV)
    a = ops.mlp_backward(rows, W0, b0, W1, b1, g)
    b = ops.mlp_backward(rows, W0, b0, W1, b1, g, colors)
    torch.cuda.synchronize()
    for x, y in zip(a, b):
        assert torch.equal(x, y)


def test_huber_loss_and_gradient():
    """Fused Huber colour loss (value 1e-5, gradient 1e-4) vs the oracle's torch ops; both branches,
    exact ties and a size that is not a multiple of the block."""
    from voxneus_b200.rendering import compute_huber_color_loss

    torch.manual_seed(21)
    pred = torch.rand(10007, 3)
    tgt = pred + (torch.rand(10007, 3) - 0.5) * 0.5  # |d| spans both sides of delta = 0.1
    tgt[:5] = pred[:5]  # d = 0
    pr = pred.clone().requires_grad_(True)
    ref = O.huber(pr, tgt, 0.1)
    ref.backward()
    pd = to(pred).requires_grad_(True)
    loss = compute_huber_color_loss(pd, to(tgt), 0.1)
    assert_close(loss, ref.detach(), VAL_TOL, "huber loss")
    (loss * 3.0).backward()
    assert_close(pd.grad, 3.0 * pr.grad, GRAD_TOL, "huber grad")


@pytest.mark.parametrize("ld", [52, 56])
def test_appearance_rows_match_oracle(ld):
    """The MLP input rows the training forward writes ([hash 32 | SH 16 | normal 3 | 0]) against the
    oracle's hash encoding, SH and normals: 397 rays x 127 samples (many 64-sample blocks and a
    partial last one), a progressive level mask of 9.5 levels (one level weighted 0.5, six skipped),
    contiguous rows (52) and a wider stride (56)."""
    from voxneus_b200 import _lib, ops

    torch.manual_seed(21)
    cfg = ops.HashConfig(16, 2, 14)
    nr, ns = 397, 127
    emb = torch.rand(16, 2 ** 14, 2) * 0.2 - 0.1
    o = torch.randn(nr, 3)
    o = 2.5 * o / o.norm(dim=-1, keepdim=True)
    d = -o / o.norm(dim=-1, keepdim=True) + 0.1 * torch.randn(nr, 3)
    d = d / d.norm(dim=-1, keepdim=True)
    mid = torch.sort(torch.rand(nr, ns) * 3.0 + 0.5, dim=-1).values
    nrm = torch.randn(nr * ns, 3)
    ws = [torch.randn(64, 51) * 0.1, torch.zeros(64), torch.randn(3, 64) * 0.1, torch.zeros(3)]
    lo, hi = (-1.0, -1.0, -1.0), (1.0, 1.0, 1.0)
    ed, od, dd, md, nd = (to(t.contiguous()) for t in (emb, o, d, mid, nrm))
    wd = [to(t) for t in ws]
    rows = torch.full((nr * ns, ld), float("nan"), device=DEV)
    colors = torch.empty(nr * ns, 3, device=DEV)
    P = _lib.ptr
    _lib.call("vx_appearance_mlp_forward", P(ed), 16, 14, 2, cfg._res_c, cfg.level_weights(9.5), P(od), P(dd), P(md),
              ns, _lib.f3(lo), _lib.f3(hi), nr * ns, P(nd), *[P(t) for t in wd], P(colors), P(rows), ld,
              _lib.stream_ptr(torch.device(DEV)))
    torch.cuda.synchronize()
    pts = o.unsqueeze(1) + d.unsqueeze(1) * mid.unsqueeze(-1)
    nx = (pts - torch.tensor(lo)) / (torch.tensor(hi) - torch.tensor(lo) + 1e-8)
    hf = O.hash_encode(nx.reshape(-1, 3), emb, cfg.resolutions, 9.5)
    sh = O.sh4(d.unsqueeze(1).expand(nr, ns, 3).reshape(-1, 3))
    got = rows.cpu()
    assert_close(got[:, :32], hf, VAL_TOL, "hash features")
    assert torch.equal(got[:, 32:48], sh)  # each product rounded in the reference's order: its bits
    assert torch.equal(got[:, 48:51], nrm) and bool((got[:, 51] == 0).all())
    assert bool((got[:, 2 * 10:32] == 0).all())  # levels 10..15 are skipped


def test_chunked_inference_appearance_matches_rows_path():
    """The inference form (rows through a small scratch, whole rays per chunk) gives the same colour
    bits as the training form that keeps all rows: a 5-ray scratch (many chunks, a partial last one)
    and a single-chunk scratch; the in-shared-memory fused kernel agrees within 1e-5; a scratch
    smaller than one ray is refused."""
    from voxneus_b200 import _lib, ops

    torch.manual_seed(22)
    cfg = ops.HashConfig(16, 2, 14)
    nr, ns = 397, 127
    emb = torch.rand(16, 2 ** 14, 2) * 0.2 - 0.1
    o = torch.randn(nr, 3)
    o = 2.5 * o / o.norm(dim=-1, keepdim=True)
    d = -o / o.norm(dim=-1, keepdim=True) + 0.1 * torch.randn(nr, 3)
    d = d / d.norm(dim=-1, keepdim=True)
    mid = torch.sort(torch.rand(nr, ns) * 3.0 + 0.5, dim=-1).values
    ed, od, dd, md, nd = (to(t.contiguous()) for t in (emb, o, d, mid, torch.randn(nr * ns, 3)))
    wd = [to(t) for t in (torch.randn(64, 51) * 0.3, torch.randn(64) * 0.1, torch.randn(3, 64) * 0.3,
                          torch.randn(3) * 0.1)]
    P = _lib.ptr
    lo, hi = _lib.f3((-1.0, -1.0, -1.0)), _lib.f3((1.0, 1.0, 1.0))
    head = (P(ed), 16, 14, 2, cfg._res_c, cfg.level_weights(None), P(od), P(dd), P(md), ns, lo, hi, nr * ns, P(nd),
            *[P(t) for t in wd])
    st = _lib.stream_ptr(torch.device(DEV))
    rows = torch.empty(nr * ns, 52, device=DEV)
    ref = torch.empty(nr * ns, 3, device=DEV)
    _lib.call("vx_appearance_mlp_forward", *head, P(ref), P(rows), 52, st)
    for n_rows in (5 * ns, 262144):
        scratch = torch.empty(n_rows, 36, device=DEV)
        got = torch.full((nr * ns, 3), float("nan"), device=DEV)
        _lib.call("vx_appearance_mlp_forward_chunked", *head, P(got), P(scratch), n_rows, st)
        torch.cuda.synchronize()
        assert torch.equal(got, ref), n_rows
    fused = torch.empty(nr * ns, 3, device=DEV)
    _lib.call("vx_appearance_mlp_forward", *head, P(fused), None, 0, st)
    torch.cuda.synchronize()
    assert_close(fused, ref, VAL_TOL, "rgb", scale=1.0)
    small = torch.empty(ns - 1, 36, device=DEV)
    with pytest.raises(RuntimeError, match="fewer than one ray"):
        _lib.call("vx_appearance_mlp_forward_chunked", *head, P(fused), P(small), ns - 1, st)


@pytest.mark.parametrize("nr,ns", [(397, 127), (3, 1), (64, 128), (5, 256)])
def test_compact_rows_match_full_rows(nr, ns):
    """The compact rows [hash 32 | normal 3 | pad] of the training path against the full 52-float
    rows [hash | SH | normal | pad]: the stored hash and normal columns are the same bits. Where the
    samples of a ray do not fill whole 128-row tiles (127, 1), the MLP kernels rebuild SH(d) in the
    staging and the colours and every adjoint output are the same bits; where they do (128, 256),
    the folded MLP adds SH(d) as a per-ray bias of the hidden layer and takes the SH columns of dW0
    from per-tile column sums, so the results agree within FP32 rounding: colours to 1e-6, weight
    gradients to 1e-5 of their scale, the per-sample cotangents to 1e-5 of scale on samples whose
    hidden pre-activations are all clear of zero (a ReLU at |z| < 1e-5 may switch)."""
    from voxneus_b200 import _lib, ops

    torch.manual_seed(23 + nr)
    cfg = ops.HashConfig(16, 2, 14)
    emb = torch.rand(16, 2 ** 14, 2) * 0.2 - 0.1
    o = torch.randn(nr, 3)
    o = 2.5 * o / o.norm(dim=-1, keepdim=True)
    d = -o / o.norm(dim=-1, keepdim=True) + 0.1 * torch.randn(nr, 3)
    d = d / d.norm(dim=-1, keepdim=True)
    mid = torch.sort(torch.rand(nr, ns) * 3.0 + 0.5, dim=-1).values
    p = nr * ns
    ed, od, dd, md, nd = (to(t.contiguous()) for t in (emb, o, d, mid, torch.randn(p, 3)))
    wd = [to(t) for t in (torch.randn(64, 51) * 0.3, torch.randn(64) * 0.1, torch.randn(3, 64) * 0.3,
                          torch.randn(3) * 0.1)]
    P = _lib.ptr
    lo, hi = _lib.f3((-1.0, -1.0, -1.0)), _lib.f3((1.0, 1.0, 1.0))
    head = (P(ed), 16, 14, 2, cfg._res_c, cfg.level_weights(None), P(od), P(dd), P(md), ns, lo, hi, p, P(nd),
            *[P(t) for t in wd])
    st = _lib.stream_ptr(torch.device(DEV))
    full, compact = torch.empty(p, 52, device=DEV), torch.empty(p, 36, device=DEV)
    c_full, c_compact = torch.empty(p, 3, device=DEV), torch.empty(p, 3, device=DEV)
    _lib.call("vx_appearance_mlp_forward", *head, P(c_full), P(full), 52, st)
    _lib.call("vx_appearance_mlp_forward", *head, P(c_compact), P(compact), 36, st)
    torch.cuda.synchronize()
    assert torch.equal(compact[:, :32], full[:, :32]) and torch.equal(compact[:, 32:35], full[:, 48:51])
    folded = ns % 128 == 0
    if folded:
        assert float((c_compact - c_full).abs().max()) <= 1e-6
    else:
        assert torch.equal(c_compact, c_full)
    g = to(torch.randn(p, 3) * 0.1)
    z = full[:, :51].double() @ wd[0].double().t() + wd[1].double()
    clear = (z.abs().min(dim=1).values > 1e-5).cpu()
    assert float(clear.double().mean()) > 0.99
    for colors in (None, c_full):
        a = ops.mlp_backward(full[:, :51], *wd, g, colors)
        b = ops.mlp_backward(compact, *wd, g, colors, dd, ns)
        for name, x, y in zip(("d_hash", "d_normal", "dW0", "db0", "dW1", "db1"), a, b):
            if not folded:
                assert torch.equal(x, y), name
                continue
            x, y = x.cpu(), y.cpu()
            if name in ("d_hash", "d_normal"):
                x, y = x[clear], y[clear]
            scale = max(float(x.abs().max()), 1e-30)
            assert float((x - y).abs().max()) <= 1e-5 * scale, (name, float((x - y).abs().max()), scale)
    with pytest.raises(RuntimeError, match="compact MLP rows"):
        ops.mlp_backward(full[:, :36], *wd, g, None, dd, ns)


def test_deterministic_mode_is_bitwise_reproducible(golden):
    """Sorted segmented-reduction adjoints: identical bits on repeated runs, 1e-4 of the atomic mode."""
    from voxneus_b200 import ops
    from voxneus_b200.rendering import RaySampler, compute_huber_color_loss

    g = golden("render_perturb.npz")

    def grads(det):
        ops.set_deterministic(det)
        try:
            m = _scene_from(g)
            out = m.render(to(g["rays_o"]), to(g["rays_d"]), RaySampler(16, 16, perturb=True), to(g["near"]),
                           to(g["far"]), randoms=(to(g["t_rand"]), to(g["us"])))
            compute_huber_color_loss(out["rgb"], to(g["target"]), 0.1).backward()
            return m.sdf_grid.grid.grad.clone(), m.radiance_hash.encoder.embeddings.grad.clone()
        finally:
            ops.set_deterministic(False)

    a, b, c = grads(True), grads(True), grads(False)
    assert torch.equal(a[0], b[0]) and torch.equal(a[1], b[1])
    assert_close(a[0], c[0], GRAD_TOL, "grid grad det vs atomic")
    assert_close(a[1], c[1], GRAD_TOL, "table grad det vs atomic")
    assert_close(a[0], g["grid_grad"], GRAD_TOL, "grid grad det vs golden")


def test_masked_adam_leaves_zero_grad_untouched():
    """tests/test_cuda_parity.py:128-146."""
    from voxneus_b200.training import SparseGridAdam

    p = torch.ones(1000, device=DEV, requires_grad=True)
    p.grad = torch.zeros_like(p)
    p.grad[10:20] = 0.5
    p.grad[50:60] = -0.5
    SparseGridAdam([p], lr=0.05).step()
    assert p[0].item() == 1.0 and p[30].item() == 1.0 and p[999].item() == 1.0
    assert p[10].item() < 1.0 and p[50].item() > 1.0


def _occ_compare(dens_gpu, mask_gpu, dens_ref, mask_ref, threshold=0.01):
    """Density within VAL_TOL; the mask bit-exact except where the oracle's value sits within
    VAL_TOL of the threshold (a comparison that one ulp of SDF can flip)."""
    assert_close(dens_gpu, dens_ref, VAL_TOL, "occupancy density")
    m_gpu = mask_gpu.cpu()
    border = (dens_ref.double() - threshold).abs() <= VAL_TOL * (abs(threshold) + float(dens_ref.abs().max()))
    assert bool(((m_gpu == mask_ref) | border).all()), int((m_gpu != mask_ref).sum())


def test_occupancy_update_golden(golden):
    """The reference's three EMA updates (its own cell draws) replayed through the kernel."""
    from voxneus_b200 import ops

    g = golden("occupancy.npz")
    lo, hi = (-1.0, -1.0, -1.0), (1.0, 1.0, 1.0)
    grid = to(g["grid"])
    density = torch.zeros(32, 32, 32, device=DEV)
    mask = torch.ones(32, 32, 32, dtype=torch.bool, device=DEV)
    for k in range(3):
        idx = [to(g[f"idx{k}"][a].contiguous()) for a in range(3)]
        s = torch.tensor(float(g[f"s{k}"]), device=DEV)
        ops.occupancy_update(density, mask, idx, lo, hi, s, False, 0.0, k == 0, 0.95, 0.01, grid=grid,
                             grid_bounds=(lo, hi))
        torch.cuda.synchronize()
        _occ_compare(density, mask, g[f"density{k}"], g[f"mask{k}"])


def test_occupancy_update_full_size_matches_oracle():
    """128^3 occupancy grid, a quarter of the cells per update (524,288 draws with repeats), 96^3
    SDF grid, s from the variance parameter, three updates against the oracle on the same draws."""
    from voxneus_b200.models import VoxNeuS

    torch.manual_seed(3)
    m = VoxNeuS(grid_res=96, hash_log2_size=12).to(DEV)
    with torch.no_grad():
        m.sdf_grid.grid.add_(0.02 * torch.randn_like(m.sdf_grid.grid))
    lo, hi = (-1.0, -1.0, -1.0), (1.0, 1.0, 1.0)
    glo, ghi = torch.tensor(lo), torch.tensor(hi)
    grid_cpu = m.sdf_grid.grid.detach().cpu()
    dens = torch.zeros(128, 128, 128)
    mask = torch.ones(128, 128, 128, dtype=torch.bool)
    gen = torch.Generator(device=DEV)
    for k, v in enumerate([0.3, 0.45, 0.6]):
        with torch.no_grad():
            m.variance_net.variance.fill_(v)
        gen.manual_seed(40 + k)
        m.update_occupancy_grid(0.25, generator=gen)
        gen.manual_seed(40 + k)
        idx = torch.stack([torch.randint(0, 128, (128 ** 3 // 4,), device=DEV, generator=gen) for _ in range(3)]).cpu()
        s = O.variance_s(torch.tensor(v))
        O.occupancy_update(dens, mask, idx, lambda p: O.query_sdf(grid_cpu, p, glo, ghi), s, k == 0, lo, hi)
        torch.cuda.synchronize()
        _occ_compare(m.occupancy_grid.density_grid, m.occupancy_grid.occupancy_mask, dens, mask)
    assert m.occupancy_grid.total_updates == 3
    assert 0.0 < m.occupancy_grid.occupied_percentage < 100.0


def test_occupancy_repeated_cell_reads_previous_density():
    """A cell drawn many times in one update decays once (gather before scatter)."""
    from voxneus_b200 import ops

    lo, hi = (-1.0, -1.0, -1.0), (1.0, 1.0, 1.0)
    density = torch.full((8, 8, 8), 1.0, device=DEV)
    mask = torch.ones(8, 8, 8, dtype=torch.bool, device=DEV)
    idx = [torch.full((5000,), 7, dtype=torch.int64, device=DEV) for _ in range(3)]
    far = torch.full((5000,), 10.0, device=DEV)  # density ~0, not near the surface
    ops.occupancy_update(density, mask, idx, lo, hi, torch.tensor(30.0, device=DEV), False, 0.0, False, 0.95, 0.01,
                         sdf_values=far)
    torch.cuda.synchronize()
    assert float(density[7, 7, 7]) == float(torch.tensor(0.95))
    assert float(density[0, 0, 0]) == 1.0 and bool(mask[7, 7, 7])


def test_occupancy_callable_known_answer_and_query():
    """tests/test_neus2_features.py:30-55 through the module API on the GPU (an analytic SDF
    callable), and is_occupied bit-exact against the oracle, points outside the box included."""
    from voxneus_b200.models import OccupancyGrid

    torch.manual_seed(5)
    occ = OccupancyGrid(resolution=32, threshold=0.01).to(DEV)
    for _ in range(5):
        occ.update_from_sdf(lambda p: torch.linalg.norm(p, dim=-1, keepdim=True) - 0.5, torch.tensor(30.0), 1.0)
    surf = torch.tensor([[0.5, 0.0, 0.0], [0.0, 0.5, 0.0], [0.0, 0.0, 0.5]], device=DEV)
    far = torch.tensor([[0.95, 0.95, 0.95], [-0.95, -0.95, -0.95]], device=DEV)
    assert bool(occ.is_occupied(surf).all()) and not bool(occ.is_occupied(far).all())
    pts = (torch.rand(20000, 3) * 2.4 - 1.2)
    pts[:5] = torch.tensor([[1.0, 1.0, 1.0], [-1.0, -1.0, -1.0], [1.0000001, 0.0, 0.0], [0.0, -1.0, 0.5],
                            [0.99999994, 0.99999994, 0.99999994]])
    got = occ.is_occupied(to(pts.reshape(100, 200, 3))).cpu().reshape(-1)
    ref = O.is_occupied(occ.occupancy_mask.cpu(), pts, torch.tensor([-1.0] * 3), torch.tensor([1.0] * 3))
    assert torch.equal(got, ref)


def test_fused_adam_matches_torch_adam():
    """FusedAdam (one multi-tensor launch, torch.optim.Adam's formula) against torch.optim.Adam:
    three groups with their own learning rates, vector bodies with scalar tails, zero gradients,
    and a parameter whose grad is None for one step (skipped, its step count held back)."""
    from voxneus_b200.training import FusedAdam

    torch.manual_seed(7)
    shapes = [(16, 4099, 2), (64, 51), (64,), (3, 64), (3,), ()]
    base = [torch.randn(s) for s in shapes]
    ours = [b.clone().to(DEV).requires_grad_(True) for b in base]
    ref = [b.clone().to(DEV).requires_grad_(True) for b in base]

    def groups(ps):
        return [{"params": ps[:1], "lr": 1e-2}, {"params": ps[1:5], "lr": 1e-3}, {"params": ps[5:], "lr": 5e-4}]

    opt = FusedAdam(groups(ours), betas=(0.9, 0.999), eps=1e-8)
    opt_ref = torch.optim.Adam(groups(ref), betas=(0.9, 0.999), eps=1e-8, foreach=False)
    for step in range(5):
        grads = [torch.randn(s) * (torch.rand(s) > 0.3) for s in shapes]
        for ps in (ours, ref):
            for k, p in enumerate(ps):
                p.grad = None if (step == 2 and k == 3) else grads[k].to(DEV)
        opt.step()
        opt_ref.step()
        for a, b in zip(ours, ref):
            assert_close(a.detach(), b.detach(), 1e-6, "adam param", scale=1.0)
    for a, b in zip(ours, ref):
        sa, sb = opt.state[a], opt_ref.state[b]
        assert sa["step"] == int(sb["step"])
        assert_close(sa["exp_avg"], sb["exp_avg"], 1e-6, "exp_avg", scale=1.0)
        assert_close(sa["exp_avg_sq"], sb["exp_avg_sq"], 1e-6, "exp_avg_sq", scale=1.0)


@pytest.mark.parametrize("offset", [0, 1])
def test_masked_adam_reference_formula(offset):
    """vx_masked_adam_upd / vx_adam_upd against the extension's formula (adam_upd_kernel.cu:40-82)
    in float64, on a 16-byte aligned buffer (float4 body + tail) and on one offset by 4 bytes
    (scalar path); gradient-0 elements keep p, m and v bit for bit in the masked form."""
    from voxneus_b200 import ops

    torch.manual_seed(8)
    n = 1_000_003
    bufs = [torch.randn(n + offset) for _ in range(4)]
    bufs[1][torch.rand(n + offset) < 0.6] = 0.0  # grad
    bufs[3] = bufs[3].abs()  # exp_avg_sq >= 0
    for masked in (True, False):
        p, g, m, v = (b.clone().to(DEV)[offset:] for b in bufs)
        p0, g0, m0, v0 = (b[offset:].double() for b in bufs)
        step, b1, b2, lr, eps = 3, 0.9, 0.99, 0.1, 1e-8
        ops.adam_update(p, g, m, v, step, b1, b2, lr, eps, masked=masked)
        torch.cuda.synchronize()
        ss = lr * math.sqrt(1 - b2 ** step) / (1 - b1 ** step)
        m1 = b1 * m0 + (1 - b1) * g0
        v1 = b2 * v0 + (1 - b2) * g0 * g0
        p1 = p0 - ss * m1 / (v1.sqrt() + eps)
        if masked:
            keep = g0 == 0
            m1[keep], v1[keep], p1[keep] = m0[keep], v0[keep], p0[keep]
            assert torch.equal(p.cpu()[keep], bufs[0][offset:][keep])
            assert torch.equal(m.cpu()[keep], bufs[2][offset:][keep])
        assert_close(p, p1, 1e-6, "adam p", scale=1.0)
        assert_close(m, m1, 1e-6, "adam m", scale=1.0)
        assert_close(v, v1, 1e-6, "adam v", scale=1.0)


def test_sorted_field_query_is_bitwise_identical():
    """The Morton-ordered query of scattered points (sdf, Eq.7 gradient, normal) writes the same
    bits as the plain query at every point's own index, points outside the box included."""
    from voxneus_b200 import ops

    torch.manual_seed(31)
    res = [160, 144, 176]
    lo, hi = (-1.0, -1.0, -1.0), (1.0, 1.0, 1.0)
    axes = [torch.linspace(-1, 1, r) for r in res]
    gx, gy, gz = torch.meshgrid(*axes, indexing="ij")
    grid = to((torch.sqrt(gx ** 2 + gy ** 2 + gz ** 2) - 0.6 + 0.01 * torch.randn(*res)).reshape(1, 1, *res))
    pts = to((torch.rand(300_001, 3) * 2.2 - 1.1).contiguous())
    a = ops.field_query(grid, lo, hi, pts, sdf=True, grad=True, normal=True)
    b = ops.field_query_sorted(grid, lo, hi, pts, sdf=True, grad=True, normal=True)
    torch.cuda.synchronize()
    for x, y in zip(a[:3], b[:3]):
        assert torch.equal(x, y)


@pytest.mark.parametrize("res", [128, 241, 256, 321, 451, 511, 512])
def test_relax_sphere_membership_at_the_boundary(res):
    """The relax filter |xyz_min + i * eps| < 1.2 of V_R (training/trainer.py:262-266) on every
    lattice vertex within 1e-4 of the radius. Membership equals the oracle's (the reference's
    float32 ops on the host, torch.linalg.norm) wherever the exact distance is more than two ulps
    from the float32 radius; inside that band any float32 evaluation order may decide either way,
    and the disagreements there (with the host norm and with torch's CUDA norm) are printed."""
    from voxneus_b200 import ops

    eps = torch.tensor(2.0 / (res - 1), dtype=torch.float32)
    lo = torch.tensor([-1.0, -1.0, -1.0])
    i = torch.arange(res)
    ii, jj = torch.meshgrid(i, i, indexing="ij")
    c = (-1.0 + i.double() * float(eps))
    rem = 1.2 ** 2 - c[ii] ** 2 - c[jj] ** 2
    ok = rem > 0
    kc = ((torch.sqrt(rem.clamp(min=0)) + 1.0) / float(eps)).round().long()
    cand = []
    for dk in (-1, 0, 1):
        for k in (kc + dk, (res - 1) - kc - dk):  # the +z and -z crossings of the sphere
            cand.append(torch.stack([ii, jj, k], -1)[ok & (k >= 0) & (k < res)])
    verts = torch.unique(torch.cat(cand).reshape(-1, 3), dim=0)
    wc = lo + verts.to(torch.float32) * eps  # the reference's float32 world corners
    r64 = wc.double().norm(dim=-1)
    near = (r64 - 1.2).abs() < 1e-4
    verts, wc, r64 = verts[near], wc[near], r64[near]
    assert verts.shape[0] > 0
    host = torch.linalg.norm(wc, dim=-1) < 1.2
    dev_norm = (torch.linalg.norm(wc.to(DEV), dim=-1) < 1.2).cpu()
    rs = [res] * 3
    bm = ops.new_bitmap(rs, DEV)
    ops.vr_mark_corners(to(verts), rs, bm)
    counts = ops.vr_count(bm, None, rs, (-1.0,) * 3, (1.0,) * 3, 1.2, 0.0)
    n = int(counts[1])
    _, lin = ops.vr_compact(bm, None, rs, (-1.0,) * 3, (1.0,) * 3, 1.2, 0.0, counts, n)
    vlin = verts[:, 0] * res * res + verts[:, 1] * res + verts[:, 2]
    kern = torch.isin(vlin, lin.cpu())
    r32 = float(torch.tensor(1.2, dtype=torch.float32))
    ambiguous = (r64 - r32).abs() <= 2 * 2.0 ** -23 * r32
    assert torch.equal(kern[~ambiguous], host[~ambiguous])
    print(f"res {res}: {verts.shape[0]} vertices within 1e-4 of r = 1.2, {int(ambiguous.sum())} within 2 ulps; "
          f"kernel vs host norm differ on {int((kern != host).sum())}, vs CUDA norm on {int((kern != dev_norm).sum())}")


def test_radiance_mlp_module_on_the_fused_kernels():
    """RadianceMLP.forward (models/radiance_mlp.py:81-98) runs the tensor-core MLP, forward and
    adjoint, against the oracle; the view embedding takes no gradient (an error when asked)."""
    from voxneus_b200.models import RadianceMLP

    torch.manual_seed(17)
    mlp = RadianceMLP().to(DEV)
    l0, l1 = mlp.net[0], mlp.net[2]
    p = 3000
    h, v, n = torch.randn(p, 32), torch.randn(p, 16), torch.randn(p, 3)
    with torch.no_grad():
        z64 = torch.cat([h, v, n], -1).double() @ l0.weight.detach().cpu().double().T + l0.bias.detach().cpu().double()
        keep = (z64.abs() > 1e-6 * float(z64.abs().max())).all(dim=1)  # away from the ReLU kinks
    h, v, n = h[keep], v[keep], n[keep]
    ws = [t.detach().cpu().clone().requires_grad_(True) for t in (l0.weight, l0.bias, l1.weight, l1.bias)]
    hr, nr = h.clone().requires_grad_(True), n.clone().requires_grad_(True)
    ref = O.radiance_mlp(hr, v, nr, *ws)
    cot = torch.randn(ref.shape)
    (ref * cot).sum().backward()
    hd, nd = to(h).requires_grad_(True), to(n).requires_grad_(True)
    out = mlp(hd.reshape(-1, 1, 32), to(v).reshape(-1, 1, 16), nd.reshape(-1, 1, 3)).reshape(-1, 3)
    assert_close(out, ref.detach(), VAL_TOL, "rgb")
    (out * to(cot)).sum().backward()
    assert_close(hd.grad, hr.grad, GRAD_TOL, "d hash")
    assert_close(nd.grad, nr.grad, GRAD_TOL, "d normal")
    for a, b, nm in zip((l0.weight, l0.bias, l1.weight, l1.bias), ws, ("W0", "b0", "W1", "b1")):
        assert_close(a.grad, b.grad, GRAD_TOL, nm)
    with pytest.raises(NotImplementedError):
        mlp(hd, to(v).requires_grad_(True), nd)


@pytest.mark.parametrize("res,offset", [((64, 48, 80), 0), ((37, 41, 29), 0), ((64, 48, 80), 1)])
def test_geometry_forward_matches_field_query_bitwise(res, offset):
    """The render geometry forward (positions o + d*t from rays and midpoints) and the field query
    (the same positions given as points) give the same bits: SDF, Eq.7 gradient and normal, for rays
    crossing the whole box (border cells with their one-sided differences included), odd row
    lengths, and a grid view 4 bytes off 16-byte alignment."""
    from voxneus_b200 import ops

    torch.manual_seed(41 + offset)
    n_vox = res[0] * res[1] * res[2]
    store = torch.randn(n_vox + 4, device=DEV) * 0.3
    grid = store[offset:offset + n_vox].view(1, 1, *res)
    lo, hi = (-1.0, -0.8, -1.2), (1.0, 0.9, 1.1)
    nr, ns = 300, 128
    o = torch.randn(nr, 3)
    o = 2.5 * o / o.norm(dim=-1, keepdim=True)
    d = -o / o.norm(dim=-1, keepdim=True) + 0.2 * torch.randn(nr, 3)
    d = d / d.norm(dim=-1, keepdim=True)
    mid = torch.sort(torch.rand(nr, ns) * 4.0 + 0.5, dim=-1).values
    od, dd, md = to(o), to(d), to(mid)
    sdf = torch.empty(nr, ns, device=DEV)
    nrm = torch.empty(nr, ns, 3, device=DEV)
    gr = torch.empty(nr, ns, 3, device=DEV)
    ops.call("vx_render_geometry_forward", ops.ptr(grid), ops.i3(res), ops.f3(lo), ops.f3(hi), ops.ptr(od),
             ops.ptr(dd), ops.ptr(md), nr, ns, ops.ptr(sdf), ops.ptr(nrm), ops.ptr(gr), None, ops.stream_ptr(DEV))
    pts = (od[:, None, :] + dd[:, None, :] * md[..., None]).reshape(-1, 3).contiguous()
    f_sdf = torch.empty(nr * ns, device=DEV)
    f_nrm = torch.empty(nr * ns, 3, device=DEV)
    f_gr = torch.empty(nr * ns, 3, device=DEV)
    ops.call("vx_field_query", ops.ptr(grid), ops.i3(res), ops.f3(lo), ops.f3(hi), ops.ptr(pts), nr * ns,
             ops.ptr(f_sdf), ops.ptr(f_gr), ops.ptr(f_nrm), None, None, ops.stream_ptr(DEV))
    torch.cuda.synchronize()
    assert torch.equal(sdf.reshape(-1), f_sdf)
    assert torch.equal(gr.reshape(-1, 3), f_gr)
    assert torch.equal(nrm.reshape(-1, 3), f_nrm)


def test_field_query_at_512():
    """The large-grid field query workload (512^3 grid of 32 Gaussian-bump spheres): 2^20 scattered
    points through the Morton-sorted path equal the unsorted kernel bit for bit; a subset of them
    and of a 320^3 lattice match the oracle's grid_sample SDF and Eq.7 normals (lattice normals within
    the float32 oracle's own distance from float64; models/sdf_grid.py:
    90-160, geometry/gradients.py:59-139, the batched query of geometry/mesh.py:80-114)."""
    from voxneus_b200 import ops, synthetic

    res = 512
    grid = synthetic.bumpy_spheres_grid(res, 32, seed=3, device=DEV).contiguous()
    lo, hi = (-1.0, -1.0, -1.0), (1.0, 1.0, 1.0)
    g = torch.Generator(device=DEV).manual_seed(5)
    pts = (torch.rand(1 << 20, 3, device=DEV, generator=g) * 2 - 1).contiguous()
    assert pts.shape[0] >= ops.SORTED_QUERY_MIN_POINTS and grid.numel() * 4 >= ops.SORTED_QUERY_MIN_GRID_BYTES
    s_sorted, _, n_sorted, _, _ = ops.field_query(grid, lo, hi, pts, sdf=True, normal=True)
    o_sdf = torch.empty(pts.shape[0], device=DEV)
    o_nrm = torch.empty(pts.shape[0], 3, device=DEV)
    ops.call("vx_field_query", ops.ptr(grid), ops.i3([res] * 3), ops.f3(lo), ops.f3(hi), ops.ptr(pts), pts.shape[0],
             ops.ptr(o_sdf), None, ops.ptr(o_nrm), None, None, ops.stream_ptr(DEV))
    assert torch.equal(s_sorted, o_sdf) and torch.equal(n_sorted, o_nrm)
    g5 = grid.cpu()
    pick = torch.randperm(pts.shape[0], generator=torch.Generator().manual_seed(6))[:4096]
    p = pts.cpu()[pick]
    lo_t, hi_t = torch.tensor(lo), torch.tensor(hi)
    assert_close(s_sorted.cpu()[pick], O.query_sdf(g5, p, lo_t, hi_t).squeeze(-1), VAL_TOL, "sdf 512")
    _, nrm, _, _ = O.query_normals(g5, p, lo_t, hi_t)
    assert_close(n_sorted.cpu()[pick], nrm, VAL_TOL, "normal")
    # lattice: 320^3 points spanning [-1, 1] at the values of torch.linspace on the device (its
    # two-sided split; the host's vectorised linspace differs from it by an ulp in places, which
    # moves an Eq.7 normal of this bumpy field by up to ~3e-5), z fastest
    lat = 320
    ls, ln = ops.field_query_lattice(grid, lo, hi, [lat] * 3, lo, hi)
    ax = torch.linspace(-1.0, 1.0, lat, device=DEV).cpu()
    idx = torch.randint(0, lat, (4096, 3), generator=torch.Generator().manual_seed(7))
    q = torch.stack([ax[idx[:, 0]], ax[idx[:, 1]], ax[idx[:, 2]]], -1)
    flat = (idx[:, 0] * lat + idx[:, 1]) * lat + idx[:, 2]
    assert_close(ls.cpu()[flat], O.query_sdf(g5, q, lo_t, hi_t).squeeze(-1), VAL_TOL, "lattice sdf")
    # normals of this bumpy field are ill-conditioned in float32 at a few points (the float32 oracle
    # itself is up to ~3e-5 from float64): the bound is the float32 oracle's own distance from the
    # float64 one (at least 1e-5), measured against float64
    _, qn, _, _ = O.query_normals(g5, q, lo_t, hi_t)
    _, qn64, _, _ = O.query_normals(g5.double(), q.double(), lo_t.double(), hi_t.double())
    bound = max(VAL_TOL, 2.0 * float((qn.double() - qn64).abs().max()))
    got = ln.cpu()[flat].double()
    assert float((got - qn64).abs().max()) <= bound, ("lattice normal", float((got - qn64).abs().max()), bound)
    assert float(((got - qn.double()).abs() > VAL_TOL).any(-1).double().mean()) < 0.005

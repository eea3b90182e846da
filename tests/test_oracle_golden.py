"""Pins the oracle (oracle/reference_path.py) to vectors produced by the reference itself.

CPU only. Float comparisons are exact where the oracle repeats the reference's op sequence
on the same device, otherwise within 1e-6 relative; integer outputs are bit-exact.
"""

import math

import numpy as np
import torch

from oracle import reference_path as O


def close(a, b, rtol=1e-6, atol_scale=1e-6):
    a = torch.as_tensor(a, dtype=torch.float64)
    b = torch.as_tensor(b, dtype=torch.float64)
    scale = max(1.0, float(b.abs().max())) if b.numel() else 1.0
    return torch.allclose(a, b, rtol=rtol, atol=atol_scale * scale)


def test_field_query(golden):
    g = golden("field_query.npz")
    grid = g["grid"].clone().requires_grad_(True)
    lo = torch.tensor([-1.0, -1.0, -1.0])
    hi = torch.tensor([1.0, 1.0, 1.0])
    sdf = O.query_sdf(grid, g["pts"], lo, hi)
    grad, normal, corners, weights = O.query_normals(grid, g["pts"], lo, hi)
    assert torch.equal(corners, g["corners"])
    assert close(sdf, g["sdf"]) and close(grad, g["grad"]) and close(normal, g["normal"])
    assert close(weights, g["weights"])
    loss = (grad * g["c1"]).sum() + (sdf * g["c2"]).sum() + (normal * g["c3"]).sum()
    loss.backward()
    assert close(grid.grad, g["grid_grad"], rtol=1e-5, atol_scale=1e-6)


def test_sample_pdf_and_near_far(golden):
    g = golden("sampler.npz")
    det = O.sample_pdf(g["bins"], g["weights"], 16, det=True)
    assert close(det, g["det"])
    sto = O.sample_pdf(g["bins"], g["weights"], 16, det=False, u=g["u"])
    assert close(sto, g["sto"])
    near, far = O.near_far_from_sphere(g["rays_o"], g["rays_d"])
    assert torch.equal(near, g["near"]) and torch.equal(far, g["far"])
    # rays.py known answer (tests/test_rays.py:48-57): o=(0,0,3), d=(0,0,-1) -> (2, 4)
    n, f = O.near_far_from_sphere(torch.tensor([[0.0, 0.0, 3.0]]), torch.tensor([[0.0, 0.0, -1.0]]))
    assert abs(n.item() - 2.0) < 1e-3 and abs(f.item() - 4.0) < 1e-3


def _scene(g):
    params = [g[k].clone().requires_grad_(True) for k in ("grid", "variance", "embeddings", "w0", "b0", "w1", "b1")]
    return O.OracleScene(*params, occupancy=g["occupancy"])


def _check_render(g, perturb):
    sc = _scene(g)
    kw = dict(n_samples=16, n_importance=16, steps=4, perturb=perturb)
    if perturb:
        kw.update(t_rand=g["t_rand"], us=list(g["us"]))
    z, dists, mid = O.sample_multistep_sdf(g["rays_o"], g["rays_d"], g["near"], g["far"], sc.sdf_fn,
                                           16, 16, 4, perturb, sc.occ_fn,
                                           t_rand=kw.get("t_rand"), us=kw.get("us"))
    assert close(z, g["z"]) and close(dists, g["dists"]) and close(mid, g["mid"])
    out = sc.render(g["rays_o"], g["rays_d"], g["near"], g["far"], **kw)
    for k in ("rgb", "depth", "normal", "opacity", "weights", "alpha", "transmittance", "pts", "sdf_samples",
              "normal_samples", "grad_samples"):
        assert close(out[k], g[k]), k
    loss = O.huber(out["rgb"], g["target"], 0.1)
    assert close(loss, g["loss"])
    loss.backward()
    for k, p in zip(("grid", "variance", "embeddings", "w0", "b0", "w1", "b1"), sc.params()):
        assert close(p.grad, g[k + "_grad"], rtol=1e-5, atol_scale=1e-6), k
    verts, lin = O.extract_active_vertices(out["corner_indices"], sc.res())
    assert torch.equal(verts, g["vr_verts"]) and torch.equal(lin, g["vr_linear"])
    g3 = sc.grid.detach().reshape(sc.res())
    le, ge = O.eikonal(g3, verts, sc.eps(), sc.res())
    lc, gc = O.curvature(g3, verts, sc.eps(), sc.res())
    assert close(le, g["loss_eik"]) and close(ge, g["grad_eik"].reshape(ge.shape))
    assert close(lc, g["loss_curv"]) and close(gc, g["grad_curv"].reshape(gc.shape))


def test_render_deterministic(golden):
    _check_render(golden("render_det.npz"), perturb=False)


def test_render_perturbed(golden):
    _check_render(golden("render_perturb.npz"), perturb=True)


def test_sampler_draw_order(golden):
    """The reference draws rand_like(z) (N,64) then rand(N,16) per step; same seed, same draws."""
    g = golden("render_perturb.npz")
    torch.manual_seed(6)
    t_rand, us = O.sampler_draws(24, 16, 16, 4, True)
    assert torch.equal(t_rand, g["t_rand"]) and torch.equal(torch.stack(us), g["us"])


def test_regularizers(golden):
    g = golden("regularizers.npz")
    g3 = g["grid"].reshape(16, 14, 12)
    le, ge = O.eikonal(g3, g["verts"], g["voxel_size"], (16, 14, 12))
    lc, gc = O.curvature(g3, g["verts"], g["voxel_size"], (16, 14, 12))
    assert close(le, g["loss_eik"]) and close(ge, g["grad_eik"].reshape(ge.shape))
    assert close(lc, g["loss_curv"]) and close(gc, g["grad_curv"].reshape(gc.shape))
    v, lin = O.extract_active_vertices(g["corners"], (16, 14, 12))
    assert torch.equal(v, g["vr_verts"]) and torch.equal(lin, g["vr_linear"])


def test_regularizers_vs_fp64_autograd():
    """tests/test_regularization_grads.py:30-102 pattern: closed form vs float64 autograd, < 1e-6."""
    torch.manual_seed(42)
    verts = torch.tensor([[5, 5, 5], [6, 5, 5], [7, 8, 9], [10, 11, 12], [4, 8, 6]])
    eps = torch.tensor([0.1, 0.1, 0.1], dtype=torch.float64)
    grid = torch.randn(16, 16, 16, dtype=torch.float64, requires_grad=True)
    i, j, k = verts.T
    n = torch.stack([(grid[i + 1, j, k] - grid[i - 1, j, k]) / 0.2, (grid[i, j + 1, k] - grid[i, j - 1, k]) / 0.2,
                     (grid[i, j, k + 1] - grid[i, j, k - 1]) / 0.2], -1)
    loss = torch.mean((torch.sqrt((n ** 2).sum(-1) + 1e-12) - 1.0) ** 2)
    loss.backward()
    le, ge = O.eikonal(grid.detach(), verts, eps, (16, 16, 16))
    assert abs(le.item() - loss.item()) < 1e-6
    assert (ge - grid.grad).abs().max().item() < 1e-6


def test_upsample(golden):
    g = golden("upsample.npz")
    assert close(O.upsample_grid(g["grid"], [17, 13, 11]), g["out_a"])
    assert close(O.upsample_grid(g["grid"], 12), g["out_b"])


def test_hash_and_sh(golden):
    g = golden("hash.npz")
    res = O.hash_level_resolutions(16)
    assert close(O.hash_encode(g["x"], g["embeddings"], res), g["feats"])
    assert close(O.hash_encode(g["x"], g["embeddings"], res, active_levels=5.5), g["feats_l55"])
    assert torch.equal(O.sh4(torch.as_tensor(g["dirs"])), torch.as_tensor(g["sh"]))  # the reference's bits
    # uint32 hash arithmetic equals the reference int64 hash modulo 2^19
    c = np.random.default_rng(0).integers(0, 2050, size=(1000, 3))
    h64 = torch.remainder((torch.from_numpy(c[:, 0]) * 1) ^ (torch.from_numpy(c[:, 1]) * 2654435761)
                          ^ (torch.from_numpy(c[:, 2]) * 805459861), 1 << 19)
    assert np.array_equal(O.hash_index_np(c, 19), h64.numpy())


def test_alpha_and_composite(golden):
    g = golden("alpha.npz")
    n = g["sdf"].shape[1]
    a = O.neus_alpha(g["sdf"].unsqueeze(-1), g["normals"], g["dirs"].unsqueeze(1).expand(-1, n, -1), g["dists"], g["s"])
    assert close(a, g["alpha"])
    w, t = O.composite_weights(g["acut"])
    assert torch.equal(w, g["wcut"]) and torch.equal(t, g["tcut"])
    assert w[0, 3].item() == 0.0 and t[0, 3].item() < 1e-4


def test_alpha_known_answers():
    """tests/test_neus_alpha.py:12-41: alpha(0) > 0.5 and alpha(1) < 1e-4 at s=50, delta=0.05, cos=-1."""
    d = torch.tensor([[0.0, 0.0, -1.0]])
    n = torch.tensor([[0.0, 0.0, 1.0]])
    a0 = O.neus_alpha(torch.tensor([[0.0]]), n, d, torch.tensor([[0.05]]), torch.tensor(50.0))
    a1 = O.neus_alpha(torch.tensor([[1.0]]), n, d, torch.tensor([[0.05]]), torch.tensor(50.0))
    assert a0.item() > 0.5 and a1.item() < 1e-4


def test_hash_resolutions():
    res = O.hash_level_resolutions(16)
    assert res[0] == 16 and res[-1] == 2048 and all(b >= a for a, b in zip(res, res[1:]))
    assert math.isclose(O.level_weight(5, 5.5), 0.5)


def test_occupancy_update(golden):
    """Three EMA updates replayed at the reference's own cell draws reproduce its grids exactly."""
    g = golden("occupancy.npz")
    lo, hi = (-1.0, -1.0, -1.0), (1.0, 1.0, 1.0)
    glo, ghi = torch.tensor(lo), torch.tensor(hi)
    density = torch.zeros(32, 32, 32)
    mask = torch.ones(32, 32, 32, dtype=torch.bool)
    for k in range(3):
        O.occupancy_update(density, mask, g[f"idx{k}"], lambda p: O.query_sdf(g["grid"], p, glo, ghi), g[f"s{k}"],
                           k == 0, lo, hi)
        assert torch.equal(density, g[f"density{k}"]) and torch.equal(mask, g[f"mask{k}"])
    # untouched cells keep the initial state: density 0, mask True
    drawn = torch.zeros(32, 32, 32, dtype=torch.bool)
    for k in range(3):
        i = g[f"idx{k}"]
        drawn[i[0], i[1], i[2]] = True
    assert bool((density[~drawn] == 0).all()) and bool(mask[~drawn].all())
    assert bool((~mask[drawn]).any()) and bool(mask[drawn].any())


def test_occupancy_sphere_known_answer():
    """tests/test_neus2_features.py:30-55: sphere r=0.5 on a 32^3 grid, s=30, five full-ratio
    updates -> the three axis surface points are occupied and two far points are not both occupied."""
    torch.manual_seed(0)
    lo, hi = (-1.0, -1.0, -1.0), (1.0, 1.0, 1.0)
    density = torch.zeros(32, 32, 32)
    mask = torch.ones(32, 32, 32, dtype=torch.bool)
    for k in range(5):
        idx = torch.stack([torch.randint(0, 32, (32 ** 3,)) for _ in range(3)])
        O.occupancy_update(density, mask, idx, lambda p: torch.linalg.norm(p, dim=-1) - 0.5, 30.0, k == 0, lo, hi)
    surf = O.is_occupied(mask, torch.tensor([[0.5, 0.0, 0.0], [0.0, 0.5, 0.0], [0.0, 0.0, 0.5]]), torch.tensor(lo),
                         torch.tensor(hi))
    far = O.is_occupied(mask, torch.tensor([[0.95, 0.95, 0.95], [-0.95, -0.95, -0.95]]), torch.tensor(lo),
                        torch.tensor(hi))
    assert bool(surf.all()) and not bool(far.all())

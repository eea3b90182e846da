"""Generate golden vectors from the reference implementation (rishidevde/VoxNeus).

Run in a container where the reference source tree is available (read-only), pointing at the
reference's ``Code/`` directory by argument or by the VOXNEUS_REFERENCE environment variable:

    python tests/golden/make_golden.py --reference <reference>/Code [--only NAME ...]

It imports the reference's own Python modules in their pure-PyTorch mode (the reference's
optional CUDA extension is not built, so every call takes its plain torch path), runs each
hot-path function on small seeded inputs on the CPU and writes ``tests/golden/*.npz``.
The fixtures are what pins the oracle; the GPU box never needs the reference tree.
"""

from __future__ import annotations

import argparse
import math
import os
import sys

import numpy as np
import torch

HERE = os.path.dirname(os.path.abspath(__file__))


def _import_reference(path: str):
    sys.dont_write_bytecode = True
    sys.path.insert(0, path)
    import voxneus.cuda as vcuda  # noqa: F401

    if vcuda.is_cuda_available():
        raise RuntimeError("reference CUDA backend is importable; golden vectors must use the torch path")
    from voxneus.geometry import upsample as up
    from voxneus.models.radiance_hash import PyTorchHashGrid
    from voxneus.models.embedder import SphericalHarmonicsEmbedder
    from voxneus.models.sdf_grid import DenseSDFGrid
    from voxneus.models.voxneus import VoxNeuS
    from voxneus.regularization.active_vertices import extract_active_vertices
    from voxneus.regularization.curvature import compute_curvature_loss_and_gradient
    from voxneus.regularization.eikonal import compute_eikonal_loss_and_gradient
    from voxneus.rendering import rays as rrays
    from voxneus.rendering import sampler as rsampler
    from voxneus.rendering import neus_alpha as ralpha
    from voxneus.rendering import volume_render as rvr
    from voxneus.training import scheduler as rsched
    from voxneus.rendering.occupancy_grid import OccupancyGrid

    return dict(OccupancyGrid=OccupancyGrid, up=up, PyTorchHashGrid=PyTorchHashGrid, SH=SphericalHarmonicsEmbedder, DenseSDFGrid=DenseSDFGrid,
                VoxNeuS=VoxNeuS, eav=extract_active_vertices, curv=compute_curvature_loss_and_gradient,
                eik=compute_eikonal_loss_and_gradient, rays=rrays, sampler=rsampler, alpha=ralpha, vr=rvr,
                sched=rsched)


def hemisphere_rays(n_rays: int, seed: int, radius: float = 3.0, n_cams: int = 9, focal: float = 40.0,
                    w: int = 64, h: int = 48):
    """Pinhole rays from cameras on a radius-3 hemisphere aimed at the origin (OpenCV convention)."""
    g = torch.Generator().manual_seed(seed)
    cams = []
    for c in range(n_cams):
        el = math.radians(10.0 + 70.0 * (c + 0.5) / n_cams)
        az = 2.0 * math.pi * c / n_cams
        pos = torch.tensor([radius * math.cos(el) * math.cos(az), radius * math.cos(el) * math.sin(az),
                            radius * math.sin(el)])
        fwd = -pos / pos.norm()
        up = torch.tensor([0.0, 0.0, 1.0])
        right = torch.linalg.cross(fwd, up)
        right = right / right.norm()
        down = torch.linalg.cross(fwd, right)
        cams.append((pos, torch.stack([right, down, fwd], dim=1)))
    ci = torch.randint(0, n_cams, (n_rays,), generator=g)
    px = torch.randint(0, w, (n_rays,), generator=g).float() + 0.5
    py = torch.randint(0, h, (n_rays,), generator=g).float() + 0.5
    o = torch.zeros(n_rays, 3)
    d = torch.zeros(n_rays, 3)
    for r in range(n_rays):
        pos, rot = cams[int(ci[r])]
        v = torch.tensor([(px[r] - w / 2) / focal, (py[r] - h / 2) / focal, 1.0])
        dd = rot @ v
        o[r] = pos
        d[r] = dd / dd.norm()
    return o, d


def save(name: str, **arrays):
    out = {}
    for k, v in arrays.items():
        if isinstance(v, torch.Tensor):
            v = v.detach().cpu().numpy()
        out[k] = np.asarray(v)
    np.savez_compressed(os.path.join(HERE, name), **out)
    print(f"wrote {name}: " + ", ".join(f"{k}{list(v.shape)}" for k, v in out.items()))


def gen_field_query(R):
    torch.manual_seed(1)
    res = [12, 10, 9]
    m = R["DenseSDFGrid"](resolution=res, init_mode="sphere")
    with torch.no_grad():
        m.grid.data.copy_(torch.randn_like(m.grid) * 0.3 + m.grid.data)
    pts = torch.rand(300, 3) * 2.2 - 1.1
    pts[:6] = torch.tensor([[1.0, 1.0, 1.0], [-1.0, -1.0, -1.0], [1.0, 0.0, -1.0], [0.9999, -0.9999, 0.5],
                            [0.0, 0.0, 0.0], [-1.0, 1.0, 0.3]])
    sdf = m.query_sdf(pts)
    grad, normal, corners, weights = m.query_normals(pts, gradient_mode="interpolated")
    c1, c2, c3 = torch.randn(300, 3), torch.randn(300, 1), torch.randn(300, 3)
    loss = (grad * c1).sum() + (sdf * c2).sum() + (normal * c3).sum()
    loss.backward()
    save("field_query.npz", grid=m.grid.detach(), pts=pts, sdf=sdf, grad=grad, normal=normal, corners=corners,
         weights=weights, c1=c1, c2=c2, c3=c3, grid_grad=m.grid.grad, voxel_size=m.voxel_size)


def gen_sampler(R):
    torch.manual_seed(2)
    bins = torch.sort(torch.rand(7, 12) * 3.0 + 1.0, dim=-1)[0]
    weights = torch.rand(7, 11) ** 3
    weights[0] = 0.0
    det = R["sampler"].sample_pdf(bins, weights, 16, det=True)
    torch.manual_seed(3)
    u = torch.rand(7, 16)
    torch.manual_seed(3)
    sto = R["sampler"].sample_pdf(bins, weights, 16, det=False)
    o = torch.tensor([[0.0, 0.0, 3.0], [0.1, -2.5, 1.0], [2.0, 2.0, 2.0], [0.3, 0.2, -2.9]])
    d = torch.tensor([[0.0, 0.0, -1.0], [0.0, 1.0, -0.2], [-1.0, -1.0, -1.0], [0.05, -0.1, 1.0]])
    d = d / d.norm(dim=-1, keepdim=True)
    near, far = R["rays"].near_far_from_sphere(o, d, radius=1.0)
    save("sampler.npz", bins=bins, weights=weights, det=det, u=u, sto=sto, rays_o=o, rays_d=d, near=near, far=far)


def gen_render(R, perturb: bool, name: str, n_samples: int = 16, n_importance: int = 16, grid_res: int = 24,
               hash_log2: int = 8, n_rays: int = 24):
    torch.manual_seed(4)
    model = R["VoxNeuS"](grid_res=grid_res, hash_n_levels=16, hash_log2_size=hash_log2, occupancy_res=8,
                         force_pytorch=True)
    with torch.no_grad():
        model.sdf_grid.grid.add_(torch.randn_like(model.sdf_grid.grid) * 0.01)
        model.radiance_hash.encoder.embeddings.uniform_(-0.5, 0.5)
        occ = torch.rand(8, 8, 8) > 0.3
        model.occupancy_grid.occupancy_mask.copy_(occ)
    o, d = hemisphere_rays(n_rays, seed=5)
    near, far = R["rays"].near_far_from_sphere(o, d, radius=1.0)
    sampler = R["sampler"].RaySampler(n_samples=n_samples, n_importance=n_importance, perturb=perturb)
    target = torch.rand(n_rays, 3)
    per = n_importance // 4
    torch.manual_seed(6)
    t_rand = torch.rand(n_rays, n_samples) if perturb else torch.zeros(0)
    us = [torch.rand(n_rays, per) for _ in range(4)] if perturb else []
    torch.manual_seed(6)
    z, dists, mid = sampler.sample_multistep_sdf(o, d, near, far, lambda p: model.sdf_grid.query_sdf(p).squeeze(-1),
                                                 n_samples=n_samples, n_importance=n_importance, up_sample_steps=4,
                                                 occupancy_grid=model.occupancy_grid)
    torch.manual_seed(6)
    out = model.render(o, d, sampler, near, far, up_sample_steps=4, sphere_radius=1.0)
    loss = R["vr"].compute_huber_color_loss(out["rgb"], target, delta=0.1)
    loss.backward()
    res = model.sdf_grid.res
    verts, lin = R["eav"](out["corner_indices"], res)
    le, ge = R["eik"](model.sdf_grid.grid.detach(), verts, model.sdf_grid.voxel_size, res)
    lc, gc = R["curv"](model.sdf_grid.grid.detach(), verts, model.sdf_grid.voxel_size, res)
    sd = model.state_dict()
    save(name, grid=sd["sdf_grid.grid"], variance=sd["variance_net.variance"],
         embeddings=sd["radiance_hash.encoder.embeddings"], w0=sd["radiance_mlp.net.0.weight"],
         b0=sd["radiance_mlp.net.0.bias"], w1=sd["radiance_mlp.net.2.weight"], b1=sd["radiance_mlp.net.2.bias"],
         occupancy=model.occupancy_grid.occupancy_mask, rays_o=o, rays_d=d, near=near, far=far, target=target,
         t_rand=t_rand, us=torch.stack(us) if us else torch.zeros(0), z=z, dists=dists, mid=mid,
         rgb=out["rgb"], depth=out["depth"], normal=out["normal"], opacity=out["opacity"], weights=out["weights"],
         alpha=out["alpha"], transmittance=out["transmittance"], pts=out["pts"], sdf_samples=out["sdf_samples"],
         normal_samples=out["normal_samples"], grad_samples=out["grad_samples"], loss=loss,
         grid_grad=model.sdf_grid.grid.grad, variance_grad=model.variance_net.variance.grad,
         embeddings_grad=model.radiance_hash.encoder.embeddings.grad,
         w0_grad=model.radiance_mlp.net[0].weight.grad, b0_grad=model.radiance_mlp.net[0].bias.grad,
         w1_grad=model.radiance_mlp.net[2].weight.grad, b1_grad=model.radiance_mlp.net[2].bias.grad,
         vr_verts=verts, vr_linear=lin, loss_eik=le, grad_eik=ge, loss_curv=lc, grad_curv=gc)


def gen_regularizers(R):
    torch.manual_seed(7)
    res = torch.tensor([16.0, 14.0, 12.0])
    vs = torch.tensor([2.0 / 15, 2.0 / 13, 2.0 / 11])
    grid = torch.randn(1, 1, 16, 14, 12)
    verts = torch.stack([torch.randint(0, 16, (400,)), torch.randint(0, 14, (400,)), torch.randint(0, 12, (400,))], -1)
    # distinct vertices (border ones included), kept in first-occurrence order
    _, first = np.unique((verts[:, 0] * 168 + verts[:, 1] * 12 + verts[:, 2]).numpy(), return_index=True)
    verts = verts[torch.from_numpy(np.sort(first))]
    le, ge = R["eik"](grid, verts, vs, res)
    lc, gc = R["curv"](grid, verts, vs, res)
    corners = torch.stack([torch.randint(-1, 17, (50, 8)), torch.randint(0, 14, (50, 8)),
                           torch.randint(0, 13, (50, 8))], -1)
    vr, vl = R["eav"](corners, res)
    save("regularizers.npz", grid=grid, verts=verts, voxel_size=vs, loss_eik=le, grad_eik=ge, loss_curv=lc,
         grad_curv=gc, corners=corners, vr_verts=vr, vr_linear=vl)


def gen_upsample(R):
    torch.manual_seed(8)
    g = torch.randn(1, 1, 9, 7, 5)
    save("upsample.npz", grid=g, out_a=R["up"].upsample_sdf_grid(g, [17, 13, 11]), out_b=R["up"].upsample_sdf_grid(g, 12))


def gen_hash(R):
    torch.manual_seed(9)
    enc = R["PyTorchHashGrid"](n_levels=16, n_features_per_level=2, log2_hashmap_size=8)
    with torch.no_grad():
        enc.embeddings.uniform_(-1.0, 1.0)
    x = torch.rand(200, 3)
    x[:4] = torch.tensor([[0.0, 0.0, 0.0], [1.0, 1.0, 1.0], [0.5, 1.0, 0.0], [0.999999, 0.0, 0.25]])
    f_all = enc(x)
    f_55 = enc(x, active_levels=5.5)
    sh = R["SH"](degree=4)(torch.nn.functional.normalize(torch.randn(50, 3), dim=-1))
    dirs = torch.nn.functional.normalize(torch.randn(50, 3), dim=-1)
    save("hash.npz", embeddings=enc.embeddings.detach(), x=x, feats=f_all, feats_l55=f_55, dirs=dirs,
         sh=R["SH"](degree=4)(dirs), sh_unused=sh)


def gen_alpha(R):
    torch.manual_seed(10)
    n = 64
    sdf = torch.randn(4, n) * 0.2
    nrm = torch.nn.functional.normalize(torch.randn(4, n, 3), dim=-1)
    dirs = torch.nn.functional.normalize(torch.randn(4, 3), dim=-1)
    dists = torch.rand(4, n) * 0.1
    s = torch.tensor(37.0)
    a = R["alpha"].compute_neus_alpha(sdf.unsqueeze(-1), nrm, dirs.unsqueeze(1).expand(-1, n, -1), dists, s)
    acut = torch.zeros(2, 10)
    acut[0, 0] = 0.999
    acut[0, 1] = 0.999
    acut[1] = torch.rand(10)
    w, t = R["vr"].composite_weights(acut)
    save("alpha.npz", sdf=sdf, normals=nrm, dirs=dirs, dists=dists, s=s, alpha=a, acut=acut, wcut=w, tcut=t)


def gen_occupancy(R):
    """OccupancyGrid.update_from_sdf (rendering/occupancy_grid.py:62-119): three EMA updates of a
    32^3 occupancy grid from a perturbed sphere SDF on a 20^3 grid. The cell draws of each update
    are replayed from the same seed first so that the fixture carries the indices the reference drew."""
    torch.manual_seed(11)
    m = R["DenseSDFGrid"](resolution=20, init_mode="sphere")
    with torch.no_grad():
        m.grid.add_(0.03 * torch.randn_like(m.grid))
    occ = R["OccupancyGrid"](resolution=32)
    out = dict(grid=m.grid.detach())
    for k, (s, ratio) in enumerate([(30.0, 0.05), (45.0, 0.05), (80.0, 0.0)]):
        seed = 100 + k
        torch.manual_seed(seed)
        n = max(int(32 ** 3 * ratio), 1024)
        idx = torch.stack([torch.randint(0, 32, (n,)) for _ in range(3)])
        torch.manual_seed(seed)
        occ.update_from_sdf(m.query_sdf, torch.tensor(s), subsample_ratio=ratio)
        out[f"idx{k}"] = idx
        out[f"s{k}"] = np.float32(s)
        out[f"density{k}"] = occ.density_grid.clone()
        out[f"mask{k}"] = occ.occupancy_mask.clone()
    save("occupancy.npz", **out)


class _FixedBatch:
    """Dataset stand-in for the reference trainer: every sample_rays call returns the same batch
    and draws no random numbers, so the sampler's draws are the only ones inside a step."""

    def __init__(self, o, d, rgb):
        self.o, self.d, self.rgb = o, d, rgb
        self.test_views = []

    def sample_rays(self, batch_size):
        return {"rays_o": self.o, "rays_d": self.d, "rgb": self.rgb}


def _trainer_snapshot(prefix, model, trainer, out):
    """Parameters, gradients and both optimizers' Adam moments, keyed by the state_dict names."""
    named = dict(model.named_parameters())
    for k, p in named.items():
        out[f"{prefix}param/{k}"] = p.detach().clone()
        if p.grad is not None:
            out[f"{prefix}grad/{k}"] = p.grad.detach().clone()
    for opt in trainer.optimizers.values():
        for k, p in named.items():
            st = opt.state.get(p)
            if st:
                out[f"{prefix}exp_avg/{k}"] = st["exp_avg"].clone()
                out[f"{prefix}exp_avg_sq/{k}"] = st["exp_avg_sq"].clone()
                out[f"{prefix}adam_step/{k}"] = torch.tensor(float(st["step"]))


def gen_train_step(R):
    """Steps 1 and 2 of the reference's own VoxNeuSTrainer.train_step (training/trainer.py:166-393):
    render with RaySampler(64, 64, perturb=True), Huber loss, backward, V_R in the relax sphere,
    eikonal + curvature into grid.grad at the scheduler's weights, the k = 5 s amplification
    (s_warmup_steps = 0, so it is live), the cosine learning rates and the amplified variance rate,
    SparseGridAdam(0.9, 0.99) on the grid (its torch path) and Adam on the rest. Steps 1 and 2 draw
    no occupancy cells (the refresh runs at multiples of 16). The targets are the first seeded ones
    whose s gradient is negative (amplified) at step 1 and positive at step 2, so both branches of
    the rule are pinned. The sampler's uniforms of each step are regenerated from its seed and
    saved, with the z it returned. The trainer state after step 2 is also written with the
    reference's own save_checkpoint (checkpoint_step2.pt), with a deterministic render of that
    model."""
    import contextlib
    import io
    import tempfile

    from voxneus.training.checkpoint import save_checkpoint
    from voxneus.training.trainer import VoxNeuSTrainer

    n_rays, ns, ni = 32, 64, 64
    o, d = hemisphere_rays(n_rays, seed=9)
    cfg = {"training": {"total_steps": 40000, "batch_size": n_rays, "loss_type": "Huber",
                        "occupancy_update_interval": 16, "progressive_hash": False, "save_interval": 10 ** 9},
           "sampler": {"n_samples": ns, "n_importance": ni, "perturb": True, "up_sample_steps": 4},
           "scheduler": {"s_warmup_steps": 0, "s_amplification_k": 5.0},
           "optimizer": {"lr_sdf": 0.1, "lr_hash": 0.01, "lr_mlp": 0.001, "lr_variance": 0.0005},
           "model": {}, "logging": {"dashboard_interval": 10 ** 9, "print_interval": 10 ** 9}}

    def build(target_seed):
        torch.manual_seed(8)
        model = R["VoxNeuS"](grid_res=20, hash_n_levels=16, hash_log2_size=7, occupancy_res=8, force_pytorch=True)
        with torch.no_grad():
            model.sdf_grid.grid.add_(torch.randn_like(model.sdf_grid.grid) * 0.01)
            model.radiance_hash.encoder.embeddings.uniform_(-0.5, 0.5)
            model.occupancy_grid.occupancy_mask.copy_(torch.rand(8, 8, 8) > 0.3)
        tgt = torch.rand(n_rays, 3, generator=torch.Generator().manual_seed(target_seed))
        tr = VoxNeuSTrainer(model, _FixedBatch(o, d, tgt), cfg, output_dir=tempfile.mkdtemp(prefix="vx_golden_"),
                            device=torch.device("cpu"))
        return model, tr, tgt

    def run(model, tr, out, steps=(1, 2)):
        _trainer_snapshot("init/", model, tr, out)
        seen = {}
        sample = tr.sampler.sample_multistep_sdf

        def recording(*args, **kw):  # keeps the sampler's z of the step (behaviour unchanged)
            r = sample(*args, **kw)
            seen["z"] = r[0].detach().clone()
            return r

        tr.sampler.sample_multistep_sdf = recording
        for k in steps:
            torch.manual_seed(100 + k)
            out[f"step{k}/t_rand"] = torch.rand(n_rays, ns)
            out[f"step{k}/us"] = torch.stack([torch.rand(n_rays, ni // 4) for _ in range(4)])
            torch.manual_seed(100 + k)
            met = tr.train_step(k)
            for key in ("loss_rgb", "loss_eik", "loss_curv", "w_eik", "w_curv", "lr_hash", "lr_mlp", "lr_s"):
                out[f"step{k}/{key}"] = torch.tensor(float(met[key]), dtype=torch.float64)
            out[f"step{k}/s_amplified"] = torch.tensor(bool(met["s_amplified"]))
            out[f"step{k}/z"] = seen["z"]
            _trainer_snapshot(f"step{k}/", model, tr, out)

    for seed in range(64):  # the first target whose s gradient is negative at step 1 and positive at step 2
        model, tr, tgt = build(seed)
        out = {"rays_o": o, "rays_d": d, "target": tgt, "occupancy": model.occupancy_grid.occupancy_mask.clone(),
               "target_seed": torch.tensor(seed)}
        with contextlib.redirect_stdout(io.StringIO()):
            run(model, tr, out)
        if bool(out["step1/s_amplified"]) and not bool(out["step2/s_amplified"]):
            break
    else:
        raise RuntimeError("no target seed gives both s-gradient signs")
    save("train_step.npz", **out)
    path = os.path.join(HERE, "checkpoint_step2.pt")
    save_checkpoint(path, 2, model, tr.optimizers, {"note": "golden fixture"},
                    {"loss_rgb": float(out["step2/loss_rgb"])})
    ro, rd = hemisphere_rays(16, seed=21)
    near, far = R["rays"].near_far_from_sphere(ro, rd, radius=1.0)
    with torch.no_grad():
        rend = model.render(ro, rd, R["sampler"].RaySampler(n_samples=ns, n_importance=ni, perturb=False), near, far,
                            up_sample_steps=4, sphere_radius=1.0)
    save("checkpoint_render.npz", rays_o=ro, rays_d=rd, rgb=rend["rgb"], depth=rend["depth"], normal=rend["normal"],
         opacity=rend["opacity"])
    print(f"wrote checkpoint_step2.pt ({os.path.getsize(path)} bytes)")


GENERATORS = {
    "field_query": gen_field_query,
    "sampler": gen_sampler,
    "render_det": lambda R: gen_render(R, perturb=False, name="render_det.npz"),
    "render_perturb": lambda R: gen_render(R, perturb=True, name="render_perturb.npz"),
    # the throughput workload's sampler: 64 stratified + 4 x 16 upsampled = 128 samples per ray
    "render_128": lambda R: gen_render(R, perturb=True, name="render_128.npz", n_samples=64, n_importance=64,
                                       grid_res=20, hash_log2=7, n_rays=24),
    "train_step": gen_train_step,
    "regularizers": gen_regularizers,
    "upsample": gen_upsample,
    "hash": gen_hash,
    "alpha": gen_alpha,
    "occupancy": gen_occupancy,
}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default=os.environ.get("VOXNEUS_REFERENCE"),
                    help="the reference's Code/ directory (default: $VOXNEUS_REFERENCE)")
    ap.add_argument("--only", nargs="*", choices=sorted(GENERATORS), help="fixtures to write (default: all)")
    args = ap.parse_args()
    if not args.reference:
        ap.error("give --reference <reference>/Code or set VOXNEUS_REFERENCE")
    torch.set_num_threads(1)
    R = _import_reference(args.reference)
    for name in args.only or list(GENERATORS):
        GENERATORS[name](R)


if __name__ == "__main__":
    main()

"""Training-step throughput of the fused VoxNeuS hot path on B200 (one JSON line on rank 0).

Workload (the throughput configuration): 256^3 FP32 SDF grid, upsampled on the device from a
128^3 union of 8 random spheres/boxes + N(0, 0.005) noise; 8192 rays per step per GPU from 64
hemisphere cameras at 800x600 (focal 700 px); 64 stratified + 4 x 16 upsampled samples per ray
(perturbed); appearance 16-level hash grid (2 features, 2^19 entries) + 64-wide MLP; V_R =
render corners within the 1.2 relax sphere and the |f| < 3 voxel narrow band; eikonal 0.1,
curvature 5e-4; Huber loss on U[0,1] targets; optimizer steps included. A step is one full
training iteration over one ray batch.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

--impl reference times the oracle (a CPU restatement of the reference's own PyTorch path) on
the host cores, all threads, on bounded ray samples of the same workload.
"""

from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

import torch

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "fwd+bwd rays/s at 256^3 grid (fused training step)"
UNIT = "rays/s"
N_SAMPLES, N_IMPORTANCE, STEPS_UP = 64, 64, 4
CPU_SAMPLE_RAYS = 1024
# the timed steps are numbered from here: past the trainer's s_warmup_steps (5000), so the k = 5
# s-gradient amplification and its variance learning-rate rule are live, as in 35k of the 40k steps;
# a multiple of the 16-step occupancy refresh, so the first warm-up step refreshes the mask as a
# run's first step does
STEP0 = 5008


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="fused", choices=["fused", "reference"])
    ap.add_argument("--rays", type=int, default=8192)
    ap.add_argument("--res", type=int, default=256)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--eager", action="store_true", help="train: launch every kernel from the host (no CUDA graph)")
    ap.add_argument("--workload", default="train", choices=["train", "field", "serving"],
                    help="train (the metric line), field (512^3 queries), serving (the request mix)")
    ap.add_argument("--duration", type=float, default=10.0, help="serving: seconds of arrivals")
    ap.add_argument("--no-extras", action="store_true",
                    help="train: skip the field-query and short serving-mix summaries of the default line")
    ap.add_argument("--extras-duration", type=float, default=3.0, help="train: seconds of the serving mix summary")
    return ap.parse_args()


def config(args, world):
    return {"workload": "training step, 256^3 grid from 128^3 shapes, 8192 rays x (64+4x16) samples per GPU",
            "grid": args.res, "rays_per_gpu": args.rays, "global_rays": args.rays * world,
            "samples_per_ray": N_SAMPLES + N_IMPORTANCE, "hash": "16 levels x 2 x 2^19", "mlp": "51-64-3",
            "band_voxels": 3, "w_eik": 0.1, "w_curv": 5e-4, "perturb": True, "optimizer_step": True,
            "steps_from": STEP0, "s_amplification": "live (k = 5, steps past the 5000-step warm-up)",
            "parallelism": f"dp{world}" if world > 1 else "single",
            "l2": "working set (grid, hash table, grads, Adam state > 700 MiB) exceeds the 126 MB L2"}


def make_scene(res, device, seed=0):
    from voxneus_b200 import synthetic

    return synthetic.throughput_scene(res, device, seed=seed)


class ClockSampler:
    """SM clock, max clock, power and clock-event reasons sampled during the timed region: NVML
    read every 5 ms from a thread (one sample taken on entry and one on exit, so a region shorter
    than the period still has samples); `nvidia-smi -lms 50` when NVML is not importable."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")
    NAMES = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")

    def __init__(self, index: int, period_s: float = 0.005):
        self.index = index
        self.period = period_s
        self.proc = None
        self.nvml = None
        self.samples = []  # (sm_mhz, max_mhz, reasons set)

    def _nvml_sample(self):
        nv, h = self.nvml, self.handle
        sm = nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)
        mx = nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM)
        bits = nv.nvmlDeviceGetCurrentClocksEventReasons(h)
        masks = (nv.nvmlClocksEventReasonHwSlowdown, nv.nvmlClocksEventReasonHwThermalSlowdown,
                 nv.nvmlClocksEventReasonSwThermalSlowdown, nv.nvmlClocksEventReasonSwPowerCap)
        self.samples.append((float(sm), float(mx), {nm for nm, m in zip(self.NAMES, masks) if bits & m}))

    def _loop(self):
        while not self._stop.wait(self.period):
            try:
                self._nvml_sample()
            except Exception:  # a failed read only loses that sample
                pass

    def __enter__(self):
        try:
            import pynvml

            pynvml.nvmlInit()
            self.nvml = pynvml
            self.handle = self._nvml_handle(pynvml)
            self._nvml_sample()
            self._stop = threading.Event()
            self._thread = threading.Thread(target=self._loop, daemon=True)
            self._thread.start()
            return self
        except Exception:
            self.nvml = None
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "50"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
        return self

    def _nvml_handle(self, nv):
        """NVML enumerates every GPU of the machine: find this process's CUDA device by PCI address."""
        pr = torch.cuda.get_device_properties(self.index)
        bus = f"{pr.pci_domain_id:08X}:{pr.pci_bus_id:02X}:{pr.pci_device_id:02X}.0"
        return nv.nvmlDeviceGetHandleByPciBusId(bus)

    def __exit__(self, *exc):
        if self.nvml is not None:
            self._stop.set()
            self._thread.join(timeout=2)
            try:
                self._nvml_sample()
                self.nvml.nvmlShutdown()
            except Exception:
                pass
            return
        if self.proc is not None:
            self.proc.terminate()
            try:
                out, _ = self.proc.communicate(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
                out, _ = self.proc.communicate()
            for ln in out.splitlines():
                parts = [p.strip() for p in ln.split(",")]
                if len(parts) < 8:
                    continue
                try:
                    sm, mx = float(parts[0]), float(parts[1])
                except ValueError:
                    continue
                self.samples.append((sm, mx, {nm for nm, v in zip(self.NAMES, parts[4:8])
                                              if v.lower().startswith("active")}))

    def summary(self):
        sm = [x[0] for x in self.samples]
        mx = self.samples[-1][1] if self.samples else None
        reasons = set().union(*[x[2] for x in self.samples]) if self.samples else set()
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm), "source": "nvml" if self.nvml is not None else "nvidia-smi"}


def peak_hbm():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


def algorithmic_bytes(name, n_rays, n_samples, res, n_levels=16, ld=52, nnz=None):
    """Logical global-memory bytes of one launch (each operand counted once; no cache credit)."""
    P = n_rays * n_samples
    per = N_IMPORTANCE // STEPS_UP
    q = N_SAMPLES + (STEPS_UP - 1) * per
    occ = sum(N_SAMPLES + k * per - 1 for k in range(STEPS_UP))
    voxels = res ** 3
    table = {
        "vx_sample_multistep": n_rays * (24 + 4 * N_SAMPLES + 4 * N_IMPORTANCE + 32 * q + occ + 8 * n_samples),
        "vx_render_geometry_forward": n_rays * 24 + P * (4 + 128 + 4 + 12 + 4),
        "vx_appearance_forward": n_rays * 24 + P * (4 + n_levels * 8 * 8 + 12 + 4 * ld),
        # fused appearance + MLP: the ray, midpoint, the hash gathers (16 levels x 8 corners x 2
        # features) and the normal in, colours out. The compact rows this design keeps for the
        # adjoint (144 B a sample, written and read back) are its own cache, not algorithmic bytes:
        # they show in the DRAM traffic reported beside the figure.
        "vx_appearance_mlp_forward": n_rays * 24 + P * (4 + n_levels * 8 * 8 + 12 + 12),
        "vx_composite_forward": n_rays * (24 + 32) + P * 48,
        "vx_composite_backward": n_rays * (24 + 32) + P * 64,
        "vx_hash_encode_backward": n_rays * 24 + P * (4 + 4 * 2 * n_levels + n_levels * 8 * 16),
        "vx_render_geometry_backward": n_rays * 24 + P * (4 + 4 + 12 + 12 + 128 + 256),
        "vx_vr_count": voxels // 8,
        "vx_reg_stencil": voxels * 12 + voxels // 8,
    }
    if nnz is not None:
        table["vx_masked_adam_upd"] = voxels * 4 + nnz * 24
    return table.get(name)


# FP32 FLOPs per sample of the MLP kernels (51 -> 64 ReLU -> 3 Sigmoid; the 52nd input column is padding)
MLP_FLOPS = {
    # hidden layer 2*52*64 + colour layer 2*64*3
    "vx_appearance_mlp_forward": 2 * 52 * 64 + 2 * 64 * 3,
    # hidden recompute (the colours come from the forward), dL/dh 2*3*64, dW1 2*3*64, dW0 (+db0)
    # 2*52*64, dX (35 columns) 2*64*35
    "vx_radiance_mlp_backward": 2 * 52 * 64 + 2 * 3 * 64 * 2 + 2 * 52 * 64 + 2 * 64 * 35,
    # the same adjoint on the compact rows (SH(d) recomputed from the ray direction: ~40 FLOPs, not counted)
    "vx_appearance_mlp_backward": 2 * 52 * 64 + 2 * 3 * 64 * 2 + 2 * 52 * 64 + 2 * 64 * 35,
}


def mlp_tensor(per_kernel, n_points):
    """FLOP rate of the MLP kernels: FP32-equivalent, and the tf32 tensor-core rate they issue (three
    tf32 products per FP32 product, hi*hi + hi*lo + lo*hi) against the dense tf32 peak, taken as half
    the measured bf16 GEMM peak (MEASURED_PEAKS.json)."""
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            bf16, kind = float(json.load(f)["bf16_tflops"]), "measured bf16 / 2"
    except (OSError, KeyError, ValueError):
        bf16, kind = 1590.0, "fallback bf16 / 2"
    out = {"peak_tf32_tflops": bf16 / 2, "peak_kind": kind}
    for k, fl in MLP_FLOPS.items():
        if k in per_kernel and per_kernel[k] > 0:
            tf = n_points * fl / (per_kernel[k] / 1e3) / 1e12
            out[k] = {"fp32_flops_per_sample": fl, "fp32_equiv_tflops": tf, "tf32_issued_tflops": 3 * tf,
                      "frac": 3 * tf / (bf16 / 2)}
    return out


def load_traffic():
    p = os.path.join(ROOT, "profiles", "ncu_traffic.json")
    try:
        with open(p) as f:
            return json.load(f)
    except (OSError, ValueError):
        return {}


def cpu_baseline(args, n_rays=CPU_SAMPLE_RAYS, steps=3):
    """The oracle's training step on the host cores (bounded sample of the same workload)."""
    threads = torch.get_num_threads()
    torch.set_num_threads(os.cpu_count() or 1)
    try:
        return _cpu_baseline(args, n_rays, steps)
    finally:  # every host thread busy in later legs (the serving engine) would contend with its thread
        torch.set_num_threads(threads)


def _cpu_baseline(args, n_rays, steps):
    from oracle import reference_path as O
    from voxneus_b200 import synthetic

    torch.manual_seed(0)
    g128 = synthetic.shapes_grid(args.res // 2, seed=0)
    grid = O.upsample_grid(g128, args.res).clone().requires_grad_(True)
    emb = (torch.rand(16, 2 ** 19, 2) * 2e-2 - 1e-2).requires_grad_(True)
    l0 = torch.nn.Linear(51, 64)
    l1 = torch.nn.Linear(64, 3)
    sc = O.OracleScene(grid, torch.tensor(0.3, requires_grad=True), emb, l0.weight.detach().clone().requires_grad_(True),
                       l0.bias.detach().clone().requires_grad_(True), l1.weight.detach().clone().requires_grad_(True),
                       l1.bias.detach().clone().requires_grad_(True), occupancy=torch.ones(128, 128, 128, dtype=torch.bool))
    pool = synthetic.RayPool(seed=1)
    times = []
    for i in range(steps + 1):
        o, d = pool.sample(n_rays)
        tgt = torch.rand(n_rays, 3)
        t_rand, us = O.sampler_draws(n_rays, N_SAMPLES, N_IMPORTANCE, STEPS_UP, True)
        t0 = time.perf_counter()
        sc.train_step(o, d, tgt, band_voxels=3.0, optimize=True, n_samples=N_SAMPLES, n_importance=N_IMPORTANCE,
                      steps=STEPS_UP, perturb=True, t_rand=t_rand, us=us)
        if i > 0:
            times.append(time.perf_counter() - t0)
    med = statistics.median(times)
    return {"value": n_rays / med, "unit": UNIT, "cores": torch.get_num_threads(), "kind": "port",
            "sample": f"{n_rays} rays/step of the 256^3 workload, median of {steps} steps after 1 warm-up "
                      f"(oracle: the reference's torch ops restated, float32 on CPU)"}, med


def _oracle_scene_of(m, device, grad=True, dtype=torch.float32):
    """The oracle's scene holding copies of a fused model's parameters and occupancy mask."""
    from oracle import reference_path as O

    l0, l1 = m.radiance_mlp.net[0], m.radiance_mlp.net[2]
    ps = [t.detach().to(device, dtype).clone().requires_grad_(grad) for t in (
        m.sdf_grid.grid, m.variance_net.variance, m.radiance_hash.encoder.embeddings, l0.weight, l0.bias, l1.weight,
        l1.bias)]
    return O.OracleScene(*ps, occupancy=m.occupancy_grid.occupancy_mask.detach().to(device).clone())


def parity_leg(m, batch, dev, n_rays=CPU_SAMPLE_RAYS):
    """The timed step's numbers against the oracle's (the checker, on the host cores) on a
    n_rays slice of a timed batch, with the fused model's parameters after the timed steps:
    one fused training step without the optimizers (s amplification live) and the oracle's step
    on the samples the fused sampler drew, plus the end-to-end sampler agreement."""
    from oracle import reference_path as O
    from voxneus_b200 import ops
    from voxneus_b200.rendering import RaySampler
    from voxneus_b200.training import FusedTrainer

    o, d, t = (x[:n_rays].contiguous() for x in batch)
    tr = FusedTrainer(m, RaySampler(N_SAMPLES, N_IMPORTANCE, perturb=True), band_voxels=3.0, s_warmup_steps=0,
                      optimize=False, occupancy_update_interval=0)
    gen = torch.Generator(device=dev).manual_seed(1234)
    t_rand, u = m.draw_sampler_randoms(n_rays, N_SAMPLES, N_IMPORTANCE, STEPS_UP, dev, generator=gen)
    out = tr.step(o, d, t, step=0, randoms=(t_rand, u))
    lo, hi = m.sdf_grid.bounds()
    occ = m.occupancy_grid
    z, _, _ = ops.sample_multistep(m.sdf_grid.grid.detach(), lo, hi, o, d, None, None, N_SAMPLES, N_IMPORTANCE,
                                   STEPS_UP, True, t_rand, u, occ.occupancy_mask, *occ.bounds(), want_z=True)
    torch.cuda.synchronize()
    sc = _oracle_scene_of(m, "cpu")
    oc, dc, tc = o.cpu(), d.cpu(), t.cpu()
    ref = sc.train_step(oc, dc, tc, band_voxels=3.0, amplify_k=5.0, step=0, s_warmup_steps=0, z_vals=z.cpu())
    # the same step in float64: a gradient's bound is the float32 oracle's own distance from it
    # (at least 1e-4); the variance gradient sums many cancelling terms, so float32 rounding of
    # the colours alone moves it by more than 1e-4 of its size
    sc64 = _oracle_scene_of(m, "cpu", dtype=torch.float64)
    ref64 = sc64.train_step(oc.double(), dc.double(), tc.double(), band_voxels=3.0, amplify_k=5.0, step=0,
                            s_warmup_steps=0, z_vals=z.cpu().double())
    near, far = O.near_far_from_sphere(oc, dc)
    zr, _, _ = O.sample_multistep_sdf(oc, dc, near, far, sc.sdf_fn, N_SAMPLES, N_IMPORTANCE, STEPS_UP, True, sc.occ_fn,
                                      t_rand=t_rand.cpu(), us=[u[k].cpu() for k in range(STEPS_UP)])
    zd, zrd = z.cpu().double(), zr.double()
    outside = int(((zd - zrd).abs() > 1e-5 * (zrd.abs() + float(zrd.abs().max()))).any(dim=1).sum())

    def rel(a, b):
        a, b = torch.as_tensor(a).detach().double().cpu(), torch.as_tensor(b).detach().double().cpu()
        return float((a - b).abs().max() / max(float(b.abs().max()), 1e-30))

    l0, l1 = m.radiance_mlp.net[0], m.radiance_mlp.net[2]
    gp = {"grid": m.sdf_grid.grid, "variance": m.variance_net.variance,
          "embeddings": m.radiance_hash.encoder.embeddings, "w0": l0.weight, "b0": l0.bias, "w1": l1.weight,
          "b1": l1.bias}
    grads = {k: rel(p.grad, ref["grads"][k]) for k, p in gp.items()}
    grads64 = {k: rel(p.grad, ref64["grads"][k]) for k, p in gp.items()}
    bounds = {k: max(1e-4, 2.0 * rel(ref["grads"][k], ref64["grads"][k])) for k in gp}
    losses = {k: rel(out[k], ref[k]) for k in ("loss_rgb", "loss_eik", "loss_curv")}
    amp = bool(tr.amp_flag.item())
    res = {"rays": n_rays, "loss_rel_err": losses, "grad_rel_err": grads, "grad_rel_err_vs_float64": grads64,
           "grad_bound": bounds,
           "n_active": [int(out["n_active"]), int(ref["n_active"])], "amplified": [amp, bool(ref["amplified"])],
           "sampler_rays_outside_1e-5": outside,
           "tolerance": {"loss": 1e-5, "grad": "grad_bound: max(1e-4, 2 x the float32 oracle's distance from "
                                                 "the float64 oracle)", "n_active": "equal", "amplified": "equal"},
           "how": "one training step without the optimizers on a slice of a timed batch, parameters after the "
                  "timed steps; the oracle (float32 and float64, host cores) steps on the fused sampler's "
                  "samples; sampler_rays_outside_1e-5 compares the two samplers end to end on the same uniforms"}
    res["within_tolerance"] = (max(losses.values()) <= 1e-5 and all(grads[k] <= bounds[k] for k in grads)
                               and res["n_active"][0] == res["n_active"][1] and amp == bool(ref["amplified"]))
    for p in gp.values():
        p.grad = None
    return res


def same_gpu_torch_leg(m, batches, dev, steps=3, step0=0):
    """The reference's plain PyTorch training step on this GPU: its torch ops as the oracle
    restates them (the golden-pinned checker, here the baseline being timed, never the product)
    on a copy of the fused scene, the full workload (all rays of a batch, 64 + 4 x 16 samples, the
    narrow band, both optimizers), FP32 with TF32 off. Median of `steps` CUDA-event-timed steps
    after one warm-up step."""
    from oracle import reference_path as O

    prev = torch.backends.cuda.matmul.allow_tf32, torch.backends.cudnn.allow_tf32
    torch.backends.cuda.matmul.allow_tf32 = False
    torch.backends.cudnn.allow_tf32 = False
    try:
        sc = _oracle_scene_of(m, dev)
        n = batches[0][0].shape[0]
        times = []
        for i in range(steps + 1):
            o, d, t = batches[i % len(batches)]
            t_rand, us = O.sampler_draws(n, N_SAMPLES, N_IMPORTANCE, STEPS_UP, True, device=dev)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize()
            e0.record()
            sc.train_step(o, d, t, band_voxels=3.0, amplify_k=5.0, optimize=True, step=step0 + i, n_samples=N_SAMPLES,
                          n_importance=N_IMPORTANCE, steps=STEPS_UP, perturb=True, t_rand=t_rand, us=us)
            e1.record()
            torch.cuda.synchronize()
            if i > 0:
                times.append(e0.elapsed_time(e1))
        ms = statistics.median(times)
        del sc
        torch.cuda.empty_cache()
    finally:
        torch.backends.cuda.matmul.allow_tf32, torch.backends.cudnn.allow_tf32 = prev
    return {"value": n / (ms / 1e3), "unit": UNIT, "ms_per_step": ms, "steps": steps, "warmup": 1,
            "what": "the reference's plain PyTorch training step (its torch ops as the oracle restates them, "
                    "golden-pinned) on this GPU at the full workload, FP32, TF32 off"}


def reference_kernels_leg(m, batch, dev, reps=20):
    """The reference's own CUDA kernels (voxneus/cuda/*.cu built from its sources into oracle/_ref by
    oracle/build_ref.py: the checker's second comparison point, never the product) against this
    library's drop-in entry points, on the inputs of one timed step: Eq.7 interpolation forward and
    backward at the step's 1M sample positions, eikonal and curvature on the narrow-band vertex list,
    masked Adam on the 256^3 grid. CUDA-event means over `reps` calls each."""
    from oracle import build_ref
    from voxneus_b200 import cuda as vcuda
    from voxneus_b200 import ops

    ref = build_ref.load()
    if ref is None:
        return {"unavailable": "the reference extension was not built (oracle/build_ref.py)"}

    def timed(fn):
        for _ in range(3):
            fn()
        s_, e_ = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        s_.record()
        for _ in range(reps):
            fn()
        e_.record()
        torch.cuda.synchronize()
        return s_.elapsed_time(e_) / reps

    def rel(a, b):
        a, b = a.detach().double(), b.detach().double()
        return float((a - b).abs().max() / b.abs().max().clamp_min(1e-30))

    o, d, _ = batch
    n = o.shape[0]
    gen = torch.Generator(device=dev).manual_seed(77)
    t_rand, u = m.draw_sampler_randoms(n, N_SAMPLES, N_IMPORTANCE, STEPS_UP, dev, generator=gen)
    lo, hi = m.sdf_grid.bounds()
    occ = m.occupancy_grid
    grid5 = m.sdf_grid.grid.detach()
    grid3 = grid5[0, 0].contiguous()
    res = list(grid3.shape)
    _, _, mid = ops.sample_multistep(grid5, lo, hi, o, d, None, None, N_SAMPLES, N_IMPORTANCE, STEPS_UP, True, t_rand,
                                     u, occ.occupancy_mask, *occ.bounds(), want_z=False)
    pts = (o[:, None, :] + d[:, None, :] * mid[..., None]).reshape(-1, 3)
    lo_t, hi_t = torch.tensor(lo, device=dev), torch.tensor(hi, device=dev)
    rt = torch.tensor(res, dtype=torch.float32, device=dev)
    coords = ((pts - lo_t) / (hi_t - lo_t + 1e-8) * (rt - 1.0)).contiguous()  # geometry/coordinates.py:10-29
    vs = ((hi_t - lo_t) / (rt - 1.0)).contiguous()
    out = {"points": int(coords.shape[0])}
    g_ref = ref.gradient_interp_forward(grid3, coords, vs)
    g_our = vcuda.cuda_gradient_interp(grid3, coords, vs)
    out["gradient_interp_forward"] = {"reference_ms": timed(lambda: ref.gradient_interp_forward(grid3, coords, vs)),
                                      "ours_ms": timed(lambda: ops.gradient_interp_raw(grid3, coords, vs.tolist())),
                                      "max_rel_diff": rel(g_our, g_ref)}
    gout = torch.randn(coords.shape, device=dev, generator=torch.Generator(device=dev).manual_seed(78))
    ga, gb = torch.zeros_like(grid3), torch.zeros_like(grid3)
    ref.gradient_interp_backward(gout, coords, ga, vs)
    eps = vs.tolist()
    ops.call("vx_gradient_interp_backward", ops.ptr(gout), ops.ptr(coords), coords.shape[0], ops.ptr(gb), ops.i3(res),
             ops.f3(eps), ops.stream_ptr(dev))
    out["gradient_interp_backward"] = {
        "reference_ms": timed(lambda: ref.gradient_interp_backward(gout, coords, ga, vs)),
        "ours_ms": timed(lambda: ops.call("vx_gradient_interp_backward", ops.ptr(gout), ops.ptr(coords),
                                          coords.shape[0], ops.ptr(gb), ops.i3(res), ops.f3(eps),
                                          ops.stream_ptr(dev))),
        "max_rel_diff": rel(gb, ga)}
    # the narrow band |f| < 3 voxels inside the relax sphere, as a vertex list (V_R of a dense render)
    band = float(torch.tensor(3.0 * eps[0], dtype=torch.float32))
    bm = torch.full((ops.bitmap_words(res),), -1, dtype=torch.int32, device=dev)
    counts = ops.vr_count(bm, grid5, res, lo, hi, 1.2, band)
    nv = int(ops.final_count(counts, 1.2, band))
    verts, _ = ops.vr_compact(bm, grid5, res, lo, hi, 1.2, band, counts, nv)
    out["vertices"] = nv
    for kind, rf in (("eikonal", ref.eikonal_grad), ("curvature", ref.curvature_grad)):
        ga.zero_()
        gb.zero_()
        rf(grid3, verts, ga, vs, 0.1)
        ops.reg_list(kind, grid3, verts, eps, 0.1, gb)
        out[f"{kind}_grad"] = {"reference_ms": timed(lambda: rf(grid3, verts, ga, vs, 0.1)),
                               "ours_ms": timed(lambda: ops.reg_list(kind, grid3, verts, eps, 0.1, gb)),
                               "max_rel_diff": rel(gb, ga)}
    p0 = grid3.clone()
    g = torch.randn(p0.shape, device=dev, generator=torch.Generator(device=dev).manual_seed(79))
    g = torch.where(torch.rand(p0.shape, device=dev, generator=torch.Generator(device=dev).manual_seed(80)) < 0.5, g,
                    torch.zeros_like(g))
    pa, pb = p0.clone(), p0.clone()
    ma, va, mb, vb = (torch.zeros_like(p0) for _ in range(4))
    ref.masked_adam_upd(pa, g, ma, va, 1, 0.9, 0.99, 0.1, 1e-8)
    ops.adam_update(pb, g, mb, vb, 1, 0.9, 0.99, 0.1, 1e-8, masked=True)
    out["masked_adam_upd"] = {"reference_ms": timed(lambda: ref.masked_adam_upd(pa, g, ma, va, 2, 0.9, 0.99, 0.1, 1e-8)),
                              "ours_ms": timed(lambda: ops.adam_update(pb, g, mb, vb, 2, 0.9, 0.99, 0.1, 1e-8,
                                                                       masked=True)),
                              "max_rel_diff_after_one_step": rel(pb - p0, pa - p0)}
    for v in out.values():
        if isinstance(v, dict) and v.get("reference_ms"):
            v["speedup"] = v["reference_ms"] / v["ours_ms"]
    out["what"] = ("the reference's own CUDA extension (voxneus/cuda, built from its sources for sm_100a; legacy "
                   "stream, voxel size read with .item()) against this library's drop-ins, same inputs")
    return out


# Render forward per ray, the unit of the "render kernel" target: sampler 4,444 B (112 SDF queries x
# 32 B + occupancy + z) + Eq.7 stencil 128 x 128 B + appearance hand-off 128 x 36 B + ray I/O 64 B
RENDER_BYTES_PER_RAY = 4444 + 16384 + 4608 + 64
HASH_FWD_BYTES_PER_RAY = (N_SAMPLES + N_IMPORTANCE) * 16 * 8 * 2 * 4  # 16 levels x 8 corners x 2 features
RENDER_KERNELS = ("vx_sample_multistep", "vx_render_geometry_forward", "vx_composite_forward")


def render_roofline(per_kernel, n_rays, peak, peak_kind):
    """Render-forward bytes per ray over the summed device time of its kernels (one step's
    attribution pass), without and with the appearance forward (hash gathers + MLP)."""
    ms = sum(per_kernel.get(k, 0.0) for k in RENDER_KERNELS)
    out = {"bound": "hbm", "kernels": list(RENDER_KERNELS), "bytes_per_ray": RENDER_BYTES_PER_RAY, "ms": ms,
           "peak": peak, "peak_kind": peak_kind, "unit": "GB/s"}
    if ms > 0:
        out["achieved"] = n_rays * RENDER_BYTES_PER_RAY / (ms / 1e3) / 1e9
        out["frac"] = out["achieved"] / peak
    app = per_kernel.get("vx_appearance_mlp_forward")
    if app and ms > 0:
        b = RENDER_BYTES_PER_RAY + HASH_FWD_BYTES_PER_RAY
        ach = n_rays * b / ((ms + app) / 1e3) / 1e9
        out["with_appearance"] = {"bytes_per_ray": b, "ms": ms + app, "achieved": ach, "frac": ach / peak}
    return out


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    steps = max(1, min(args.steps, 5))
    cb, med = cpu_baseline(args, CPU_SAMPLE_RAYS, steps)
    line = {"metric": METRIC, "value": cb["value"], "unit": UNIT, "n_gpus": args.gpus, "steps": steps,
            "warmup": 1, "ms_per_step": med * 1e3, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic", "impl": "reference",
            "config": config(args, 1), "cpu_baseline": cb,
            "e2e": {"value": cb["value"], "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def run_fused(args):
    from voxneus_b200 import _lib, ops
    from voxneus_b200 import synthetic
    from voxneus_b200.rendering import RaySampler
    from voxneus_b200.training import GRAPH_WARMUP_STEPS, FusedTrainer

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    exchange = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        from voxneus_b200.dataparallel import GradExchange

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=dev)
        exchange = GradExchange()
    _lib.load()
    torch.backends.cuda.matmul.allow_tf32 = False
    m, up_ms = make_scene(args.res, dev)
    tr = FusedTrainer(m, RaySampler(N_SAMPLES, N_IMPORTANCE, perturb=True), band_voxels=3.0, exchange=exchange,
                      cuda_graph=not args.eager)
    graph_mode = tr.cuda_graph  # data-parallel ranks: two graphs, the exchange eager between them
    pool = synthetic.RayPool(seed=100 + rank)
    nb = 8
    batches = []
    for _ in range(nb):
        o, d = pool.sample(args.rays)
        batches.append((o.to(dev), d.to(dev), torch.rand(args.rays, 3).to(dev)))

    def barrier():
        if world > 1:
            import torch.distributed as dist

            dist.barrier()

    # warm-up, with a per-kernel attribution pass on one eager step (the last warm-up step, or in
    # graph mode the last eager step before the capture); the capture then records CUDA events
    # around the dominant calls only
    n_warm = max(args.warmup, 3)
    attr_at = GRAPH_WARMUP_STEPS - 1 if graph_mode else n_warm - 1
    dom_timer = None
    for i in range(n_warm):
        if i == attr_at:
            timer = _lib.KernelTimer()
            _lib.set_timer(timer)
        elif graph_mode and dom_timer is not None and tr.graph() is None:
            _lib.set_timer(dom_timer)  # this step captures the graph
        o, d, t = batches[i % nb]
        tr.step(o, d, t, step=STEP0 + i)
        _lib.set_timer(None)
        if i == attr_at:
            torch.cuda.synchronize()
            per_kernel = {k: sum(v) for k, v in timer.durations_ms().items()}
            nnz = int((m.sdf_grid.grid.grad != 0).sum().item()) if m.sdf_grid.grid.grad is not None else None
            sizes = dict(n_rays=args.rays, n_samples=N_SAMPLES + N_IMPORTANCE, res=args.res, nnz=nnz)
            hbm_cands = {k: v for k, v in per_kernel.items() if algorithmic_bytes(k, **sizes) is not None}
            hbm_dom = max(hbm_cands, key=hbm_cands.get)  # the longest HBM/L2-bound call
            cands = dict(hbm_cands)
            cands.update({k: v for k, v in per_kernel.items() if k in MLP_FLOPS})
            dominant = max(cands, key=cands.get)  # the longest call overall (tensor-core MLP or HBM-bound)
            dom_timer = _lib.KernelTimer(sorted({dominant, hbm_dom}))
    torch.cuda.synchronize()
    graph_timer = GraphEventTimer(tr.graph(), dom_timer, args.steps) if graph_mode else None

    # timed region: K steps, events around the dominant calls (eager: recorded by the library's
    # timer; graph: the captured event nodes re-pointed to a fresh pair before each replay),
    # clocks sampled alongside
    l0 = _lib.launch_count()
    r0 = tr.replayed_launches
    barrier()
    torch.cuda.synchronize()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        ev0.record()
        if not graph_mode:
            dom_timer = _lib.KernelTimer(sorted({dominant, hbm_dom}))
            _lib.set_timer(dom_timer)
        for i in range(args.steps):
            o, d, t = batches[i % nb]
            if graph_timer is not None:
                graph_timer.arm(i)
            tr.step(o, d, t, step=STEP0 + n_warm + i)
        _lib.set_timer(None)
        ev1.record()
        torch.cuda.synchronize()
    barrier()
    launches = _lib.launch_count() - l0 + tr.replayed_launches - r0
    ms = ev0.elapsed_time(ev1) / args.steps
    if world > 1:
        import torch.distributed as dist

        t_ms = torch.tensor([ms], device=dev)
        dist.all_reduce(t_ms, op=dist.ReduceOp.MAX)
        ms = float(t_ms.item())
    value = args.rays * world / (ms / 1e3)
    timed = graph_timer.durations_ms() if graph_timer is not None else dom_timer.durations_ms()
    peak, peak_kind = peak_hbm()

    def hbm_roofline(name):
        d = timed[name]
        k_ms = sum(d) / len(d)
        ab = algorithmic_bytes(name, **sizes)
        ach = ab / (k_ms / 1e3) / 1e9
        return {"bound": "hbm", "kernel": name, "achieved": ach, "peak": peak, "peak_kind": peak_kind, "unit": "GB/s",
                "frac": ach / peak, "traffic": load_traffic().get(name), "algorithmic_bytes_per_launch": ab,
                "ms_per_launch": k_ms}

    def tensor_roofline(name):
        d = timed[name]
        k_ms = sum(d) / len(d)
        mt = mlp_tensor({name: k_ms}, args.rays * (N_SAMPLES + N_IMPORTANCE))
        r = mt[name]
        return {"bound": "tensor", "kernel": name, "achieved": r["tf32_issued_tflops"], "peak": mt["peak_tf32_tflops"],
                "peak_kind": mt["peak_kind"], "unit": "TFLOP/s", "frac": r["frac"],
                "traffic": load_traffic().get(name), "fp32_equiv_tflops": r["fp32_equiv_tflops"],
                "ms_per_launch": k_ms,
                "note": "tf32 products issued (3 per FP32 product: hi*hi + hi*lo + lo*hi); the kernel is "
                        "latency/issue bound at one CTA per SM, not at the tensor pipe"}

    # the dominant call's binding limit: where it has both an algorithmic byte count and tensor-core
    # FLOPs (the appearance forward: hash gathers + MLP), the bound it comes closer to
    if dominant in MLP_FLOPS and algorithmic_bytes(dominant, **sizes) is not None:
        r_t, r_h = tensor_roofline(dominant), hbm_roofline(dominant)
        roofline = r_t if r_t["frac"] >= r_h["frac"] else r_h
    else:
        roofline = tensor_roofline(dominant) if dominant in MLP_FLOPS else hbm_roofline(dominant)
    roofline_hbm = hbm_roofline(hbm_dom)

    # end to end through the public API: pinned host rays/targets handed to FusedTrainer.step
    # (which copies them to the device, in graph mode straight into the graph's input buffers),
    # every step's loss copied back to pinned host memory and read by the host one step later (as
    # a training loop logs it), so the readback does not drain the launch queue
    # each batch as one pinned (3, N, 3) tensor whose slices are the rays and targets: the step
    # copies it to the device in one transfer
    host = []
    for o, d, t in batches:
        hb = torch.stack([o, d, t]).cpu().pin_memory()
        host.append((hb[0], hb[1], hb[2]))
    slots = torch.empty(2, dtype=torch.float32).pin_memory()
    evts = [torch.cuda.Event(), torch.cuda.Event()]
    host_losses = []
    barrier()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for i in range(args.steps):
        ho, hd, ht = host[i % nb]
        out = tr.step(ho, hd, ht, step=STEP0 + n_warm + args.steps + i)
        slots[i % 2:i % 2 + 1].copy_(out["loss_rgb"].reshape(1), non_blocking=True)
        evts[i % 2].record()
        if i >= 1:
            evts[(i - 1) % 2].synchronize()
            host_losses.append(float(slots[(i - 1) % 2]))
    evts[(args.steps - 1) % 2].synchronize()
    host_losses.append(float(slots[(args.steps - 1) % 2]))
    e2e_s = (time.perf_counter() - t0) / args.steps
    if not all(math.isfinite(v) for v in host_losses):
        raise RuntimeError("non-finite training loss")
    if world > 1:
        import torch.distributed as dist

        t_e = torch.tensor([e2e_s], device=dev)
        dist.all_reduce(t_e, op=dist.ReduceOp.MAX)
        e2e_s = float(t_e.item())
    e2e = {"value": args.rays * world / e2e_s, "unit": UNIT, "h2d_bytes_per_step": args.rays * 9 * 4,
           "d2h_bytes_per_step": 4.5, "ms_per_step": e2e_s * 1e3,
           "readback": "every step's loss (4 B) to pinned host memory, read by the host one step later; the "
                       "trainer's tensor-core status word (4 B) every 8 steps"}

    if rank != 0:
        if world > 1:
            import torch.distributed as dist

            dist.destroy_process_group()
        return
    cb = parity = same_gpu = ref_kernels = None
    if world == 1 and not args.no_cpu_baseline:
        cb, _ = cpu_baseline(args)
        parity = parity_leg(m, batches[0], dev)
        same_gpu = same_gpu_torch_leg(m, batches, dev, step0=STEP0 + n_warm)
        same_gpu["fused_over_same_gpu_torch"] = value / same_gpu["value"]
        same_gpu["fused_e2e_over_same_gpu_torch"] = e2e["value"] / same_gpu["value"]
        ref_kernels = reference_kernels_leg(m, batches[0], dev)
    field = serving = None
    if world == 1 and not args.no_extras:
        del tr
        torch.cuda.empty_cache()
        field = field_summary(args)
        serving = serving_subprocess(args.extras_duration)
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded scene, rays and targets)",
            "config": config(args, world), "e2e": e2e, "gpu_launches": int(launches),
            "launch": ("eager (every kernel launched from the host)" if not graph_mode else
                       "one CUDA graph replay per step (render .. optimizer; occupancy refresh and input copies "
                       "eager)" if exchange is None else
                       "two CUDA graph replays per step (render + backward; V_R + regularizer + optimizers) with the "
                       "gradient exchange's collectives issued eagerly between them"),
            "roofline": roofline, "roofline_hbm": roofline_hbm,
            "kernels_ms_per_step": {k: round(v, 4) for k, v in sorted(per_kernel.items(), key=lambda x: -x[1])},
            "mlp_tensor": mlp_tensor(per_kernel, args.rays * (N_SAMPLES + N_IMPORTANCE)),
            "roofline_render": render_roofline(per_kernel, args.rays, peak, peak_kind),
            "grid_upsample_128_to_256_ms": up_ms, "clocks": clk.summary(), "cpu_baseline": cb,
            "same_gpu_torch": same_gpu, "parity": parity, "reference_cuda_kernels": ref_kernels,
            "field_query_512": field, "serving_mix": serving}
    print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist

        dist.destroy_process_group()


class GraphEventTimer:
    """Per-replay CUDA events around kernels inside a captured step graph.

    The capture recorded one external event pair around each timed call (the library's
    KernelTimer under capture); before replay i, `arm(i)` points those event-record nodes of the
    executable graph at the i-th fresh pair (cudaGraphExecEventRecordNodeSetEvent affects only
    later launches), so each replay's kernel time is kept, on the stream the kernel runs on."""

    def __init__(self, step_graph, captured, steps):
        from cuda.bindings import runtime as rt

        self.rt = rt
        g = rt.cudaGraph_t(init_value=step_graph.graph.raw_cuda_graph())
        self.exec = rt.cudaGraphExec_t(init_value=step_graph.graph.raw_cuda_graph_exec())
        err, _, n = rt.cudaGraphGetNodes(g, 0)
        self._check(err, "cudaGraphGetNodes")
        err, nodes, _ = rt.cudaGraphGetNodes(g, n)
        self._check(err, "cudaGraphGetNodes")
        by_event = {}
        for nd in nodes:
            err, typ = rt.cudaGraphNodeGetType(nd)
            self._check(err, "cudaGraphNodeGetType")
            if typ == rt.cudaGraphNodeType.cudaGraphNodeTypeEventRecord:
                err, ev = rt.cudaGraphEventRecordNodeGetEvent(nd)
                self._check(err, "cudaGraphEventRecordNodeGetEvent")
                by_event[int(ev)] = nd
        self.nodes = {}
        for name, pairs in captured.events.items():
            if len(pairs) != 1:
                raise RuntimeError(f"{name}: {len(pairs)} captured calls per step; the timer takes one")
            s, e = pairs[0]
            self.nodes[name] = (by_event[s.cuda_event], by_event[e.cuda_event])
        self.pairs = {name: [] for name in self.nodes}
        for name in self.nodes:
            for _ in range(steps):
                a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                a.record()  # creates the event handles
                b.record()
                self.pairs[name].append((a, b))

    def _check(self, err, what):
        if err != self.rt.cudaError_t.cudaSuccess:
            raise RuntimeError(f"{what}: {err}")

    def arm(self, i: int) -> None:
        for name, (ns, ne) in self.nodes.items():
            a, b = self.pairs[name][i]
            for nd, ev in ((ns, a), (ne, b)):
                (err,) = self.rt.cudaGraphExecEventRecordNodeSetEvent(self.exec, nd,
                                                                      self.rt.cudaEvent_t(init_value=ev.cuda_event))
                self._check(err, "cudaGraphExecEventRecordNodeSetEvent")

    def durations_ms(self):
        return {name: [a.elapsed_time(b) for a, b in pairs] for name, pairs in self.pairs.items()}


def _events():
    return torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)


def run_field(args):
    print(json.dumps(field_summary(args)), flush=True)


def field_summary(args):
    """Large-grid field query: 512^3 grid of 32 Gaussian-bump spheres; SDF + Eq.7 normal on a 320^3
    lattice and on 2^24 uniform points; the full-grid eikonal + curvature stencil (every voxel in
    V_R, deterministic gather form)."""
    from voxneus_b200 import _lib, ops, synthetic

    _lib.load()
    dev = torch.device("cuda")
    res = 512
    grid = synthetic.bumpy_spheres_grid(res, 32, seed=3, device=dev).contiguous()
    lo, hi = (-1.0, -1.0, -1.0), (1.0, 1.0, 1.0)
    peak, peak_kind = peak_hbm()
    out = {"metric": "field query points/s (512^3 grid)", "unit": "points/s", "data": "synthetic",
           "config": {"workload": "512^3 grid, 32 Gaussian-bump spheres; 320^3 lattice, 2^24 random points, "
                                  "full-grid eikonal+curvature stencil", "grid": res}, "peak_hbm_gbs": peak,
           "peak_kind": peak_kind}
    reps = max(args.steps, 3)

    def timed(fn):
        for _ in range(3):
            fn()
        s, e = _events()
        torch.cuda.synchronize()
        s.record()
        for _ in range(reps):
            fn()
        e.record()
        torch.cuda.synchronize()
        return s.elapsed_time(e) / reps

    n_lat = 320 ** 3
    ms = timed(lambda: ops.field_query_lattice(grid, lo, hi, [320] * 3, lo, hi))
    out["lattice_320"] = {"points_per_s": n_lat / (ms / 1e3), "ms": ms, "bytes_per_point": 144,
                          "achieved_gbs": n_lat * 144 / (ms / 1e3) / 1e9}
    g = torch.Generator(device=dev).manual_seed(5)
    pts = (torch.rand(1 << 24, 3, device=dev, generator=g) * 2 - 1).contiguous()
    ms = timed(lambda: ops.field_query(grid, lo, hi, pts, sdf=True, normal=True))
    out["random_2^24"] = {"points_per_s": (1 << 24) / (ms / 1e3), "ms": ms, "bytes_per_point": 156,
                          "achieved_gbs": (1 << 24) * 156 / (ms / 1e3) / 1e9}
    bm = torch.full((ops.bitmap_words([res] * 3),), -1, dtype=torch.int32, device=dev)
    fb = ops.new_filtered([res] * 3, dev)
    counts = ops.vr_count(bm, grid, [res] * 3, lo, hi, 0.0, 0.0, filtered=fb)
    gg = torch.zeros_like(grid)
    ms = timed(lambda: ops.reg_stencil(grid, fb, [res] * 3, lo, hi, 0.0, 0.0, counts, 0.1, 5e-4, gg))
    vox = res ** 3
    out["stencil_full_grid"] = {"voxels_per_s": vox / (ms / 1e3), "ms": ms, "bytes_per_voxel": 12,
                                "achieved_gbs": vox * 12 / (ms / 1e3) / 1e9, "deterministic": True}
    out["value"] = out["random_2^24"]["points_per_s"]
    del grid, pts, bm, fb, gg
    torch.cuda.empty_cache()
    return out


def serving_subprocess(duration):
    """The serving mix measured in a process of its own, as a serving deployment runs (its engine
    thread shares the interpreter with nothing else): `bench.py --workload serving`."""
    cmd = [sys.executable, os.path.abspath(__file__), "--workload", "serving", "--duration", str(duration)]
    try:
        out = subprocess.run(cmd, cwd=ROOT, stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True,
                             timeout=600)
    except subprocess.TimeoutExpired:
        return {"error": "serving subprocess timed out"}
    lines = [ln for ln in out.stdout.splitlines() if ln.startswith("{")]
    if out.returncode != 0 or not lines:
        return {"error": f"serving subprocess rc={out.returncode}: {out.stderr.strip().splitlines()[-1:]}"}
    res = json.loads(lines[-1])
    res["process"] = "separate (bench.py --workload serving)"
    return res


def run_serving(args):
    print(json.dumps(serving_summary(args, args.duration)), flush=True)


def serving_summary(args, duration):
    """Serving mix: 16 resident 256^3 scenes (own hash table and MLP each), Poisson arrivals at
    200 req/s, 50/50 renders (log-uniform 4,096-480,000 rays from random views of the 64 cameras,
    128 samples, deterministic sampler) and SDF/normal queries (log-uniform 2^16-2^22 points)."""
    import math
    import random

    from voxneus_b200 import _lib, synthetic
    from voxneus_b200.models import VoxNeuS
    from voxneus_b200.serving import Request, SceneStore, ServingEngine, latency_stats

    _lib.load()
    dev = torch.device("cuda")
    store = SceneStore(dev)
    n_scenes = 16
    for i in range(n_scenes):
        torch.manual_seed(i)
        m = VoxNeuS(grid_res=args.res // 2, occupancy_res=128).to(dev)
        with torch.no_grad():
            m.sdf_grid.grid.copy_(synthetic.shapes_grid(args.res // 2, seed=i).to(dev))
            m.radiance_hash.encoder.embeddings.uniform_(-1e-2, 1e-2)
        m.sdf_grid.scale_volume_grid(args.res)
        store.add(f"scene{i}", m)
    t0 = time.perf_counter()
    eng = ServingEngine(store)
    capture_s = time.perf_counter() - t0
    # device time of one replay of each scene-0 graph (the engine thread is idle until submissions)
    graph_ms = {}
    for (name, kind, size), gb in eng.graphs.items():
        if name != "scene0":
            continue
        with torch.cuda.stream(eng.compute):
            for _ in range(3):
                gb.graph.replay()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(eng.compute)
            for _ in range(10):
                gb.graph.replay()
            e1.record(eng.compute)
        e1.synchronize()
        ms = e0.elapsed_time(e1) / 10
        graph_ms[f"{kind}_{size}"] = {"ms": ms, ("rays_per_s" if kind == "render" else "points_per_s"): size / ms * 1e3}
    rng = random.Random(11)
    pool = synthetic.RayPool(seed=12)
    views = [pool.view(c) for c in range(0, 64, 4)]  # 16 full 800x600 views (480,000 rays each)
    views = [(o.pin_memory(), d.pin_memory()) for o, d in views]
    qpool = [(torch.rand(1 << 22, 3, generator=torch.Generator().manual_seed(k)) * 2 - 1).pin_memory()
             for k in range(4)]
    # warm-up before the measured window, as a deployed server is warmed: the largest and smallest
    # request of each kind once per scene, so that the allocator's pools and the staging ring exist
    # before the first timed arrival (first-use growth stalled the engine thread for up to a second)
    warm = []
    for i in range(n_scenes):
        for n in (480000, 4096):
            warm.append(eng.submit(Request(f"scene{i}", "render", (views[0][0][:n], views[0][1][:n]))))
        for n in (1 << 22, 1 << 16):
            warm.append(eng.submit(Request(f"scene{i}", "query", (qpool[0][:n],))))
    for r in warm:
        r.wait(600)
    torch.cuda.synchronize()
    duration = float(duration)
    rate = 200.0
    t = 0.0
    plan = []
    while True:
        t += rng.expovariate(rate)
        if t >= duration:
            break
        scene = f"scene{rng.randrange(n_scenes)}"
        if rng.random() < 0.5:
            n = int(round(math.exp(rng.uniform(math.log(4096), math.log(480000)))))
            o, d = views[rng.randrange(len(views))]
            s = rng.randrange(0, 480000 - n + 1)
            plan.append((t, Request(scene, "render", (o[s:s + n], d[s:s + n]))))
        else:
            n = int(round(math.exp(rng.uniform(math.log(1 << 16), math.log(1 << 22)))))
            q = qpool[rng.randrange(len(qpool))]
            s = rng.randrange(0, (1 << 22) - n + 1)
            plan.append((t, Request(scene, "query", (q[s:s + n],))))
    def collect():  # a client that consumes each result as it arrives (keeps host memory bounded)
        for _, r in plan:
            try:
                r.wait(600)
            except Exception:  # counted through r.error (latency_stats skips failed requests)
                pass
            r.outputs = {}

    with ClockSampler(0) as clk:
        start = time.perf_counter()
        collector = threading.Thread(target=collect, daemon=True)
        collector.start()
        for when, req in plan:
            now = time.perf_counter() - start
            if when > now:
                time.sleep(when - now)
            req.arrival = start + when
            eng.submit(req)
        collector.join()
        wall = time.perf_counter() - start
    eng.close()
    reqs = [r for _, r in plan]
    rend = [r for r in reqs if r.kind == "render"]
    qry = [r for r in reqs if r.kind == "query"]
    line = {"metric": "serving render rays/s and p50/p99 latency (16 resident 256^3 scenes, Poisson 200 req/s)",
            "value": sum(r.n for r in rend) / wall, "unit": "rays/s", "data": "synthetic",
            "config": {"workload": "16 scenes 256^3 + 2^19 hash tables; 50/50 render (4K-480K rays, 128 samples) / "
                                   "query (2^16-2^22 points); Poisson 200 req/s",
                       "duration_s": duration, "requests": len(reqs), "buckets_render": eng.RENDER_BUCKETS,
                       "buckets_query": eng.QUERY_BUCKETS, "graph_capture_s": capture_s},
            "graph_replay": graph_ms,
            "offered": {"rays_per_s": sum(r.n for r in rend) / duration, "points_per_s": sum(r.n for r in qry) / duration},
            "query_points_per_s": sum(r.n for r in qry) / wall, "wall_s": wall,
            "latency_all": latency_stats(reqs), "latency_render": latency_stats(rend),
            "latency_query": latency_stats(qry),
            # p50 over the first, middle and last third of the arrivals: a stall shows as a backlog
            # that the later thirds inherit
            "latency_p50_ms_by_third": [latency_stats(reqs[k * len(reqs) // 3:(k + 1) * len(reqs) // 3]).get("p50_ms")
                                        for k in range(3)],
            "clocks": clk.summary()}
    del eng, store, views, qpool
    torch.cuda.empty_cache()
    return line


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
    elif args.workload == "field":
        run_field(args)
    elif args.workload == "serving":
        run_serving(args)
    else:
        run_fused(args)


if __name__ == "__main__":
    main()

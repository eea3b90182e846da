"""The bench's algorithmic-byte and FLOP bookkeeping against the per-unit figures it is defined by
(the reference workload: 8192 rays, 64 + 4 x 16 samples, a 256^3 grid, 16 hash levels), on CPU.

These numbers are the numerators of every roofline fraction the bench reports, so a slip here
would misstate a kernel's efficiency without failing any kernel test.
"""

import importlib.util
import os

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _bench():
    spec = importlib.util.spec_from_file_location("bench_module", os.path.join(ROOT, "bench.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def test_render_forward_and_hash_bytes_per_ray():
    b = _bench()
    s = b.N_SAMPLES + b.N_IMPORTANCE  # 128 evaluation samples a ray
    q = b.N_SAMPLES + (b.STEPS_UP - 1) * (b.N_IMPORTANCE // b.STEPS_UP)  # 112 sampler SDF queries
    assert (s, q) == (128, 112)
    sampler = q * 32 + 348 + 512  # SDF corners, occupancy bytes, z out
    stencil = s * 128  # 32-value Eq.7 neighbourhood per sample
    handoff = s * (12 + 12 + 12)  # normal, position/direction, colour
    assert b.RENDER_BYTES_PER_RAY == sampler + stencil + handoff + 64 == 25500
    assert b.HASH_FWD_BYTES_PER_RAY == s * 16 * 8 * 2 * 4 == 131072


def test_appearance_forward_counts_no_design_buffers():
    """The fused appearance forward's algorithmic bytes: the ray, the midpoint, the 16-level hash
    gathers, the normal in and the colour out; the compact rows it keeps for the adjoint are the
    design's own buffer and are not counted."""
    b = _bench()
    n_rays, n_samples = 8192, 128
    p = n_rays * n_samples
    ab = b.algorithmic_bytes("vx_appearance_mlp_forward", n_rays, n_samples, 256)
    assert ab == n_rays * 24 + p * (4 + 16 * 8 * 8 + 12 + 12)
    assert ab == 1103298560


def test_mlp_flops_per_sample():
    b = _bench()
    fwd = 2 * 52 * 64 + 2 * 64 * 3  # hidden layer (K padded to 52) and colour layer
    bwd = 2 * 52 * 64 + 2 * 3 * 64 * 2 + 2 * 52 * 64 + 2 * 64 * 35  # Z recompute, dL/dh + dW1, dW0, dX
    assert b.MLP_FLOPS["vx_appearance_mlp_forward"] == fwd == 7040
    assert b.MLP_FLOPS["vx_appearance_mlp_backward"] == bwd == 18560

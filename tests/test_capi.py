"""CPU checks of the drop-in boundary: the library loads and exports every symbol the header declares."""

import ctypes
import os
import re

import pytest

from voxneus_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "voxneus_b200.h")


def header_symbols():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(vx_[a-z0-9_]+)\s*\(", src)))


def test_header_declares_bound_symbols():
    decl = set(header_symbols())
    bound = set(_lib.exported_symbols())
    assert decl == bound, (decl - bound, bound - decl)


def test_library_exports_every_declared_symbol():
    if not os.path.exists(_lib.library_path()):
        pytest.skip("library not built")
    lib = ctypes.CDLL(_lib.library_path())
    for name in header_symbols():
        assert hasattr(lib, name), name


def test_size_queries_without_gpu():
    if not os.path.exists(_lib.library_path()):
        pytest.skip("library not built")
    assert _lib.query("vx_vr_bitmap_words", _lib.i3([256, 256, 256])) == 256 ** 3 // 32
    # persistent stencil grid: min(tiles / 8, 4 blocks per SM on 148 SMs)
    assert _lib.query("vx_reg_stencil_blocks", _lib.i3([256, 256, 256])) == 148 * 4
    assert _lib.query("vx_reg_stencil_blocks", _lib.i3([8, 8, 32])) == 1
    # 3 loss doubles per block + one flag byte per 32x4x4 tile
    assert _lib.query("vx_reg_stencil_workspace", _lib.i3([256, 256, 256])) == 3 * 148 * 4 + 8 * 64 * 64 // 8
    assert _lib.query("vx_reg_stencil_workspace", _lib.i3([8, 8, 32])) == 3 + 1
    assert _lib.query("vx_composite_workspace_blocks", 8192) >= 1
    # occupancy update: a float value and an int32 cell per draw, each half 16-byte padded
    assert _lib.query("vx_occupancy_workspace", 524288) == 8 * 524288
    assert _lib.query("vx_occupancy_workspace", 1) == 32
    assert _lib.query("vx_occupancy_workspace", 0) == 0
    lib = _lib.load(require_cuda=False)
    assert lib.vx_version().startswith(b"voxneus_b200")


def test_invalid_arguments_are_rejected_before_launch():
    """Validation errors come back as status codes with a message, no device touched."""
    if not os.path.exists(_lib.library_path()):
        pytest.skip("library not built")
    lib = _lib.load(require_cuda=False)
    st = lib.vx_grid_upsample(None, _lib.i3([0, 4, 4]), None, _lib.i3([8, 8, 8]), None)
    assert st == 1 and b"positive" in lib.vx_last_error()
    st = lib.vx_sample_multistep(None, _lib.i3([8, 8, 8]), _lib.f3([-1] * 3), _lib.f3([1] * 3), None, None, None,
                                 None, 4, 16, 200, 4, 0, None, None, None, None, None, 0, None, None, None, None,
                                 None, None)
    assert st == 1 and b"<= 32" in lib.vx_last_error()
    # occupancy update with neither an SDF grid nor SDF values
    st = lib.vx_occupancy_update(None, None, None, None, None, 32, _lib.f3([-1] * 3), _lib.f3([1] * 3), None, None,
                                 None, 0, None, 0, 0.0, 1, 0.95, 0.01, None, None, None, 0, None, None)
    assert st == 1 and b"exactly one" in lib.vx_last_error()


def test_kernel_calls_fail_loudly_without_cuda(monkeypatch):
    """No silent fallback: without a device the ops raise."""
    import torch

    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present")
    from voxneus_b200 import ops

    with pytest.raises(RuntimeError):
        ops.near_far_from_sphere(torch.zeros(2, 3), torch.ones(2, 3))


def test_adam_step_scalar_helpers_match_the_update_formulas():
    """The host helpers behind the graph-replayed optimizer steps: torch.optim.Adam's scalars
    (lr / (1 - b1^t), 1 / sqrt(1 - b2^t), double rounded to float) and the reference formula's
    step size lr * sqrt(1 - b2^t) / (1 - b1^t) (adam_upd_kernel.cu:50, evaluated in float)."""
    import math

    import numpy as np

    from voxneus_b200 import ops

    for step in (1, 2, 7, 100, 5000, 40000):
        for b1, b2, lr in ((0.9, 0.999, 1e-2), (0.9, 0.99, 0.1), (0.9, 0.999, 5e-4 * 5.0)):
            ss, inv = ops.adam_torch_step_scalars(step, b1, b2, lr)
            f = np.float32
            lr32, b132, b232 = float(f(lr)), float(f(b1)), float(f(b2))
            assert ss == float(f(lr32 / (1.0 - b132 ** step)))
            assert inv == float(f(1.0 / math.sqrt(1.0 - b232 ** step)))
            ref = ops.adam_reference_step_size(step, b1, b2, lr)
            want = lr32 * math.sqrt(1.0 - b232 ** step) / (1.0 - b132 ** step)
            # float evaluation: 1 - b^t cancels (b^t near 1 carries ~6e-8 absolute error)
            assert abs(ref - want) <= 1e-4 * abs(want)

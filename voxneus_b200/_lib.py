"""ctypes binding of libvoxneus_b200.so (the C ABI declared in include/voxneus_b200.h).

The library is loaded lazily on first use. There is no fallback: if the library is missing or
no CUDA device is present, every kernel-backed call raises RuntimeError.
"""

from __future__ import annotations

import ctypes
import os
import threading
from typing import Optional, Sequence

import torch

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libvoxneus_b200.so")

P = ctypes.c_void_p  # device pointer / stream
I32 = ctypes.c_int
I64 = ctypes.c_int64
F32 = ctypes.c_float
HI3 = ctypes.POINTER(ctypes.c_int32)  # host int32[3]
HF3 = ctypes.POINTER(ctypes.c_float)  # host float[3]
SZ = ctypes.c_size_t

# name -> argument types; every function returns int status unless listed in _RESTYPES
_PROTOS = {
    "vx_gradient_interp_forward": [P, HI3, P, I64, HF3, P, P],
    "vx_gradient_interp_backward": [P, P, I64, P, HI3, HF3, P],
    "vx_reg_list_blocks": [I64],
    "vx_eikonal_grad": [P, HI3, P, I64, P, HF3, F32, P, I32, P, P, P],
    "vx_curvature_grad": [P, HI3, P, I64, P, HF3, F32, P, I32, P, P, P],
    "vx_adam_upd": [P, P, P, P, I64, I32, F32, F32, F32, F32, P],
    "vx_masked_adam_upd": [P, P, P, P, I64, I32, F32, F32, F32, F32, P],
    "vx_field_query": [P, HI3, HF3, HF3, P, I64, P, P, P, P, P, P],
    "vx_field_query_backward": [P, HI3, HF3, HF3, P, I64, P, P, P, P, P],
    "vx_field_query_sorted_workspace": [I64, HI3],
    "vx_field_query_sorted": [P, HI3, HF3, HF3, P, I64, P, P, P, P, I64, P],
    "vx_corners_weights": [P, I64, HI3, P, P, P],
    "vx_field_query_lattice": [P, HI3, HF3, HF3, HI3, HF3, HF3, P, P, P],
    "vx_near_far_from_sphere": [P, P, I64, F32, P, P, P],
    "vx_sample_multistep": [P, HI3, HF3, HF3, P, P, P, P, I64, I32, I32, I32, I32, P, P, P, P, P, I32, HF3, HF3,
                            P, P, P, P],
    "vx_up_sample": [P, P, P, P, I64, I32, I32, F32, P, P, P, I32, HF3, HF3, P, P],
    "vx_sample_pdf": [P, P, P, I64, I32, I32, P, P, P, P, P],
    "vx_render_geometry_forward": [P, HI3, HF3, HF3, P, P, P, I64, I32, P, P, P, P, P],
    "vx_render_geometry_backward": [P, HI3, HF3, HF3, P, P, P, I64, I32, P, P, P, I64, P, P, P, P],
    "vx_appearance_forward": [P, I32, I32, I32, HI3, HF3, P, P, P, P, I32, HF3, HF3, I64, P, I64, I32, P, I64, I32,
                              P, I32, P],
    "vx_hash_encode_backward": [P, I32, I32, I32, HI3, HF3, P, P, P, P, I32, HF3, HF3, I64, P, I64, P],
    "vx_geometry_backward_det_workspace": [I64, I32, HI3],
    "vx_render_geometry_backward_det": [P, HI3, HF3, HF3, P, P, P, I64, I32, P, P, P, I64, P, P, SZ, P],
    "vx_hash_backward_det_workspace": [I64, I32, I32],
    "vx_hash_encode_backward_det": [P, I32, I32, I32, P, P, P, P, P, P, I32, HF3, HF3, I64, P, I64, P, SZ, P],
    "vx_radiance_mlp_forward": [P, I64, I64, I32, I32, I32, P, P, P, P, P, P],
    "vx_appearance_mlp_forward": [P, I32, I32, I32, HI3, HF3, P, P, P, I32, HF3, HF3, I64, P, P, P, P, P, P, P, I64,
                                  P],
    "vx_appearance_mlp_forward_chunked": [P, I32, I32, I32, HI3, HF3, P, P, P, I32, HF3, HF3, I64, P, P, P, P, P,
                                          P, P, I64, P],
    "vx_mlp_blocks": [I64],
    "vx_mlp_partial_floats": [],
    "vx_tensor_core_timeouts": [],
    "vx_huber_loss_blocks": [I64],
    "vx_huber_loss": [P, P, I64, F32, P, P, P, I64, P],
    "vx_cat_z_vals": [P, P, P, P, I64, I32, I32, P, P, P],
    "vx_radiance_mlp_backward": [P, I64, I64, I32, I32, I32, P, P, P, P, P, P, P, P, P, P, P, P, P, I64, P],
    "vx_appearance_mlp_backward": [P, P, I32, I64, P, P, P, P, P, P, P, P, P, P, P, P, P, I64, P],
    "vx_composite_workspace_blocks": [I64],
    "vx_composite_forward": [P, P, P, P, I64, I64, P, P, P, P, P, I32, F32, F32, P, I32, I32, F32, I64, I32, P, P, P,
                             P, P, P, P, P],
    "vx_composite_backward": [P, P, P, P, I64, I64, P, P, P, P, P, I32, F32, F32, P, I32, I32, F32, I64, I32, P, P, P,
                              P, P, P, P, P, P, P, P, I32, P, P, F32, P, P],
    "vx_neus_alpha": [P, P, P, I64, I64, P, P, I32, F32, I64, I32, P, P, P, P, P, P],
    "vx_composite_weights": [P, I64, I32, P, P, P, P, P, P],
    "vx_vr_bitmap_words": [HI3],
    "vx_vr_compact_blocks": [HI3],
    "vx_vr_mark_corners": [P, I64, HI3, P, P],
    "vx_vr_count": [P, P, HI3, HF3, HF3, F32, F32, P, P, P],
    "vx_vr_compact": [P, P, HI3, HF3, HF3, F32, F32, P, P, I64, P, P, I64, P],
    "vx_vr_compact_noalloc": [P, P, HI3, HF3, HF3, F32, F32, P, P, P, I64, P],
    "vx_reg_stencil_blocks": [HI3],
    "vx_reg_stencil_workspace": [HI3],
    "vx_reg_stencil": [P, P, HI3, HF3, HF3, F32, F32, P, F32, F32, P, P, I64, P, P, P, P],
    "vx_grid_upsample": [P, HI3, P, HI3, P],
    "vx_occupancy_workspace": [I64],
    "vx_adam_torch": [P, I32, F32, F32, F32, P],
    "vx_masked_adam_torch": [P, I32, F32, F32, F32, P],
    "vx_tc_guard": [P, I64],
    "vx_adam_reference_step_size": [I32, F32, F32, F32],
    "vx_adam_torch_step_scalars": [I64, F32, F32, F32, HF3],
    "vx_masked_adam_upd_dev": [P, P, P, P, I64, P, F32, F32, F32, P],
    "vx_occupancy_points": [I32, HF3, HF3, P, P, P, I64, P, P],
    "vx_occupancy_query": [P, I32, HF3, HF3, P, I64, P, P],
    "vx_occupancy_update": [P, HI3, HF3, HF3, P, I32, HF3, HF3, P, P, P, I64, P, I32, F32, I32, F32, F32, P, P, P, I64,
                            P, P],
}
_RESTYPES = {
    "vx_last_error": ctypes.c_char_p,
    "vx_version": ctypes.c_char_p,
    "vx_launch_count": ctypes.c_uint64,
    "vx_vr_bitmap_words": I64,
    "vx_vr_compact_blocks": I64,
    "vx_reg_stencil_blocks": I64,
    "vx_reg_stencil_workspace": I64,
    "vx_occupancy_workspace": I64,
    "vx_adam_reference_step_size": ctypes.c_float,
    "vx_adam_torch_step_scalars": None,
    "vx_field_query_sorted_workspace": I64,
    "vx_geometry_backward_det_workspace": ctypes.c_size_t,
    "vx_hash_backward_det_workspace": ctypes.c_size_t,
}

_lib = None
_lock = threading.Lock()


def library_path() -> str:
    return LIB_PATH


def load(require_cuda: bool = True):
    """Load the shared library (and check a CUDA device is present when require_cuda)."""
    global _lib
    if require_cuda and not torch.cuda.is_available():
        raise RuntimeError("voxneus_b200 needs a CUDA device (B200, sm_100a); none is available")
    if _lib is not None:
        return _lib
    with _lock:
        if _lib is None:
            if not os.path.exists(LIB_PATH):
                raise RuntimeError(f"voxneus_b200: {LIB_PATH} is missing; build it with "
                                   f"`python -m voxneus_b200.build` (nvcc, sm_100a)")
            lib = ctypes.CDLL(LIB_PATH)
            for name, args in _PROTOS.items():
                fn = getattr(lib, name)
                fn.argtypes = args
                fn.restype = _RESTYPES.get(name, ctypes.c_int)
            for name in ("vx_last_error", "vx_version", "vx_launch_count"):
                fn = getattr(lib, name)
                fn.argtypes = []
                fn.restype = _RESTYPES[name]
            _lib = lib
    return _lib


def exported_symbols() -> Sequence[str]:
    return list(_PROTOS) + ["vx_last_error", "vx_version", "vx_launch_count"]


class KernelTimer:
    """CUDA events around selected entry points, recorded on the launching (current) stream.

    Under stream capture the events are recorded as external event nodes of the graph, so every
    replay re-records them (the pair then times the latest replay)."""

    def __init__(self, names=None):
        self.names = None if names is None else set(names)
        self.events = {}

    def wants(self, name: str) -> bool:
        return self.names is None or name in self.names

    def durations_ms(self):
        return {k: [s.elapsed_time(e) for s, e in v] for k, v in self.events.items()}


_timer: Optional[KernelTimer] = None


def set_timer(timer: Optional[KernelTimer]) -> None:
    global _timer
    _timer = timer


def call(name: str, *args):
    """Call an entry point; raise RuntimeError with the library's message on failure."""
    lib = load()
    fn = getattr(lib, name)
    t = _timer
    if t is not None and t.wants(name):
        ext = torch.cuda.is_current_stream_capturing()
        s = torch.cuda.Event(enable_timing=True, external=ext)
        e = torch.cuda.Event(enable_timing=True, external=ext)
        s.record()
        st = fn(*args)
        e.record()
        t.events.setdefault(name, []).append((s, e))
    else:
        st = fn(*args)
    if st != 0:
        msg = lib.vx_last_error().decode(errors="replace")
        raise RuntimeError(f"{name}: {msg}")
    return st


def query(name: str, *args):
    """Call a size-query entry point (no CUDA device needed)."""
    lib = load(require_cuda=False)
    return getattr(lib, name)(*args)


def launch_count() -> int:
    return int(load(require_cuda=False).vx_launch_count())


# ------------------------------------------------------------------ argument helpers ------


def i3(v) -> ctypes.Array:
    v = [int(x) for x in v]
    return (ctypes.c_int32 * 3)(*v)


def f3(v) -> ctypes.Array:
    v = [float(x) for x in v]
    return (ctypes.c_float * 3)(*v)


def iarr(v) -> ctypes.Array:
    v = [int(x) for x in v]
    return (ctypes.c_int32 * max(len(v), 1))(*v)


def farr(v) -> ctypes.Array:
    v = [float(x) for x in v]
    return (ctypes.c_float * max(len(v), 1))(*v)


class AdamSegment(ctypes.Structure):
    """vx_adam_segment of the C header."""

    _fields_ = [("param", ctypes.c_void_p), ("grad", ctypes.c_void_p), ("exp_avg", ctypes.c_void_p),
                ("exp_avg_sq", ctypes.c_void_p), ("n", ctypes.c_int64), ("step", ctypes.c_int64),
                ("lr", ctypes.c_float), ("step_scalars", ctypes.c_void_p), ("lr_flag", ctypes.c_void_p)]


def ptr(t: Optional[torch.Tensor]):
    return None if t is None else ctypes.c_void_p(t.data_ptr())


def stream_ptr(device=None):
    return ctypes.c_void_p(torch.cuda.current_stream(device).cuda_stream)


def check_tensor(t: torch.Tensor, name: str, dtype=torch.float32, device=None, contiguous=True):
    """TORCH_CHECK-style validation: CUDA, dtype and contiguity (voxneus/cuda/adam_upd.cpp:44-46)."""
    if not isinstance(t, torch.Tensor):
        raise RuntimeError(f"{name} must be a tensor")
    if not t.is_cuda:
        raise RuntimeError(f"{name} must be a CUDA tensor")
    if t.dtype != dtype:
        raise RuntimeError(f"{name} must be {dtype}, got {t.dtype}")
    if device is not None and t.device != device:
        raise RuntimeError(f"{name} is on {t.device}, expected {device}")
    if contiguous and not t.is_contiguous():
        raise RuntimeError(f"{name} must be contiguous")
    return t

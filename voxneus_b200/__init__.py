"""voxneus_b200: the VoxNeuS geometry-and-rendering hot path on NVIDIA B200 (sm_100a).

Kernels live in libvoxneus_b200.so (C ABI, include/voxneus_b200.h); this package is the
host-side mirror of the reference's module API (voxneus.geometry / models / rendering /
regularization / training / cuda). Build the library with `python -m voxneus_b200.build`.
"""

from . import _lib  # noqa: F401

__all__ = ["geometry", "models", "rendering", "regularization", "training", "cuda", "ops"]

"""Test infrastructure: the CPU oracle for the VoxNeuS geometry-and-rendering hot path.

This package is a restatement, in plain PyTorch tensor ops, of the reference algorithm
(rishidevde/VoxNeus, ``Code/voxneus``). Every function cites the reference file:line it
follows. It is the checker, never the product: only ``tests/``, ``__graft_entry__.smoke()``
and the CPU-baseline legs of ``bench.py`` import it. The product path
(``voxneus_b200``) never imports it and fails loudly when its CUDA library is missing.

Parity pin: the oracle is checked against golden vectors produced by the reference itself
(``tests/golden/make_golden.py`` imports the reference and writes ``tests/golden/*.npz``),
and against the known-answer tests in the reference's own test suite.
"""

from . import reference_path  # noqa: F401

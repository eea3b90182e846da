"""The allocation-free V_R compaction entry point against the scratch-taking one.

vx_vr_compact_noalloc serves callers that cannot allocate device memory when they call in
(embedders whose device memory belongs to another runtime's pool, plugin hosts that forbid
allocation after start-up): its block scratch is a fixed device array inside the library. This
file checks, through the C ABI, that two consecutive calls return exactly the vertex list of
vx_vr_compact (the count pass of every call rewrites each block offset its write pass reads, so
nothing carries over between calls), that the largest grid the array covers (512^3, 4096
compaction blocks) is accepted and matches too, and that a grid one z-layer larger is rejected
before any launch. It is named to be collected last and passes alone in a fresh process as well
as after the others.
"""


import pytest
import torch

pytestmark = pytest.mark.gpu


def _compact_both(lib, L, ops, corners, res, grid, relax, band):
    dev = corners.device
    bm = ops.new_bitmap(res, dev)
    ops.vr_mark_corners(corners, res, bm)
    lo, hi = (-1.0, -1.0, -1.0), (1.0, 1.0, 1.0)
    counts = ops.vr_count(bm, grid, res, lo, hi, relax, band)
    n = int(ops.final_count(counts, relax, band))
    stream = L.stream_ptr(dev)
    # scratch-taking entry point, caller-owned block scratch
    nb = int(L.query("vx_vr_compact_blocks", L.i3(res)))
    scratch = torch.zeros(nb, dtype=torch.int32, device=dev)
    v_ref = torch.full((n, 3), -1, dtype=torch.int64, device=dev)
    l_ref = torch.full((n,), -1, dtype=torch.int64, device=dev)
    st = lib.vx_vr_compact(L.ptr(bm), L.ptr(grid), L.i3(res), L.f3(lo), L.f3(hi), relax, band, L.ptr(counts),
                           L.ptr(scratch), nb, L.ptr(v_ref), L.ptr(l_ref), n, stream)
    assert st == 0, lib.vx_last_error()
    # allocation-free entry point
    v = torch.full((n, 3), -2, dtype=torch.int64, device=dev)
    lin = torch.full((n,), -2, dtype=torch.int64, device=dev)
    st = lib.vx_vr_compact_noalloc(L.ptr(bm), L.ptr(grid), L.i3(res), L.f3(lo), L.f3(hi), relax, band,
                                   L.ptr(counts), L.ptr(v), L.ptr(lin), n, stream)
    assert st == 0, lib.vx_last_error()
    torch.cuda.synchronize()
    return v, lin, v_ref, l_ref, n


def test_noalloc_compaction_matches_scratch_entry_point_twice():
    from voxneus_b200 import _lib as L
    from voxneus_b200 import ops

    lib = L.load()
    dev = torch.device("cuda")
    torch.manual_seed(21)
    res = [96, 80, 112]
    axes = [torch.linspace(-1, 1, r) for r in res]
    gx, gy, gz = torch.meshgrid(*axes, indexing="ij")
    grid = (torch.sqrt(gx ** 2 + gy ** 2 + gz ** 2) - 0.5).reshape(1, 1, *res).to(dev)
    band = float(torch.tensor(3.0 * 2.0 / 95.0, dtype=torch.float32))
    first = torch.stack([torch.randint(0, r, (200000,)) for r in res], -1).to(dev)
    # second call: another set, on the radius-0.5 shell, so the narrow band keeps some of it
    dirs = torch.nn.functional.normalize(torch.randn(5000, 3), dim=-1) * 0.5
    second = torch.stack([((dirs[:, a] + 1.0) * 0.5 * (res[a] - 1)).round().long() for a in range(3)], -1).to(dev)
    for corners, relax, bnd in ((first, 1.2, 0.0), (second, 1.2, band)):
        v, lin, v_ref, l_ref, n = _compact_both(lib, L, ops, corners, res, grid, relax, bnd)
        assert n > 0
        assert torch.equal(v, v_ref) and torch.equal(lin, l_ref)
        assert bool((lin[1:] > lin[:-1]).all())  # ascending, like torch.unique


def test_noalloc_at_its_largest_grid():
    """512^3 needs exactly the array's 4096 compaction blocks (no SDF grid is read without a band)."""
    from voxneus_b200 import _lib as L
    from voxneus_b200 import ops

    lib = L.load()
    dev = torch.device("cuda")
    res = [512, 512, 512]
    assert int(L.query("vx_vr_compact_blocks", L.i3(res))) == 4096
    torch.manual_seed(5)
    corners = torch.stack([torch.randint(0, r, (300000,)) for r in res], -1).to(dev)
    v, lin, v_ref, l_ref, n = _compact_both(lib, L, ops, corners, res, None, 1.2, 0.0)
    assert n > 0 and torch.equal(v, v_ref) and torch.equal(lin, l_ref)


@pytest.mark.parametrize("res", [[512, 512, 513], [1024, 1024, 1024]])
def test_noalloc_rejects_grids_beyond_its_scratch(res):
    from voxneus_b200 import _lib as L

    lib = L.load()
    assert int(L.query("vx_vr_compact_blocks", L.i3(res))) > 4096
    dummy = torch.zeros(16, dtype=torch.int32, device="cuda")
    counts = torch.zeros(4, dtype=torch.int64, device="cuda")
    before = L.launch_count()
    st = lib.vx_vr_compact_noalloc(L.ptr(dummy), None, L.i3(res), L.f3([-1] * 3), L.f3([1] * 3),
                                   0.0, 0.0, L.ptr(counts), None, None, 0, L.stream_ptr())
    assert st == 1  # VX_ERR_INVALID
    assert b"2^27" in lib.vx_last_error()
    assert L.launch_count() == before  # rejected before any launch

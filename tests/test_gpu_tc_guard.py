"""A tensor-core wait that runs out is reported, not swallowed.

The MLP kernels wait on their MMAs and bulk copies with bounded mbarrier polls. `ops.tc_guard`
(vx_tc_guard) sets the poll limit and a device status word for the launches of this thread; a
limit of 0 polls makes every first wait give up at once. Each block that gives up lets the
MMA or copy it waited for finish (bounded), frees its tensor memory, increments the status word
and leaves: no fault, trap or hang, and the context stays usable (a default-limit call right
after gives the reference numbers). The training step raises one step later (the status is read
without a synchronisation) and the serving engine fails the request and stops.
"""

import pytest
import torch

pytestmark = pytest.mark.gpu

DEV = torch.device("cuda", 0)


@pytest.fixture(autouse=True)
def _lib_loaded():
    from voxneus_b200 import _lib

    _lib.load()
    yield
    _lib.query("vx_tensor_core_timeouts")  # reset the library's diagnostic counter for later tests


def _mlp_inputs(p, ld):
    torch.manual_seed(3)
    wide = torch.zeros(p, ld, device=DEV)
    wide[:, :51] = torch.randn(p, 51, device=DEV)
    l0, l1 = torch.nn.Linear(51, 64).to(DEV), torch.nn.Linear(64, 3).to(DEV)
    ws = [t.detach() for t in (l0.weight, l0.bias, l1.weight, l1.bias)]
    return wide[:, :51], ws  # 51 input columns at a row stride of ld floats


@pytest.mark.parametrize("ld", [52, 56], ids=["bulk-copy kernels", "register-prefetch kernels"])
def test_zero_poll_limit_sets_the_status_and_leaves_the_context_usable(ld):
    from voxneus_b200 import _lib, ops

    p = 128 * 148 * 2 + 77
    rows, ws = _mlp_inputs(p, ld)
    cot = torch.randn(p, 3, device=DEV)
    good = ops.mlp_forward(rows, *ws)
    gb = ops.mlp_backward(rows, *ws, cot, good)
    torch.cuda.synchronize()
    status = torch.zeros(1, dtype=torch.int32, device=DEV)
    with ops.tc_guard(status, 0):
        ops.mlp_forward(rows, *ws)
        ops.mlp_backward(rows, *ws, cot, good)
    torch.cuda.synchronize()
    n = int(status.item())
    assert n > 0, "no block reported the wait it gave up"
    assert _lib.query("vx_tensor_core_timeouts") == n
    # the same calls with the default limit: correct again, the status word untouched
    with ops.tc_guard(status):
        out = ops.mlp_forward(rows, *ws)
        b = ops.mlp_backward(rows, *ws, cot, good)
    torch.cuda.synchronize()
    assert int(status.item()) == n
    assert torch.equal(out, good)
    for x, y in zip(b, gb):
        assert torch.equal(x, y)


def test_zero_poll_limit_in_the_fused_appearance_forward():
    """The inference kernel that builds its features in shared memory (no rows kept)."""
    from voxneus_b200 import ops
    from voxneus_b200.models import VoxNeuS
    from voxneus_b200.rendering import RaySampler

    torch.manual_seed(1)
    m = VoxNeuS(grid_res=24, hash_log2_size=10, occupancy_res=8).to(DEV)
    o = torch.tensor([[0.0, 0.0, 3.0]], device=DEV).repeat(512, 1)
    d = torch.nn.functional.normalize(torch.tensor([[0.0, 0.0, -1.0]], device=DEV) +
                                      0.1 * torch.randn(512, 3, device=DEV), dim=-1)
    with torch.no_grad():
        ref = m.render(o, d, RaySampler(64, 64, perturb=False), None, None, extras=False)["rgb"]
        status = torch.zeros(1, dtype=torch.int32, device=DEV)
        with ops.tc_guard(status, 0):
            m.render(o, d, RaySampler(64, 64, perturb=False), None, None, extras=False)
        torch.cuda.synchronize()
        assert int(status.item()) > 0
        again = m.render(o, d, RaySampler(64, 64, perturb=False), None, None, extras=False)["rgb"]
    assert torch.equal(again, ref)


def test_training_step_raises_a_step_later():
    from voxneus_b200.models import VoxNeuS
    from voxneus_b200.rendering import RaySampler
    from voxneus_b200.training import FusedTrainer

    torch.manual_seed(2)
    m = VoxNeuS(grid_res=24, hash_log2_size=10, occupancy_res=8).to(DEV)
    o = torch.randn(256, 3)
    o = (3.0 * o / o.norm(dim=-1, keepdim=True)).to(DEV)
    d = torch.nn.functional.normalize(-o + 0.2 * torch.randn(256, 3, device=DEV), dim=-1)
    t = torch.rand(256, 3, device=DEV)
    tr = FusedTrainer(m, RaySampler(16, 16, perturb=False), optimize=False, tc_wait_polls=0, tc_check_every=1)
    out = tr.step(o, d, t, step=1)
    torch.cuda.synchronize()
    assert int(out["tc_status"].item()) > 0
    with pytest.raises(RuntimeError, match="gave up waiting on the tensor core"):
        tr.step(o, d, t, step=2)
    ok = FusedTrainer(m, RaySampler(16, 16, perturb=False), optimize=False)
    out = ok.step(o, d, t, step=1)
    ok.step(o, d, t, step=2)
    torch.cuda.synchronize()
    assert int(out["tc_status"].item()) == 0 and torch.isfinite(out["loss_rgb"])


def test_serving_engine_fails_the_request_and_stops():
    from voxneus_b200.models import VoxNeuS
    from voxneus_b200.serving import Request, RequestError, SceneStore, ServingEngine

    torch.manual_seed(4)
    store = SceneStore(DEV)
    store.add("s", VoxNeuS(grid_res=24, hash_log2_size=10, occupancy_res=8))
    eng = ServingEngine(store, render_buckets=(256,), query_buckets=(1024,), tc_wait_polls=0)
    try:
        o = torch.tensor([[0.0, 0.0, 3.0]]).repeat(300, 1)
        d = torch.tensor([[0.0, 0.0, -1.0]]).repeat(300, 1)
        req = eng.submit(Request("s", "render", (o, d)))
        with pytest.raises(RequestError, match="gave up waiting on the tensor core"):
            req.wait(60)
        assert eng.failed
    finally:
        eng.close()

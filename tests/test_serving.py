"""Serving loop: results alone and in a mix, and host-side failure handling (no GPU fault is made)."""

import time

import pytest
import torch

pytestmark = pytest.mark.gpu


def _store(n_scenes=3, res=48):
    from voxneus_b200 import synthetic
    from voxneus_b200.models import VoxNeuS
    from voxneus_b200.serving import SceneStore

    store = SceneStore("cuda")
    for i in range(n_scenes):
        torch.manual_seed(i)
        m = VoxNeuS(grid_res=res, hash_log2_size=14, occupancy_res=32)
        with torch.no_grad():
            m.sdf_grid.grid.copy_(synthetic.shapes_grid(res, seed=i))
            m.radiance_hash.encoder.embeddings.uniform_(-0.3, 0.3)
        store.add(f"s{i}", m)
    return store


def _engine(store, **kw):
    from voxneus_b200.serving import ServingEngine

    return ServingEngine(store, render_buckets=(512, 2048), query_buckets=(4096, 16384), **kw)


def _render_req(scene, n, seed):
    from voxneus_b200 import synthetic
    from voxneus_b200.serving import Request

    pool = synthetic.RayPool(n_cams=8, seed=seed)
    o, d = pool.sample(n)
    return Request(scene, "render", (o, d))


def _query_req(scene, n, seed):
    from voxneus_b200.serving import Request

    g = torch.Generator().manual_seed(seed)
    return Request(scene, "query", (torch.rand(n, 3, generator=g) * 2 - 1,))


def test_results_alone_and_in_the_mix_are_identical():
    from voxneus_b200.rendering import RaySampler

    store = _store()
    eng = _engine(store)
    try:
        a = eng.submit(_render_req("s1", 3000, seed=7)).wait(60)
        q = eng.submit(_query_req("s2", 20000, seed=8)).wait(60)
        alone = {k: v.clone() for k, v in a.outputs.items()}
        q_alone = {k: v.clone() for k, v in q.outputs.items()}
        # the same requests again, submitted inside a stream of other requests
        mix = []
        for i in range(12):
            mix.append(eng.submit(_render_req(f"s{i % 3}", 500 + 700 * i, seed=100 + i)))
            if i == 4:
                a2 = eng.submit(_render_req("s1", 3000, seed=7))
            if i == 6:
                q2 = eng.submit(_query_req("s2", 20000, seed=8))
            mix.append(eng.submit(_query_req(f"s{(i + 1) % 3}", 1000 + 3000 * i, seed=200 + i)))
        for r in mix + [a2, q2]:
            r.wait(120)
        for k in alone:
            assert torch.equal(alone[k], a2.outputs[k]), k
        for k in q_alone:
            assert torch.equal(q_alone[k], q2.outputs[k]), k
        # and equal to a direct render of the whole batch (reference semantics: render.py:65)
        m = store.scenes["s1"]
        with torch.no_grad():
            out = m.render(a.inputs[0].cuda(), a.inputs[1].cuda(), RaySampler(64, 64, perturb=False), None, None,
                           extras=False)
        assert torch.equal(out["rgb"].cpu(), alone["rgb"]) and torch.equal(out["depth"].cpu(), alone["depth"])
    finally:
        eng.close()


def test_malformed_and_oversized_requests_are_rejected_on_the_host():
    from voxneus_b200.serving import Request, RequestError

    eng = _engine(_store(1), budget_bytes=1 << 20)
    try:
        with pytest.raises(RequestError):
            eng.submit(Request("nope", "render", (torch.zeros(4, 3), torch.ones(4, 3))))
        bad = torch.zeros(4, 3)
        bad[1, 1] = float("nan")
        with pytest.raises(RequestError):
            eng.submit(Request("s0", "render", (torch.zeros(4, 3), bad)))
        with pytest.raises(RequestError):
            eng.submit(Request("s0", "query", (torch.zeros(4, 2),)))
        with pytest.raises(RequestError):
            eng.submit(Request("s0", "query", (torch.zeros(200000, 3),)))  # beyond the 1 MiB budget
        ok = eng.submit(_query_req("s0", 1000, seed=1)).wait(60)
        assert ok.outputs["sdf"].shape == (1000, 1)
    finally:
        eng.close()


def test_worker_exception_fails_requests_and_stops_engine():
    from voxneus_b200.serving import RequestError

    def injector(req):
        if req.rid == 2:
            raise RuntimeError("injected host-side failure")

    eng = _engine(_store(1), fault_injector=injector)
    try:
        eng.submit(_query_req("s0", 1000, seed=1)).wait(60)
        eng.submit(_query_req("s0", 1000, seed=2)).wait(60)
        r = eng.submit(_query_req("s0", 1000, seed=3))
        with pytest.raises(RequestError):
            r.wait(60)
        deadline = time.time() + 10
        while eng.failed is None and time.time() < deadline:
            time.sleep(0.01)
        assert eng.failed and "injected" in eng.failed
        with pytest.raises(RequestError):
            eng.submit(_query_req("s0", 10, seed=4))
    finally:
        eng.close()


def test_admission_waits_for_memory_then_proceeds():
    """HBM admission: with a budget that holds one request's device buffers at a time, requests
    submitted together are admitted one after another, each as the previous one's memory is
    released, and every result equals the same request served alone."""
    from voxneus_b200.serving import ServingEngine

    store = _store(n_scenes=2)
    n = 3000
    need = ServingEngine._bytes_for("render", n)
    eng = _engine(store, budget_bytes=need)
    try:
        alone = eng.submit(_render_req("s0", n, seed=3)).wait(60).outputs["rgb"].clone()
        reqs = [_render_req(f"s{i % 2}", n, seed=3 + i) for i in range(4)]  # built first: submitted together
        for r in reqs:
            eng.submit(r)
        for r in reqs:
            r.wait(120)
        assert eng.reserved == 0
        order = sorted(reqs, key=lambda r: r.admitted)
        for prev, nxt in zip(order, order[1:]):
            assert nxt.admitted >= prev.finished  # waited until the budget had room again
        waits = [r.admitted - r.arrival for r in order]
        assert waits[-1] > waits[0]
        assert torch.equal(reqs[0].outputs["rgb"], alone)
        with pytest.raises(Exception):  # larger than the whole budget: refused at submission
            eng.submit(_render_req("s0", n + 1, seed=9))
    finally:
        eng.close()


def test_small_request_overlaps_a_large_one_on_the_express_lane():
    """A small request submitted right after a large one finishes first (its chunks run on the
    higher-priority express stream beside the large request's) and equals the same request alone."""
    store = _store(n_scenes=2)
    eng = _engine(store)
    try:
        small_alone = eng.submit(_render_req("s0", 700, seed=21)).wait(60).outputs["rgb"].clone()
        big, small = _render_req("s1", 60000, seed=22), _render_req("s0", 700, seed=21)
        eng.submit(big)
        eng.submit(small)
        small.wait(60)
        big.wait(120)
        assert small._express and not big._express
        assert small.finished < big.finished
        assert torch.equal(small.outputs["rgb"], small_alone)
    finally:
        eng.close()


def test_requests_share_a_launch_and_match_alone():
    """Two bulk requests of one scene submitted together: a chunk that one of them cannot fill is
    filled with the other's rays (one launch, a segment table), and both equal the requests alone."""
    store = _store(n_scenes=2)
    eng = _engine(store)
    try:
        a_alone = eng.submit(_render_req("s0", 1500, seed=31)).wait(60).outputs["rgb"].clone()
        b_alone = eng.submit(_render_req("s0", 2600, seed=32)).wait(60).outputs["rgb"].clone()
        before = eng.packed_launches
        # a large request of the other scene keeps the engine queuing chunks, so the two arrive
        # in the same admission round
        busy, a, b = (_render_req("s1", 120000, seed=33), _render_req("s0", 1500, seed=31),
                      _render_req("s0", 2600, seed=32))
        eng.submit(busy)
        time.sleep(0.002)
        eng.submit(b)  # b's first chunk is full; its second one has room for a's rays
        eng.submit(a)
        busy.wait(120)
        a.wait(60)
        b.wait(60)
        assert eng.packed_launches > before
        assert torch.equal(a.outputs["rgb"], a_alone) and torch.equal(b.outputs["rgb"], b_alone)
    finally:
        eng.close()

"""Serving host logic that needs no GPU: request identity and latency statistics."""

import torch


def test_requests_compare_by_identity():
    from voxneus_b200.serving import Request

    a = Request("s0", "query", (torch.zeros(5, 3),))
    b = Request("s0", "query", (torch.zeros(7, 3),))
    c = Request("s0", "query", (torch.zeros(5, 3),))
    active = [a, b, c]
    active.remove(c)  # must not compare tensors of different requests
    assert active == [a, b] and active[0] is a
    assert a != c and len({a, b, c}) == 3


def test_latency_stats_percentiles_and_admission_share():
    from voxneus_b200.serving import Request, latency_stats

    reqs = []
    for i in range(100):
        r = Request("s0", "query", (torch.zeros(1, 3),))
        r.arrival, r.admitted, r.finished = 0.0, 0.001 * i / 10, 0.001 * (i + 1)
        reqs.append(r)
    failed = Request("s0", "query", (torch.zeros(1, 3),))
    failed.error = "x"
    st = latency_stats(reqs + [failed])
    assert st["n"] == 100
    assert abs(st["p50_ms"] - 50.0) < 1e-9 and abs(st["p99_ms"] - 99.0) < 1e-9
    assert abs(st["admission_wait_share"] - 495.0 / 5050.0) < 1e-9  # sum of waits / sum of latencies

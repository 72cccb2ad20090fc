"""The continuous-batching server: every answer equals the same query certified alone
(bit-exact integers), under a burst and under a memory budget small enough to force
admission to wait for completions; latencies and footprints are reported."""
from __future__ import annotations

import pytest

pytestmark = pytest.mark.gpu


def _stream(num, rate=2000.0):
    from qubitserf_b200 import workloads as W
    return W.serving_stream(rate, num=num, seed=4, pool=16)


def _alone(native, items):
    out = []
    for it in items:
        a, _ = native.Batch([it]).run()
        out.append((a[0].distance, a[0].z_weight, a[0].x_weight, a[0].proven, a[0].levels))
    return out


def test_served_answers_equal_alone(native):
    from qubitserf_b200 import serve
    reqs = _stream(80)
    items = [serve.item_of(r) for r in reqs]
    want = _alone(native, items)
    answers, summary = serve.run_stream(reqs, time_scale=0.05)   # 20x the offered rate
    got = [(a.distance, a.z_weight, a.x_weight, a.proven, a.levels) for a in answers]
    assert got == want
    assert summary["all_witnesses_verified"]
    assert summary["rounds"] > 0 and summary["p99_ms"] >= summary["p50_ms"] > 0


def test_memory_budget_admission(native):
    """A 1 MiB budget admits one request at a time (a lone request is always admitted);
    answers are unchanged."""
    from qubitserf_b200 import serve
    reqs = _stream(24)
    items = [serve.item_of(r) for r in reqs]
    want = _alone(native, items)
    answers, summary = serve.run_stream(reqs, mem_budget_bytes=1 << 20, time_scale=0.0)
    got = [(a.distance, a.z_weight, a.x_weight, a.proven, a.levels) for a in answers]
    assert got == want


def test_operator_weights_match_golden(native, golden):
    srv = native.Server()
    try:
        names = golden.names("opweight")
        ts = [srv.submit(("opweight",) + tuple(golden.mats(n))) for n in names]
        for n, t in zip(names, ts):
            a, tm = srv.wait(t)
            r = golden.results[n]
            assert (a.z_weight, a.x_weight) == (r["z_weight"], r["x_weight"]), n
            assert tm.latency_s > 0
    finally:
        srv.stop()

"""Replay a request stream through the continuous-batching server (qsfb_server_*).

    python -m qubitserf_b200.serve --rate 500 --num 2000

Requests are submitted at their Poisson arrival times (workloads.serving_stream), after an
untimed warm-up of the same server (three waited-for waves of 32 requests from another
stream); the server timestamps submission and completion itself.  Reported: p50 / p99 / max latency
(completion - submission), certificates per second (completed requests over the span from
the first submission to the last completion), and the server's round statistics.
"""
from __future__ import annotations

import argparse
import json
import os
import time

# Load every kernel when the context is created instead of at its first launch (CUDA's lazy
# loading would make the first request that needs a kernel variant wait for it mid-stream).
# Takes effect when this process has not started CUDA yet.
os.environ.setdefault("CUDA_MODULE_LOADING", "EAGER")

import numpy as np

from . import _native, workloads


def item_of(req):
    if req.kind == "classical":
        return ("classical", req.mats[0])
    if req.kind == "css":
        return ("css", req.mats[0], req.mats[1], "M")
    return ("opweight",) + tuple(req.mats)


def warm_up(srv, waves=3, per_wave=32, seed=5):
    """Untimed: a few waves of requests from another stream, each waited for, so that the
    timed stream does not pay the server's one-time costs (device allocator buckets, pinned
    staging growth) while its arrivals queue behind them."""
    reqs = workloads.serving_stream(1000.0, num=waves * per_wave, seed=seed)
    for w in range(waves):
        wave = [_native.make_query(item_of(r)) for r in reqs[w * per_wave:(w + 1) * per_wave]]
        tickets = []
        for q, keep in wave:
            t = _native.ctypes.c_longlong()
            _native._check(_native.lib().qsfb_server_submit(srv.h, _native.ctypes.byref(q),
                                                            _native.ctypes.byref(t)),
                           "qsfb_server_submit")
            tickets.append(t.value)
        for t in tickets:
            srv.wait(t)


def run_stream(reqs, intake_threads=0, mem_budget_bytes=64 << 30, max_active=0,
               time_scale=1.0, warm=True):
    """Submit every request at its arrival time, wait for all; returns (answers, summary).
    warm: run warm_up() on the server first (its rounds, busy time and codewords are not
    counted)."""
    items = [item_of(r) for r in reqs]
    queries = [_native.make_query(it) for it in items]   # marshal before the clock starts
    srv = _native.Server(intake_threads, mem_budget_bytes, max_active)
    try:
        if warm:
            warm_up(srv)
        st0 = srv.stats()
        t0 = time.perf_counter()
        tickets = []
        for r, (q, keep) in zip(reqs, queries):
            target = t0 + r.t * time_scale
            while True:
                d = target - time.perf_counter()
                if d <= 0:
                    break
                time.sleep(min(d, 0.0005))
            t = _native.ctypes.c_longlong()
            rc = _native.lib().qsfb_server_submit(srv.h, _native.ctypes.byref(q),
                                                   _native.ctypes.byref(t))
            _native._check(rc, "qsfb_server_submit")
            tickets.append(t.value)
        out = [srv.wait(t) for t in tickets]
        st = srv.stats()
    finally:
        srv.stop()
    lat = np.array([tm.latency_s for _, tm in out])
    first = min(tm.submit_s for _, tm in out)
    last = max(tm.done_s for _, tm in out)
    kinds = {}
    for r, (_, tm) in zip(reqs, out):
        kinds.setdefault(r.kind, []).append(tm.latency_s)
    summary = {
        "requests": len(reqs),
        "p50_ms": float(np.percentile(lat, 50) * 1e3),
        "p99_ms": float(np.percentile(lat, 99) * 1e3),
        "max_ms": float(lat.max() * 1e3),
        "certs_per_s": len(reqs) / max(last - first, 1e-9),
        "offered_rate": (len(reqs) / max(reqs[-1].t - reqs[0].t, 1e-9) / time_scale
                         if time_scale > 0 else float("inf")),
        "rounds": st.rounds - st0.rounds,
        "busy_s": st.busy_s - st0.busy_s,
        "span_s": last - first,
        "codewords": int(st.codewords - st0.codewords),
        "peak_footprint_mb": st.peak_footprint_bytes / 2**20,
        "p50_ms_by_kind": {k: float(np.percentile(v, 50) * 1e3) for k, v in kinds.items()},
        "p99_ms_by_kind": {k: float(np.percentile(v, 99) * 1e3) for k, v in kinds.items()},
        "all_witnesses_verified": bool(all(a.witness_ok for a, _ in out)),
    }
    return [a for a, _ in out], summary


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--rate", type=float, nargs="+", default=[50, 100, 200, 500, 1000, 2000])
    ap.add_argument("--num", type=int, default=2000)
    ap.add_argument("--budget-gb", type=float, default=64.0)
    args = ap.parse_args()
    for rate in args.rate:
        reqs = workloads.serving_stream(rate, num=args.num)
        _, s = run_stream(reqs, mem_budget_bytes=int(args.budget_gb * 2**30))
        print(json.dumps({"rate": rate, **s}), flush=True)


if __name__ == "__main__":
    main()

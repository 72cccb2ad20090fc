"""Failure handling and re-entrancy on the GPU, with failures made on the host only:
allocation failure surfaces as rc 6 and leaves the library usable; concurrent ABI calls
from many host threads (ctypes releases the GIL) each get their own stream and agree with
the serial answers."""
from __future__ import annotations

import os
import threading

import pytest

pytestmark = pytest.mark.gpu


def test_allocation_failure_is_reported_and_recoverable(native, golden):
    Hx, Hz = golden.mats("toric4")
    assert native.css_distance_raw(Hx, Hz, "bz", "M", "gpu", 0, False).distance == 4
    os.environ["QSFB_FAIL_ALLOC"] = "1"
    try:
        # a fresh problem needs fresh device memory for its rows and lists
        H = golden.mats("cfg_classical_96")[0]
        with pytest.raises(RuntimeError, match="rc=6"):
            native.classical_distance_raw(H, "bz", "gpu", 0, False)
        with pytest.raises(RuntimeError, match="rc=6"):
            native.Batch([("classical", H)]).run()
    finally:
        del os.environ["QSFB_FAIL_ALLOC"]
    assert native.css_distance_raw(Hx, Hz, "bz", "M", "gpu", 0, False).distance == 4
    H = golden.mats("cfg_classical_96")[0]
    assert native.classical_distance_raw(H, "bz", "gpu", 0, False).distance == 16


def test_concurrent_calls_from_host_threads(native, golden):
    names = ["toric3", "toric4", "surface4", "steane", "hamming4", "cfg_classical_96",
             "batch_2", "batch_514"]
    serial = {}
    mats = {n: golden.mats(n) for n in names}   # npz reads are not thread-safe: load here
    for n in names:
        r = golden.results[n]
        m = mats[n]
        serial[n] = (native.classical_distance_raw(m[0], "bz", "gpu", 0, False).distance
                     if r["kind"] == "classical" else
                     native.css_distance_raw(m[0], m[1], "bz", "M", "gpu", 0, False).distance)
    errors, got = [], {}

    def work(k):
        try:
            for rep in range(3):
                n = names[(k + rep) % len(names)]
                r = golden.results[n]
                m = mats[n]
                d = (native.classical_distance_raw(m[0], "bz", "gpu", 0, False).distance
                     if r["kind"] == "classical" else
                     native.css_distance_raw(m[0], m[1], "bz", "M", "gpu", 0, False).distance)
                got[(k, rep)] = (n, d)
        except Exception as e:   # collected and asserted below
            errors.append(repr(e))

    th = [threading.Thread(target=work, args=(k,)) for k in range(8)]
    for t in th:
        t.start()
    for t in th:
        t.join(timeout=300)
    assert not errors, errors
    assert len(got) == 24
    for (n, d) in got.values():
        assert d == serial[n] == golden.results[n]["distance"]

"""Information sets built on the device (one warp per subproblem: the greedy peel, or the
matroid partition's classes chosen on the host) against the host construction and the
reference's own (cpp/distfind/css.cpp:177-203, 336-366; cpp/qsf/gf2.cpp:42-58): every
generator matrix, rank, detector row, packed non-pivot row and detector syndrome bit for
bit, on all 1024 codes of the uneven batch and on every golden problem."""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

KEYS = ("n", "K", "stride", "ranks", "even", "count_all", "seed_upper")


def _same(a, b, what):
    for k in KEYS:
        assert a[k] == b[k], (what, k, a[k], b[k])
    for k in ("gamma", "check", "red", "syn"):
        assert a[k].shape == b[k].shape and np.array_equal(a[k], b[k]), (what, k)


def _sides(cs):
    if cs.kind == "classical":
        return [(0, cs.mats)]
    return [(1, cs.mats), (2, cs.mats)]


def test_batch_infosets_device_equals_host(native, ref):
    from qubitserf_b200 import workloads as W
    codes = W.batch_1024(1024)
    device_built, multi_set, checked_ref = 0, 0, 0
    for i, cs in enumerate(codes):
        for kind, mats in _sides(cs):
            d = native.prepare_sides(kind, *mats, on_device=True)
            h = native.prepare_sides(kind, *mats, on_device=False)
            _same(d, h, (i, kind))
            device_built += d["device"]
            multi_set += len(d["ranks"]) > 2
            if ref is not None and i % 8 == 0:
                r = ref.problem_gammas(kind, *mats)
                assert d["ranks"] == r["ranks"] and np.array_equal(d["gamma"], r["gamma"]), i
                checked_ref += 1
    assert device_built == 512 + 2 * 512   # every side of the batch has n <= 128
    assert multi_set > 100
    if ref is not None:
        assert checked_ref >= 190


def test_matroid_partition_classes_on_device(native, ref):
    """Sides whose greedy peel packs fewer full-rank sets than the matroid partition: the
    classes go to the device as explicit column lists (the batch's classical codes have
    dozens of them), and sparse random codes with zero columns exercise many-set peels."""
    from qubitserf_b200 import workloads as W
    from qubitserf_b200.workloads import classical_parity_from_rng
    classes = 0
    for cs in W.batch_1024(1024)[:512:2]:      # 256 of the classical codes
        d = native.prepare_sides(0, *cs.mats, on_device=True)
        h = native.prepare_sides(0, *cs.mats, on_device=False)
        _same(d, h, cs.n)
        classes += d["classes"]
        if ref is not None and d["classes"]:
            r = ref.problem_gammas(0, *cs.mats)
            assert d["ranks"] == r["ranks"] and np.array_equal(d["gamma"], r["gamma"])
    assert classes >= 5
    rng = np.random.default_rng(11)
    for _ in range(40):
        n = int(rng.integers(20, 100))
        k = int(rng.integers(n // 4, n // 2 + 1))
        H = classical_parity_from_rng(rng, n, k)
        H[:, rng.integers(0, n, n // 5)] = 0   # zero columns: peels of up to 13 sets
        d = native.prepare_sides(0, H, on_device=True)
        h = native.prepare_sides(0, H, on_device=False)
        _same(d, h, n)
        assert d["device"]


def test_golden_infosets_device_equals_host(native, golden, ref):
    kinds = {"classical": [0], "css": [1, 2], "opweight": [], "subsystem": [3, 4],
             "stabilizer": [5]}
    seen = 0
    for name, res in golden.results.items():
        mats = golden.mats(name)
        for kind in kinds.get(res["kind"], []):
            if kind == 5 and mats[0].shape[1] % 2:
                continue
            d = native.prepare_sides(kind, *mats, on_device=True)
            h = native.prepare_sides(kind, *mats, on_device=False)
            _same(d, h, (name, kind))
            if ref is not None:
                r = ref.problem_gammas(kind, *mats)
                assert d["ranks"] == r["ranks"] and np.array_equal(d["gamma"], r["gamma"]), name
            seen += 1
    assert seen > 40

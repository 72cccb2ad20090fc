"""The reference's own plain per-code GPU path against this engine, on the same host.

oracle/_ref/libqubitserf_cuda.so is the reference's sources with its CUDA backend
(cpp/qsf/cuda/backend_cuda.cu) compiled for sm_100a, called with backend "gpu": levels of at
least 2^18 codewords run on its bz_enumerate kernel, smaller ones on its CPU backend.  Its
answers (distance, lower bound, proven flag, levels) must equal the drop-in's and the
batched engine's.  Both seed the BZ upper bound with trials split over the host's cores
(cpp/distfind/bz.cpp:30-61), so the comparison is only meaningful on one host: the levels in
tests/golden/batch1024.json, made on another host, may differ where the seed bound does.
"""
from __future__ import annotations

import json

import pytest

from conftest import GOLDEN_DIR

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def refcuda():
    from oracle.refbind import REF_CUDA_LIB, RefCuda
    if not REF_CUDA_LIB.exists():
        pytest.skip("oracle/_ref/libqubitserf_cuda.so not built")
    eng = RefCuda()
    assert eng.available(), "the reference's CUDA backend sees no device"
    return eng


def _fields(r):
    return (r.distance, r.lower_bound, r.proven, r.levels)


def test_reference_gpu_path_equals_drop_in_on_batch_codes(native, refcuda):
    from qubitserf_b200 import workloads as W
    codes = W.batch_1024(1024)
    gold = json.loads((GOLDEN_DIR / "batch1024.json").read_text())["codes"]
    # the heaviest codes of the batch (levels on the reference's kernel) and a stride
    idx = sorted(set(range(0, 1024, 37)) | {47, 96, 168, 195, 204, 215, 219, 246, 682, 914})
    for i in idx:
        cs = codes[i]
        if cs.kind == "classical":
            a = native.classical_distance_raw(cs.mats[0], "bz", "gpu", 0, False)
            b = refcuda.classical(cs.mats[0])
        else:
            a = native.css_distance_raw(cs.mats[0], cs.mats[1], "bz", "M", "gpu", 0, False)
            b = refcuda.css(cs.mats[0], cs.mats[1])
        assert b.backend == b"cuda", i
        assert _fields(a) == _fields(b), (i, _fields(a), _fields(b))
        assert a.distance == gold[i][0], i


def test_reference_gpu_path_equals_batch(native, refcuda):
    from qubitserf_b200 import workloads as W
    codes = W.batch_1024(1024)[::8]
    batch = native.Batch(native.batch_items(codes))
    ans, _ = batch.run()
    for i, (cs, a) in enumerate(zip(codes, ans)):
        if cs.kind == "classical":
            b = refcuda.classical(cs.mats[0])
        else:
            b = refcuda.css(cs.mats[0], cs.mats[1])
        assert _fields(a) == _fields(b), (8 * i, _fields(a), _fields(b))

"""Tensor-core pair sweep: the tcgen05 operand layout (self-test against an integer matrix
product) and the sweep itself (the tensor path is taken on heavy full-rank levels, and the
answers and per-level codeword counts equal those of the CUDA-core kernels alone)."""
from __future__ import annotations

import json
import os
import subprocess
import sys

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.mark.parametrize("packed", [False, True])
@pytest.mark.parametrize("ksteps", [1, 2])
def test_selftest_matches_integer_product(native, ksteps, packed):
    rng = np.random.default_rng(10 + ksteps)
    vals = np.array([-1, 0, 1], dtype=np.int8)
    A = rng.choice(vals, size=(256, 64), p=[0.45, 0.1, 0.45]).astype(np.int8)
    B = rng.choice(vals, size=(128, 64), p=[0.45, 0.1, 0.45]).astype(np.int8)
    D = native.tc_selftest(ksteps, A, B, packed=packed)
    k = 32 * ksteps
    ref = A[:, :k].astype(np.int32) @ B[:, :k].astype(np.int32).T
    assert np.array_equal(D, ref)


def test_selftest_extremes(native):
    # all +1 rows: every product equals the column count; one row of each half negated
    A = np.ones((256, 64), dtype=np.int8)
    B = np.ones((128, 64), dtype=np.int8)
    A[7] = -1
    A[200] = -1
    B[3, :32] = -1
    D = native.tc_selftest(2, A, B)
    ref = A.astype(np.int32) @ B.astype(np.int32).T
    assert ref[7, 0] == -64 and ref[0, 3] == 0
    assert np.array_equal(D, ref)


_CHILD = r"""
import json, sys
sys.path.insert(0, sys.argv[1])
from qubitserf_b200 import _native as N, workloads as W
codes = W.batch_1024(int(sys.argv[2]))
ans, st = N.Batch(N.batch_items(codes)).run()
print(json.dumps({"ans": [[a.distance, a.lower_bound, a.proven, a.levels, a.z_weight,
                           a.x_weight] for a in ans],
                  "codewords": st.codewords, "tc": st.tc_codewords}))
"""


def _run_child(num, tensor):
    env = dict(os.environ)
    env["QSFB_TENSOR"] = "1" if tensor else "0"
    out = subprocess.run([sys.executable, "-c", _CHILD, ROOT, str(num)], env=env,
                         capture_output=True, text=True, timeout=600, check=True)
    return json.loads(out.stdout.strip().splitlines()[-1])


def test_tensor_sweep_equals_cuda_core_sweep():
    on = _run_child(128, True)
    off = _run_child(128, False)
    assert on["tc"] > 0, "no level took the tensor-core sweep"
    assert off["tc"] == 0
    assert on["ans"] == off["ans"]
    # every level still evaluates every codeword exactly once
    assert on["codewords"] == off["codewords"]


def test_bounded_wait_reports_and_device_survives(native):
    # the drill copies nothing, so the kernel's operand and accumulator waits run out; the
    # call reports rc 4 and the next launch on the same context is exact again
    A = np.ones((256, 64), dtype=np.int8)
    B = np.ones((128, 64), dtype=np.int8)
    with pytest.raises(RuntimeError, match="rc=4"):
        native.tc_selftest(-1, A, B)
    D = native.tc_selftest(2, A, B)
    assert np.array_equal(D, np.full((256, 128), 64, dtype=np.int32))

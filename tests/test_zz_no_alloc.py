"""qsfb_enumerate_plan_noalloc: the enumeration level for callers that cannot allocate
device memory (their own pool owns the device, or they must avoid the device-wide
synchronisation a cudaMalloc can cause).  It takes caller-owned device buffers and keeps
its scratch in a fixed array inside the library.  Checked through the C ABI against the
allocating entry point qsfb_enumerate_plan, bit for bit, on two calls in a row, alone or
after every other test."""
from __future__ import annotations

import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

WEIGHT_NONE = 1 << 30


def _device_buffers(torch, gamma, check, ng):
    dev = torch.device("cuda", 0)
    g = torch.from_numpy(np.ascontiguousarray(gamma).view(np.int64).reshape(-1).copy()).to(dev)
    c = torch.from_numpy(np.ascontiguousarray(check).view(np.int64).reshape(-1).copy()
                         if check.size else np.zeros(1, np.int64)).to(dev)
    best = torch.zeros(1, dtype=torch.int32, device=dev)
    counts = torch.zeros(ng, dtype=torch.int64, device=dev)
    og = torch.zeros(1, dtype=torch.int32, device=dev)
    orank = torch.zeros(1, dtype=torch.int64, device=dev)
    return g, c, best, counts, og, orank


def _noalloc(native, torch, n, K, d, gamma, check, cur, optional=True):
    """One call; optional=False passes NULL for the per-set counts and the arg-min."""
    stride = (n + 63) // 64
    ng = gamma.size // (K * stride)
    kcheck = check.size // stride
    g, c, best, counts, og, orank = _device_buffers(torch, gamma, check, ng)
    stream = torch.cuda.current_stream().cuda_stream
    opt = (counts.data_ptr(), og.data_ptr(), orank.data_ptr()) if optional else (None,) * 3
    rc = native.lib().qsfb_enumerate_plan_noalloc(
        n, stride, K, d, ng, g.data_ptr(), kcheck, c.data_ptr(), cur, best.data_ptr(),
        *opt, stream)
    torch.cuda.synchronize()
    if rc != 0:
        return rc, None
    if not optional:
        return 0, int(best.item())
    rank = int(orank.cpu().numpy().view(np.uint64)[0])
    return 0, (int(best.item()), [int(x) for x in counts.cpu().numpy().view(np.uint64)],
               int(og.item()), rank)


@pytest.mark.parametrize("K,stride,d,ng,kcheck,cur", [
    (14, 2, 4, 2, 2, WEIGHT_NONE),
    (24, 1, 6, 3, 1, 40),
    (30, 2, 5, 2, 0, WEIGHT_NONE),     # no detector: every codeword counts
    (40, 3, 4, 1, 3, 70),              # 6-word rows
])
def test_noalloc_matches_allocating_entry_point(native, K, stride, d, ng, kcheck, cur):
    torch = pytest.importorskip("torch")
    rng = np.random.default_rng(1000 * K + d)
    gamma = rng.integers(0, 2**63, (ng, K, stride), dtype=np.uint64)
    check = rng.integers(0, 2**63, (kcheck, stride), dtype=np.uint64)
    n = stride * 64
    want = native.enumerate_plan(n, K, d, gamma, check, cur)
    want = (want[0], [int(x) for x in want[1]], want[2],
            want[3] if want[2] >= 0 else (1 << 64) - 1)
    for _ in range(2):   # two calls in a row share (and must fully rewrite) the scratch
        rc, got = _noalloc(native, torch, n, K, d, gamma, check, cur)
        assert rc == 0
        assert got == want, (got, want)
    rc, got = _noalloc(native, torch, n, K, d, gamma, check, cur, optional=False)
    assert (rc, got) == (0, want[0])


def test_noalloc_rejects_sizes_beyond_its_scratch(native):
    torch = pytest.importorskip("torch")
    rng = np.random.default_rng(2)
    gamma = rng.integers(0, 2**63, (1, 129, 1), dtype=np.uint64)   # K = 129 > 128
    check = np.zeros((0, 1), np.uint64)
    rc, _ = _noalloc(native, torch, 64, 129, 3, gamma, check, WEIGHT_NONE)
    assert rc == 8
    gamma = rng.integers(0, 2**63, (1, 128, 2), dtype=np.uint64)   # lists beyond 32 MiB
    rc, _ = _noalloc(native, torch, 128, 128, 9, gamma, check, WEIGHT_NONE)
    assert rc == 8
    for d in (40, 64):   # C(128, d/2) saturates the 64-bit binomials: still rejected
        rc, _ = _noalloc(native, torch, 128, 128, d, gamma, check, WEIGHT_NONE)
        assert rc == 8

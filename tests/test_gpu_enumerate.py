"""GPU per-level enumeration (qsfb_enumerate_plan) against the oracle's brute force:
randomized raw plans in the style of the reference's cpu_enum_ref
(cpp/distfind/tests/cpu_enum_ref.cpp:78-133), bit-exact minimum, per-set counts C(K,d)
and the arg-min (set, lexicographic rank) with the smallest-(weight, set, rank) tie-break."""
from __future__ import annotations

from math import comb

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

WEIGHT_NONE = 1 << 30


def _plan(rng, K, stride, ng, kcheck):
    gamma = rng.integers(0, 2**63, (ng, K, stride), dtype=np.uint64)
    check = rng.integers(0, 2**63, (kcheck, stride), dtype=np.uint64)
    return gamma, check


def _check_case(native, orc, rng, K, stride, d, ng, kcheck, cur):
    d = max(1, min(d, K))
    g, c = _plan(rng, K, stride, ng, kcheck)
    n = stride * 64
    best, counts, ag, ar = native.enumerate_plan(n, K, d, g, c, cur)
    eb, ecounts, eg, er = orc.enumerate(n, K, d, g, c, cur)
    assert best == eb, (K, stride, d, ng, kcheck, cur, best, eb)
    assert list(counts) == [comb(K, d)] * ng
    if eb < cur:
        assert (ag, ar) == (eg, er), (ag, ar, eg, er)
    else:
        assert ag == -1


def test_random_plans_match_oracle(native, orc):
    rng = np.random.default_rng(0xC0FFEE)
    for _ in range(60):
        K = int(rng.integers(4, 15))
        stride = int(rng.integers(1, 4))
        cur = WEIGHT_NONE if rng.integers(0, 4) == 0 else int(rng.integers(0, stride * 64 + 1))
        _check_case(native, orc, rng, K, stride, int(rng.integers(1, 6)),
                    int(rng.integers(1, 4)), int(rng.integers(0, 4)), cur)


@pytest.mark.parametrize("K,stride,d,ng,kcheck,cur", [
    (8, 1, 1, 1, 0, WEIGHT_NONE),    # d == 1
    (6, 2, 1, 2, 2, WEIGHT_NONE),    # d == 1, several sets
    (5, 1, 5, 1, 1, WEIGHT_NONE),    # d == K: a single combination
    (7, 2, 4, 2, 0, WEIGHT_NONE),    # no detector: every codeword counts
    (10, 3, 3, 1, 2, 0),             # bound 0: nothing can be accepted
    (12, 1, 4, 3, 1, 1),             # very tight bound
    (20, 2, 6, 2, 2, WEIGHT_NONE),   # C(20,6)=38760: multi-job level
    (24, 1, 8, 1, 1, 30),
    (30, 2, 5, 3, 3, 60),
    (40, 4, 4, 2, 2, WEIGHT_NONE),   # 4-word rows
    (18, 8, 5, 2, 2, WEIGHT_NONE),   # 8-word rows: probe + full evaluation path
    (16, 16, 6, 1, 1, 600),          # 1024-bit rows
])
def test_edge_plans(native, orc, K, stride, d, ng, kcheck, cur):
    rng = np.random.default_rng(K * 1000 + stride * 10 + d)
    _check_case(native, orc, rng, K, stride, d, ng, kcheck, cur)


def test_large_level_counts_and_minimum(native, orc):
    """A level large enough to spread over every SM (C(34,7) = 5.4M combinations x 2 sets);
    the minimum is checked against the oracle's two-level kernel."""
    rng = np.random.default_rng(5)
    K, stride, d = 34, 2, 7
    g, c = _plan(rng, K, stride, 2, 2)
    best, counts, _, _ = native.enumerate_plan(128, K, d, g, c, WEIGHT_NONE)
    assert list(counts) == [comb(K, d)] * 2
    assert best == orc.enumerate_fast(128, K, d, g, c, WEIGHT_NONE)


def test_repeat_deterministic(native):
    rng = np.random.default_rng(9)
    g, c = _plan(rng, 26, 2, 2, 2)
    outs = {native.enumerate_plan(128, 26, 5, g, c, WEIGHT_NONE)[0::2] for _ in range(5)}
    assert len(outs) == 1

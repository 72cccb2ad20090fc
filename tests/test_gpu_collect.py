"""The codeaut low-weight collector on the GPU (codeaut_bz_* through the C ABI) against the
reference's own outputs (golden fixtures made by its codeaut_bz_collect), the C oracle and,
where oracle/_ref travels with the repository, the reference library itself: the same rows
in the same order and the same combination counts."""
from __future__ import annotations

import math
import os

import numpy as np
import pytest

from test_oracle import load_collect_goldens

pytestmark = pytest.mark.gpu


def systematic(rng, k, n):
    A = rng.integers(0, 2, size=(k, n - k), dtype=np.uint8)
    G = np.concatenate([np.eye(k, dtype=np.uint8), A], axis=1)
    return G[:, rng.permutation(n)]


@pytest.fixture
def force_probe():
    """Force the probe width and bound for the calls of one test (the library reads
    QSFB_COLLECT_HP / QSFB_COLLECT_FILT on every call)."""
    def set_probe(hp, filt):
        os.environ["QSFB_COLLECT_HP"] = str(hp)
        os.environ["QSFB_COLLECT_FILT"] = str(filt)
    yield set_probe
    os.environ.pop("QSFB_COLLECT_HP", None)
    os.environ.pop("QSFB_COLLECT_FILT", None)


def test_collect_matches_reference_goldens(native):
    for name, G, p, keep, combos, rows in load_collect_goldens():
        got, got_combos = native.collect(G, p, keep)
        assert got_combos == combos, name
        assert np.array_equal(got, rows), name


@pytest.mark.parametrize("hp,filt", [(1, 0), (2, 0), (2, 2), (4, 0), (4, 4), (4, 6), (8, 0)])
def test_collect_every_probe_variant_equals_oracle(native, orc, force_probe, hp, filt):
    rng = np.random.default_rng(100 + 10 * hp + filt)
    force_probe(hp, filt)
    for trial in range(12):
        m = int(rng.integers(1, 26))
        n = int(rng.integers(1, 300))
        p = int(rng.integers(1, 6))
        keep = int(rng.integers(1, max(2, n // 3)))
        G = rng.integers(0, 2, size=(m, n), dtype=np.uint8)
        if trial % 2 == 0 and m <= n:
            G = systematic(rng, m, n)
        if trial % 5 == 0:
            G[rng.integers(0, m)] = 0
        got, combos, st = native.collect(G, p, keep, stats=True)
        assert (st.probe_words, st.filter) == (hp, filt)
        want, want_combos = orc.collect(G, p, keep)
        assert combos == want_combos
        assert np.array_equal(got, want), (trial, m, n, p, keep)


def test_collect_large_levels_equal_reference(native, ref, orc):
    """Multi-tile terms and multi-chunk suffix ranges (lists of thousands of entries)."""
    rng = np.random.default_rng(7)
    cases = [(systematic(rng, 48, 96), 6, 14), (systematic(rng, 40, 140), 7, 36),
             (rng.integers(0, 2, size=(36, 80), dtype=np.uint8), 5, 26),
             (systematic(rng, 64, 1024), 3, 470)]
    for G, p, keep in cases:
        got, combos, st = native.collect(G, p, keep, stats=True)
        if ref is not None:
            want, want_combos = ref.collect(G, p, keep)
        else:
            want, want_combos = orc.collect(G, p, keep)
        assert combos == want_combos == sum(math.comb(G.shape[0], s)
                                            for s in range(1, min(p, G.shape[0]) + 1))
        assert np.array_equal(got, want)
        assert st.passes >= st.hits >= got.shape[0]


def test_collect_overflow_reruns_with_exact_capacity(native, orc):
    # 20 rows, p = 10, keep = n: every nonzero XOR is kept (616,665 hits before
    # deduplication), far over the first output buffer; the sweep runs again into a
    # buffer of exactly the counted size and the result is complete
    rng = np.random.default_rng(5)
    G = rng.integers(0, 2, size=(20, 40), dtype=np.uint8)
    got, combos, st = native.collect(G, 10, 40, stats=True)
    want, want_combos = orc.collect(G, 10, 40)
    assert st.reruns == 1
    assert combos == want_combos == sum(math.comb(20, s) for s in range(1, 11))
    assert np.array_equal(got, want)
    # a full-rank G gives distinct XORs for distinct subsets: nothing was dropped
    assert got.shape[0] == combos and st.hits == combos
    # 22 rows, p = 9: 1,097,789 candidate pairs, over the first candidate buffer (2^20) as
    # well: the sweeps run again into enough candidate slots, then the hits into enough rows
    G = rng.integers(0, 2, size=(22, 40), dtype=np.uint8)
    got, combos, st = native.collect(G, 9, 40, stats=True)
    want, want_combos = orc.collect(G, 9, 40)
    assert st.reruns == 2 and st.passes == combos == want_combos
    assert np.array_equal(got, want)


def test_collect_complete_at_full_depth_equals_brute_force(native):
    """The reference's own known answer (tests/codeaut/test_codeaut.py:168-187): with every
    subset size enumerated, the collected rows are ALL nonzero codewords of weight <= keep,
    checked against the 2^k codewords of the row space."""
    rng = np.random.default_rng(3)
    done = 0
    for _ in range(30):
        k = int(rng.integers(8, 14))
        n = int(rng.integers(k + 1, 2 * k + 5))
        B = rng.integers(0, 2, size=(k, n), dtype=np.uint8)
        idx = np.arange(1, 1 << k)
        U = ((idx[:, None] >> np.arange(k)) & 1).astype(np.uint8)
        C = (U @ B) % 2
        if len({r.tobytes() for r in C}) != (1 << k) - 1 or any(not r.any() for r in C):
            continue                                   # rank-deficient draw
        keep = int(rng.integers(1, n + 1))
        got, combos = native.collect(B, k, keep)
        w = C.sum(1)
        truth = {r.tobytes() for r in C[(w >= 1) & (w <= keep)]}
        assert {r.tobytes() for r in got} == truth
        assert combos == (1 << k) - 1
        done += 1
    assert done >= 10


def test_collect_edge_shapes(native, orc):
    rng = np.random.default_rng(9)
    for m, n, p, keep in [(1, 1, 1, 1), (1, 64, 1, 64), (3, 65, 3, 65), (7, 128, 7, 50),
                          (2, 1024, 2, 1024), (64, 70, 2, 6), (5, 5, 5, 5)]:
        G = rng.integers(0, 2, size=(m, n), dtype=np.uint8)
        got, combos = native.collect(G, p, keep)
        want, want_combos = orc.collect(G, p, keep)
        assert combos == want_combos and np.array_equal(got, want), (m, n, p, keep)
    # duplicate rows and a zero row: weight-0 XORs are never collected
    G = np.zeros((4, 10), np.uint8)
    G[0, :3] = 1
    G[1] = G[0]
    got, _ = native.collect(G, 4, 10)
    assert got.shape[0] == 1 and got[0].sum() == 3


def test_collect_refusals(native):
    G = np.ones((3, 5), np.uint8)
    with pytest.raises(RuntimeError, match="rc=5"):
        native.collect(G, 2, 3, backend="cpu")
    with pytest.raises(RuntimeError, match="rc=5"):
        native.collect(np.ones((3, 1025), np.uint8), 2, 3)
    assert native.lib().codeaut_backend_available(b"gpu") == 1

"""The C oracle pinned against the reference: golden vectors (made by the reference,
tests/golden/make_golden.py) and, where oracle/_ref is built, the reference library itself."""
from __future__ import annotations

import numpy as np
import pytest

# Golden cases too slow for the single-threaded oracle inside the CPU suite.
SLOW = {"cfg_css_128", "qrm_1_10", "toric7", "surface7", "cfg_classical_128"}


def _oracle_result(orc, kind, mats, extra, **kw):
    if kind == "classical":
        return orc.classical(mats[0], **kw)
    if kind == "css":
        return orc.css(mats[0], mats[1], extra.get("which", "M"), **kw)
    if kind == "subsystem":
        return orc.subsystem(mats[0], mats[1], extra.get("which", "M"), **kw)
    if kind == "stabilizer":
        return orc.stabilizer(mats[0], extra.get("which", "M"), **kw)
    raise ValueError(kind)


def test_oracle_matches_golden_distances(golden, orc):
    bad = []
    for name, res in golden.results.items():
        if name in SLOW:
            continue
        mats = golden.mats(name)
        if res["kind"] == "opweight":
            got = orc.operator_weight(*mats)
            if got != (res["z_weight"], res["x_weight"]):
                bad.append((name, got, res))
            continue
        r = _oracle_result(orc, res["kind"], mats, res)
        if r.distance != res["distance"] or r.proven != res["proven"]:
            bad.append((name, r.distance, res["distance"]))
    assert not bad, bad


def test_oracle_no_early_stop_counts_match_reference(golden, orc):
    """Per-level (w, active, C(K,w)*active) work with early termination disabled."""
    seen = 0
    for name, res in golden.results.items():
        lv = res.get("no_early_stop_levels")
        if not lv:
            continue
        mats = golden.mats(name)
        r = _oracle_result(orc, res["kind"], mats, res, no_early_stop=True, trace_cap=256)
        got = [(w, a) for (_side, w, a) in r.trace]
        want = [(x["w"], x["active"]) for x in lv]
        assert got == want, (name, got, want)
        assert r.codewords == sum(x["work"] for x in lv), name
        assert r.proven == 0
        seen += 1
    assert seen >= 5


def _random_plan(rng, K, stride, d, ng, kcheck):
    gamma = rng.integers(0, 2**63, (ng, K, stride), dtype=np.uint64)
    check = rng.integers(0, 2**63, (kcheck, stride), dtype=np.uint64)
    return gamma, check


def test_oracle_enumerate_brute_vs_two_level(orc):
    """The brute-force level (eval_combo order) and the two-level kernel agree."""
    rng = np.random.default_rng(0xC0FFEE)
    for _ in range(80):
        K = int(rng.integers(4, 15))
        stride = int(rng.integers(1, 4))
        d = int(rng.integers(1, min(K, 5) + 1))
        ng, kc = int(rng.integers(1, 4)), int(rng.integers(0, 4))
        g, c = _random_plan(rng, K, stride, d, ng, kc)
        cb = int(rng.choice([1 << 30, int(rng.integers(0, stride * 64 + 1))]))
        a = orc.enumerate(stride * 64, K, d, g, c, cb)[0]
        b = orc.enumerate_fast(stride * 64, K, d, g, c, cb)
        assert a == b, (K, stride, d, ng, kc, cb, a, b)


def test_oracle_enumerate_matches_reference_backend(orc, ref):
    """cpu_enum_ref-style randomized plans (cpp/distfind/tests/cpu_enum_ref.cpp:78-133)
    against the reference CPU backend itself, single- and multi-threaded."""
    if ref is None:
        pytest.skip("reference library not built here")
    rng = np.random.default_rng(0xC0FFEE)
    cases = []
    for _ in range(50):
        cases.append((int(rng.integers(4, 15)), int(rng.integers(1, 4)), int(rng.integers(1, 6)),
                      int(rng.integers(1, 4)), int(rng.integers(0, 4)), 0))
    cases += [(8, 1, 1, 1, 0, 0), (6, 2, 1, 2, 2, 0), (5, 1, 5, 1, 1, 0), (7, 2, 4, 2, 0, 0)]
    for T in (2, 3, 8, 16):
        cases += [(18, 2, 5, 2, 2, T), (16, 3, 6, 1, 1, T)]
    for K, st, d, ng, kc, T in cases:
        d = max(1, min(d, K))
        g, c = _random_plan(rng, K, st, d, ng, kc)
        for cb in (1 << 30, int(rng.integers(0, st * 64 + 1)), 0, 1):
            want = ref.enumerate(st * 64, st, K, d, g, c, cb, threads=T)
            got = orc.enumerate(st * 64, K, d, g, c, cb)[0]
            assert got == want, (K, st, d, ng, kc, cb, got, want)


def test_oracle_random_batch_codes_match_reference(orc, ref):
    if ref is None:
        pytest.skip("reference library not built here")
    from qubitserf_b200 import workloads as W
    codes = W.batch_1024(24)
    for i, cs in enumerate(codes):
        if cs.kind == "classical":
            assert orc.classical(cs.mats[0]).distance == ref.classical(cs.mats[0]).distance, i
        elif cs.n <= 80:
            assert orc.css(*cs.mats).distance == ref.css(*cs.mats).distance, i


def test_reference_cuda_build_equals_cpu_build_without_device(ref, golden):
    """oracle/_ref/libqubitserf_cuda.so (the reference's sources with its CUDA backend, the
    plain per-code GPU comparator) is a working build of the same library: without a device
    its CUDA backend reports unavailable, backend "gpu" runs the reference CPU backend, and
    every field equals the CPU build's."""
    from oracle.refbind import REF_CUDA_LIB, RefCuda
    if ref is None or not REF_CUDA_LIB.exists():
        pytest.skip("reference libraries not built here")
    import torch
    if torch.cuda.is_available():
        pytest.skip("a device is present: the GPU tests compare the CUDA path")
    rc = RefCuda()
    assert not rc.available()
    for name in ["hamming4", "steane", "toric3", "surface3", "batch_512"]:
        res = golden.results[name]
        mats = golden.mats(name)
        if res["kind"] == "classical":
            a, b = rc.classical(mats[0]), ref.classical(mats[0])
        else:
            a, b = rc.css(*mats), ref.css(*mats)
        assert (a.distance, a.lower_bound, a.proven, a.levels) == \
            (b.distance, b.lower_bound, b.proven, b.levels), name
        assert a.distance == res["distance"], name


def test_oracle_problem_ranks_match_reference(orc, ref, golden):
    if ref is None:
        pytest.skip("reference library not built here")
    for name in ["cfg_classical_96", "cfg_classical_128", "toric5", "surface5", "hamming4",
                 "batch_0", "batch_1", "batch_515"]:
        mats = golden.mats(name)
        kind = 0 if golden.results[name]["kind"] == "classical" else 1
        a = orc.prepare(kind, *mats)
        b = ref.problem_gammas(kind, *mats)
        assert a["ranks"] == b["ranks"] and a["K"] == b["K"], name
        assert a["seed_upper"] == b["seed_upper"] and a["even"] == b["even"], name


def load_collect_goldens():
    """(name, G, p, keep, combos, rows) of tests/golden/collect.npz (made by the reference's
    own codeaut_bz_collect, tests/golden/make_golden.py --collect)."""
    from conftest import GOLDEN_DIR
    z = np.load(GOLDEN_DIR / "collect.npz")
    names = sorted({k.split("__")[0] for k in z.files})
    out = []
    for nm in names:
        p, keep, combos, count, n = (int(v) for v in z[f"{nm}__meta"])
        rows = np.unpackbits(z[f"{nm}__rows"], axis=1)[:, :n] if count else \
            np.zeros((0, n), np.uint8)
        out.append((nm, z[f"{nm}__G"], p, keep, combos, rows))
    return out


def test_collect_oracle_matches_golden(orc):
    cases = load_collect_goldens()
    assert len(cases) >= 12
    for name, G, p, keep, combos, rows in cases:
        got, got_combos = orc.collect(G, p, keep)
        assert got_combos == combos, name
        assert np.array_equal(got, rows), name


def test_collect_oracle_matches_reference_random(orc, ref):
    if ref is None:
        pytest.skip("oracle/_ref not built")
    rng = np.random.default_rng(21)
    for trial in range(40):
        m = int(rng.integers(1, 18))
        n = int(rng.integers(1, 200))
        p = int(rng.integers(1, 7))
        keep = int(rng.integers(-2, n // 2 + 3))
        G = rng.integers(0, 2, size=(m, n), dtype=np.uint8)
        if trial % 4 == 0:
            G[:, : min(m, n)] = np.eye(m, dtype=np.uint8)[:, : min(m, n)]
        if trial % 5 == 0:
            G[rng.integers(0, m)] = 0
        a, ca = ref.collect(G, p, keep)
        b, cb = orc.collect(G, p, keep)
        assert ca == cb and np.array_equal(a, b), (trial, m, n, p, keep)


def mitm_case(engine, kind, mats, res, **kw):
    """(distance, lower_bound, proven, levels) of method "mitm" on a golden case, or
    (z_weight, x_weight, proven) for an operator weight, from the oracle or the reference."""
    which = res.get("which", "M")
    if kind == "classical":
        r = engine.classical(mats[0], method="mitm", **kw)
    elif kind == "css":
        r = engine.css(mats[0], mats[1], which, method="mitm", **kw)
    elif kind == "subsystem":
        r = engine.subsystem(mats[0], mats[1], which, method="mitm", **kw)
    elif kind == "stabilizer":
        r = engine.stabilizer(mats[0], which, method="mitm", **kw)
        r = r[1] if isinstance(r, tuple) else r
    else:
        r = engine.operator_weight(*mats, method="mitm", **kw)
        if isinstance(r, tuple):
            return [int(r[0]), int(r[1])]
        return [int(r.z_weight), int(r.x_weight)]
    return [int(r.distance), int(r.lower_bound), int(r.proven), int(r.levels)]


def test_mitm_oracle_matches_golden(golden, orc):
    import json
    from conftest import GOLDEN_DIR
    want = json.loads((GOLDEN_DIR / "mitm.json").read_text())
    assert len(want) >= 40
    for name, exp in want.items():
        res = golden.results[name]
        got = mitm_case(orc, res["kind"], golden.mats(name), res)
        assert got == exp[:len(got)], (name, got, exp)


def test_mitm_oracle_matches_reference_random(orc, ref):
    if ref is None:
        pytest.skip("oracle/_ref not built")
    import codes as C
    from qubitserf_b200 import workloads as W
    rng = np.random.default_rng(31)
    for trial in range(12):
        n = int(rng.integers(10, 34))
        Hx, Hz = W.css_from_rng(rng, n, int(rng.integers(2, n // 3 + 1)),
                                int(rng.integers(2, n // 3 + 1)))
        for which in "ZXM":
            a = ref.css(Hx, Hz, which, method="mitm")
            b = orc.css(Hx, Hz, which, method="mitm")
            assert (a.distance, a.lower_bound, a.proven, a.levels) == \
                   (b.distance, b.lower_bound, b.proven, b.levels), (trial, which)
    for trial in range(8):
        S = C.random_isotropic(rng, int(rng.integers(5, 10)), int(rng.integers(2, 5)))
        rc, a = ref.stabilizer(S, "M", method="mitm")
        b = orc.stabilizer(S, "M", method="mitm")
        assert rc == 0
        assert (a.distance, a.lower_bound, a.proven, a.levels) == \
               (b.distance, b.lower_bound, b.proven, b.levels), trial

"""GPU distances through the drop-in C ABI against the reference's golden vectors, the
reference library itself (full DistfindResult where it is present), the C oracle, and the
host verification of every returned witness.  Mirrors the reference's GPU tests
(tests/distfind/test_distance.py:129-226): strict equality, repeated runs, Z/X alternation,
deep paths and large n."""
from __future__ import annotations

import os
from math import comb

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def run(native, kind, mats, extra):
    which = extra.get("which", "M")
    if kind == "classical":
        return native.classical_distance_raw(mats[0], "bz", "gpu", 0, False)
    if kind == "css":
        return native.css_distance_raw(mats[0], mats[1], "bz", which, "gpu", 0, False)
    if kind == "subsystem":
        return native.subsystem_distance_raw(mats[0], mats[1], "bz", which, "gpu", 0, False)
    if kind == "stabilizer":
        return native.stabilizer_distance_raw(mats[0], "bz", which, "gpu", 0, False)
    raise ValueError(kind)


def ref_run(ref, kind, mats, extra):
    which = extra.get("which", "M")
    if kind == "classical":
        return ref.classical(mats[0])
    if kind == "css":
        return ref.css(mats[0], mats[1], which)
    if kind == "subsystem":
        return ref.subsystem(mats[0], mats[1], which)
    if kind == "stabilizer":
        return ref.stabilizer(mats[0], which)[1]
    raise ValueError(kind)


def distance_cases(golden):
    return [n for n, r in golden.results.items() if r["kind"] != "opweight"]


def test_golden_distances_and_witnesses(native, golden):
    bad = []
    for name in distance_cases(golden):
        res = golden.results[name]
        r = run(native, res["kind"], golden.mats(name), res)
        rep = native.last_report()
        if r.distance != res["distance"] or r.proven != res["proven"]:
            bad.append((name, r.distance, res["distance"], r.proven))
        if r.distance > 0 and not rep.witness_ok:
            bad.append((name, "witness not verified"))
        assert r.backend.decode() == "cuda"
    assert not bad, bad


def test_full_result_matches_reference(native, ref, golden):
    """distance, lower_bound, proven and levels equal the reference run on this host (same
    information sets, same random-information-set seed)."""
    if ref is None:
        pytest.skip("reference library not present on this host")
    skip = {"cfg_css_128"}
    for name in distance_cases(golden):
        if name in skip:
            continue
        res = golden.results[name]
        mats = golden.mats(name)
        a = run(native, res["kind"], mats, res)
        b = ref_run(ref, res["kind"], mats, res)
        assert (a.distance, a.lower_bound, a.proven, a.levels) == \
            (b.distance, b.lower_bound, b.proven, b.levels), name


def test_witness_is_a_minimum_weight_logical(native, golden):
    """The returned codeword lies in the code (H c = 0), is not a stabilizer/detector-trivial
    element, and has weight d."""
    H = golden.mats("cfg_classical_96")[0]
    r = native.classical_distance_raw(H, "bz", "gpu", 0, False)
    c = native.last_witness()
    assert c is not None and int(c.sum()) == r.distance == 16
    assert not (H.astype(np.int64) @ c % 2).any()
    Hx, Hz = golden.mats("toric5")
    r = native.css_distance_raw(Hx, Hz, "bz", "Z", "gpu", 0, False)
    c = native.last_witness()
    assert int(c.sum()) == r.distance == 5
    assert not (Hx.astype(np.int64) @ c % 2).any()          # commutes with X checks
    from qubitserf_b200.workloads import gf2_rank
    assert gf2_rank(np.vstack([Hz, c])) == gf2_rank(Hz) + 1  # not a Z stabilizer


def test_no_early_stop_counts_match_reference(native, golden):
    """Per-(information set, w) enumeration counts with early termination disabled equal
    the reference's DISTFIND_PROFILE work (C(K,w) per active set)."""
    os.environ["DISTFIND_NO_EARLY_STOP"] = "1"
    try:
        seen = 0
        for name, res in golden.results.items():
            lv = res.get("no_early_stop_levels")
            if not lv:
                continue
            r = run(native, res["kind"], golden.mats(name), res)
            assert r.proven == 0
            recs = native.last_counts()
            by_w = {}
            for side, w, g, cnt in recs:
                by_w.setdefault(w, []).append(cnt)
            for x in lv:
                cnts = by_w.get(x["w"], [])
                if x["active"] == 0:
                    assert not cnts
                    continue
                assert len(cnts) == x["active"], (name, x)
                assert all(cc == comb(x["K"], x["w"]) for cc in cnts), (name, x, cnts)
                assert sum(cnts) == x["work"], (name, x)
            seen += 1
        assert seen >= 5
    finally:
        del os.environ["DISTFIND_NO_EARLY_STOP"]


def test_repeated_runs_are_deterministic(native, golden):
    for name in ["toric5", "surface5", "cfg_classical_96", "batch_3"]:
        res = golden.results[name]
        mats = golden.mats(name)
        vals = set()
        for _ in range(6):
            r = run(native, res["kind"], mats, res)
            vals.add((r.distance, r.levels, r.lower_bound, tuple(native.last_witness())))
        assert len(vals) == 1, (name, vals)


def test_zx_alternation(native, golden):
    """Alternating Z and X solves never reuse stale device data (tests/distfind/
    test_distance.py:178-188)."""
    for L in (5, 6):
        Hx, Hz = golden.mats(f"toric{L}")
        for _ in range(12):
            z = native.css_distance_raw(Hx, Hz, "bz", "Z", "gpu", 0, False).distance
            x = native.css_distance_raw(Hx, Hz, "bz", "X", "gpu", 0, False).distance
            assert z == L and x == L


def test_random_batch_codes_match_oracle(native, orc):
    from qubitserf_b200 import workloads as W
    codes = W.batch_1024(48)
    for i, cs in enumerate(codes):
        if cs.kind == "classical":
            if cs.n > 110:
                continue
            a = native.classical_distance_raw(cs.mats[0], "bz", "gpu", 0, False).distance
            b = orc.classical(cs.mats[0]).distance
        else:
            if cs.n > 100:
                continue
            a = native.css_distance_raw(*cs.mats, "bz", "M", "gpu", 0, False).distance
            b = orc.css(*cs.mats).distance
        assert a == b, (i, cs.kind, cs.n, a, b)
        assert native.last_report().witness_ok == 1


def test_config_sizes_full(native, golden):
    """The three single-instance workloads at full size: d = 16, 24, 8."""
    for name, want in (("cfg_classical_96", 16), ("cfg_classical_128", 24), ("cfg_css_128", 8)):
        res = golden.results[name]
        r = run(native, res["kind"], golden.mats(name), res)
        assert r.distance == want and r.proven == 1
        rep = native.last_report()
        assert rep.witness_ok == 1 and rep.codewords > 0

"""Method "mitm" (meet in the middle) on the GPU through the distfind_* ABI, against the
reference's own results (tests/golden/mitm.json, made by its mitm_distance), the reference
library itself on random codes (where oracle/_ref travels with the repository), the C
oracle, and the BZ distances of the same codes."""
from __future__ import annotations

import json
import os

import numpy as np
import pytest

from conftest import GOLDEN_DIR
from test_oracle import mitm_case

pytestmark = pytest.mark.gpu


class Native:
    """The B200 library behind the same call shapes as oracle/refbind.py's engines."""

    def __init__(self, native):
        self.n = native

    def classical(self, H, method="bz"):
        return self.n.classical_distance_raw(H, method, "gpu", 0, False)

    def css(self, Hx, Hz, which="M", method="bz"):
        return self.n.css_distance_raw(Hx, Hz, method, which, "gpu", 0, False)

    def subsystem(self, Gx, Gz, which="M", method="bz"):
        return self.n.subsystem_distance_raw(Gx, Gz, method, which, "gpu", 0, False)

    def stabilizer(self, S, which="M", method="bz"):
        return self.n.stabilizer_distance_raw(S, method, which, "gpu", 0, False)

    def operator_weight(self, Gx, Gz, z, x, method="bz"):
        return self.n.operator_weight_raw(Gx, Gz, z, x, method, "gpu", 0, False)

    def pauli_operator_weight(self, G, op, method="bz"):
        return self.n.stabilizer_operator_weight_raw(G, op, method, "gpu", 0, False)


def golden_mitm():
    return json.loads((GOLDEN_DIR / "mitm.json").read_text())


def test_mitm_matches_reference_goldens(native, golden):
    eng = Native(native)
    want = golden_mitm()
    for name, exp in want.items():
        res = golden.results[name]
        got = mitm_case(eng, res["kind"], golden.mats(name), res)
        assert got == exp[:len(got)], (name, got, exp)


def test_mitm_exact_under_forced_tag_collisions(native, golden):
    """With QSFB_MITM_WEAK_TAGS the first table of every weight keeps 4 bits of tag, so
    different syndromes share tags; the build reports it and the tables are rebuilt with
    full tags: the answers stay the reference's."""
    eng = Native(native)
    want = golden_mitm()
    os.environ["QSFB_MITM_WEAK_TAGS"] = "1"
    try:
        for name in ["toric5", "surface5", "batch_512", "noncss_1", "hgp_2x5_x", "opw_1"]:
            res = golden.results[name]
            got = mitm_case(eng, res["kind"], golden.mats(name), res)
            assert got == want[name][:len(got)], name
    finally:
        os.environ.pop("QSFB_MITM_WEAK_TAGS", None)


def test_mitm_equals_reference_on_random_codes(native, orc, ref):
    import codes as C
    from qubitserf_b200 import workloads as W
    eng = Native(native)
    check = ref if ref is not None else orc
    rng = np.random.default_rng(41)
    for trial in range(10):
        n = int(rng.integers(12, 40))
        Hx, Hz = W.css_from_rng(rng, n, int(rng.integers(2, n // 3 + 1)),
                                int(rng.integers(2, n // 3 + 1)))
        for which in "ZXM":
            a = eng.css(Hx, Hz, which, method="mitm")
            b = check.css(Hx, Hz, which, method="mitm")
            assert (a.distance, a.lower_bound, a.proven, a.levels) == \
                   (b.distance, b.lower_bound, b.proven, b.levels), (trial, which)
    for trial in range(8):
        S = C.random_isotropic(rng, int(rng.integers(5, 11)), int(rng.integers(2, 5)))
        a = eng.stabilizer(S, "M", method="mitm")
        b = check.stabilizer(S, "M", method="mitm")
        b = b[1] if isinstance(b, tuple) else b
        assert (a.distance, a.lower_bound, a.proven, a.levels) == \
               (b.distance, b.lower_bound, b.proven, b.levels), trial
        # a Pauli operator outside the group: symplectic coset problem
        op = rng.integers(0, 2, size=S.shape[1], dtype=np.uint8)
        a = eng.pauli_operator_weight(S, op, method="mitm")
        if ref is not None:
            rc, b = ref.pauli_operator_weight(S, op, method="mitm")
            assert rc == 0
        else:
            b = orc.pauli_operator_weight(S, op, method="mitm")
        assert (a.distance, a.proven) == (b.distance, b.proven), trial
    for trial in range(6):
        n = int(rng.integers(10, 30))
        H = rng.integers(0, 2, size=(int(rng.integers(n // 2, n - 2)), n), dtype=np.uint8)
        a = eng.classical(H, method="mitm")
        b = check.classical(H, method="mitm")
        assert (a.distance, a.lower_bound, a.proven, a.levels) == \
               (b.distance, b.lower_bound, b.proven, b.levels), trial


def test_mitm_distance_equals_bz_on_larger_codes(native, golden):
    """Codes past the reference's host-side reach for mitm: the distance is the BZ one
    (golden, made by the reference), proven, and the 'min' interleave stops one level
    under the seed bound as the reference's does on the smaller tori (mitm.json)."""
    eng = Native(native)
    for name, levels in [("toric7", 6), ("surface7", 6)]:
        res = golden.results[name]
        Hx, Hz = golden.mats(name)
        r = eng.css(Hx, Hz, "M", method="mitm")
        assert (r.distance, r.lower_bound, r.proven, r.levels) == \
               (res["distance"], res["distance"], 1, levels), name
    for name in ["batch_513", "batch_517", "batch_523"]:
        res = golden.results[name]
        r = eng.css(*golden.mats(name), "M", method="mitm")
        assert r.distance == res["distance"] and r.proven == 1, name


def test_cc_routes_like_the_reference(native, golden):
    eng = Native(native)
    Hx, Hz = golden.mats("steane")
    with pytest.raises(RuntimeError, match="rc=5"):
        eng.css(Hx, Hz, "M", method="cc")
    # classical: any method but mitm is BZ
    H = golden.mats("hamming4")[0]
    assert eng.classical(H, method="cc").distance == 3

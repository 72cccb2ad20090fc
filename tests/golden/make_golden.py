"""Generate the golden vectors under tests/golden/ from the REFERENCE implementation.

Runs only where the reference CPU library has been built from its sources
(oracle/_ref/libqubitserf.so, see oracle/Makefile).  Outputs:

* golden.npz   -- the input matrices (uint8), keyed by case name
* golden.json  -- per case: the reference's distance / proven flag, and for the
                  no-early-stop cases the reference's per-level (w, active, work) trace
                  read from its DISTFIND_PROFILE lines (cpp/distfind/bz.cpp:147-155)

    python tests/golden/make_golden.py              # golden.npz + golden.json
    python tests/golden/make_golden.py --batch1024  # batch1024.json (all 1024 batch codes)
    python tests/golden/make_golden.py --collect    # collect.npz (codeaut low-weight collector)
    python tests/golden/make_golden.py --mitm       # mitm.json (method "mitm" on the golden codes)

* mitm.json    -- per golden case small enough for the reference's meet-in-the-middle on the
                  host: its [distance, lower_bound, proven, levels] with method "mitm"
                  ([z_weight, x_weight, proven] for operator weights)
* collect.npz  -- per case `<name>__G` (the generator rows), `<name>__meta` (p, keep, combos,
                  count, n) and `<name>__rows` (the reference's collected rows, bit-packed
                  with numpy.packbits along each row), from the reference's own
                  codeaut_bz_collect on its CPU backend (cpp/codeaut/bz.cpp:55-117)
"""
from __future__ import annotations

import json
import os
import re
import subprocess
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "tests"))

import codes as C  # noqa: E402
from qubitserf_b200 import workloads as W  # noqa: E402


def cases():
    """(name, kind, mats, extra) for every golden case."""
    out = []
    out.append(("cfg_classical_96", "classical", (W.single_classical_96(),), {}))
    out.append(("cfg_classical_128", "classical", (W.single_classical_128(),), {}))
    out.append(("cfg_css_128", "css", W.single_css_128(), {"which": "M"}))
    for L in range(3, 7):
        out.append((f"toric{L}", "css", C.toric(L), {"which": "M"}))
    for L in range(3, 6):
        out.append((f"surface{L}", "css", C.surface(L), {"which": "M"}))
    out.append(("surface7", "css", C.surface(7), {"which": "M"}))
    out.append(("toric7", "css", C.toric(7), {"which": "M"}))
    out.append(("steane", "css", C.steane(), {"which": "M"}))
    out.append(("shor", "css", C.shor(), {"which": "M"}))
    out.append(("hgp_2x5", "css", C.hypergraph_product(C.repetition_parity(2),
                                                       C.repetition_parity(5)), {"which": "M"}))
    out.append(("hgp_3x4", "css", C.hypergraph_product(C.repetition_parity(3),
                                                       C.repetition_parity(4)), {"which": "M"}))
    for nm, (Hx, Hz) in (("toric4", C.toric(4)), ("hgp_2x5", C.hypergraph_product(
            C.repetition_parity(2), C.repetition_parity(5)))):
        out.append((nm + "_z", "css", (Hx, Hz), {"which": "Z"}))
        out.append((nm + "_x", "css", (Hx, Hz), {"which": "X"}))
    for n in range(3, 9):
        out.append((f"rep{n}", "classical", (C.repetition_parity(n),), {}))
    out.append(("hamming3", "classical", (C.hamming_parity(3),), {}))
    out.append(("hamming4", "classical", (C.hamming_parity(4),), {}))
    out.append(("qrm_1_9", "css", C.quantum_reed_muller(1, 9), {"which": "M"}))
    out.append(("qrm_1_10", "css", C.quantum_reed_muller(1, 10), {"which": "M"}))
    out.append(("bacon_shor3", "subsystem", C.bacon_shor(3), {"which": "M"}))
    out.append(("bacon_shor4", "subsystem", C.bacon_shor(4), {"which": "M"}))
    out.append(("five_qubit", "stabilizer", (C.five_qubit(),), {"which": "M"}))
    rng = np.random.default_rng(0x5AB)
    for i in range(6):
        n = int(rng.integers(5, 11))
        S = C.random_isotropic(rng, n, int(rng.integers(2, n)))
        if S.shape[0]:
            out.append((f"noncss_{i}", "stabilizer", (S,), {"which": "M"}))
    rng = np.random.default_rng(0x09E12)
    for i in range(8):
        n = int(rng.integers(6, 16))
        Hx, Hz = C.random_css(rng, n, int(rng.integers(1, max(2, n // 2))))
        z = rng.integers(0, 2, n, dtype=np.uint8)
        x = rng.integers(0, 2, n, dtype=np.uint8)
        out.append((f"opw_{i}", "opweight", (Hx, Hz, z, x), {}))
    # first codes of the 1024-code batch (both halves)
    batch = W.batch_1024()
    for i in list(range(0, 12)) + list(range(512, 524)):
        cs = batch[i]
        if cs.kind == "classical":
            out.append((f"batch_{i}", "classical", cs.mats, {}))
        else:
            out.append((f"batch_{i}", "css", cs.mats, {"which": "M"}))
    return out


# Cases re-run with DISTFIND_NO_EARLY_STOP for the per-(information set, w) counts.
COUNT_CASES = ["rep6", "rep8", "hamming4", "toric4_z", "toric4_x", "hgp_2x5_z", "hgp_2x5_x",
               "batch_3"]
COUNT_MAX_K = 24


def run_reference(kind, mats, extra):
    from oracle.refbind import Ref
    ref = Ref()
    if kind == "classical":
        r = ref.classical(mats[0])
        return {"distance": r.distance, "proven": r.proven}
    if kind == "css":
        r = ref.css(mats[0], mats[1], extra.get("which", "M"))
        return {"distance": r.distance, "proven": r.proven}
    if kind == "subsystem":
        r = ref.subsystem(mats[0], mats[1], extra.get("which", "M"))
        return {"distance": r.distance, "proven": r.proven}
    if kind == "stabilizer":
        rc, r = ref.stabilizer(mats[0], extra.get("which", "M"))
        assert rc == 0
        return {"distance": r.distance, "proven": r.proven}
    if kind == "opweight":
        r = ref.operator_weight(*mats)
        return {"z_weight": r.z_weight, "x_weight": r.x_weight}
    raise ValueError(kind)


PROF = re.compile(r"\[prof \w+\] d=(\d+) K=(\d+) ng=(\d+)/(\d+) stride=\d+ total=(\d+) work=(\d+)")


def count_trace(name):
    """Run the reference in a child with no early stop + profiling; parse its level lines."""
    code = (
        "import sys, numpy as np\n"
        f"sys.path.insert(0, {str(ROOT)!r}); sys.path.insert(0, {str(HERE)!r})\n"
        "import make_golden as M\n"
        f"c = [c for c in M.cases() if c[0] == {name!r}][0]\n"
        "M.run_reference(c[1], c[2], c[3])\n"
    )
    env = dict(os.environ, DISTFIND_NO_EARLY_STOP="1", DISTFIND_PROFILE="1")
    p = subprocess.run([sys.executable, "-c", code], env=env, capture_output=True, text=True,
                       check=True)
    levels = []
    for m in PROF.finditer(p.stderr):
        d, K, a, t, total, work = map(int, m.groups())
        levels.append({"w": d, "K": K, "active": a, "num_sets": t, "total": total,
                       "work": work})
    return levels


def batch1024():
    """Reference distance / levels / lower bound / proven for all 1024 batch codes (the
    reference run on this host; levels depend on its core count through the seed streams)."""
    from oracle.refbind import Ref
    import time
    ref = Ref()
    out = []
    t0 = time.perf_counter()
    for c in W.batch_1024():
        r = ref.classical(c.mats[0]) if c.kind == "classical" else ref.css(*c.mats)
        out.append([int(r.distance), int(r.levels), int(r.lower_bound), int(r.proven)])
    meta = {"host_cores": os.cpu_count(), "seconds": time.perf_counter() - t0,
            "fields": ["distance", "levels", "lower_bound", "proven"]}
    (HERE / "batch1024.json").write_text(json.dumps({"meta": meta, "codes": out}))


def systematic(rng, k, n):
    """A random full-rank k x n generator in systematic form on a random column set."""
    while True:
        A = rng.integers(0, 2, size=(k, n - k), dtype=np.uint8)
        G = np.concatenate([np.eye(k, dtype=np.uint8), A], axis=1)
        return G[:, rng.permutation(n)]


def collect_cases():
    """(name, G, p, keep) of the collector's golden cases."""
    rng = np.random.default_rng(11)
    out = []
    H = C.hamming_parity(3)                      # [7,4] Hamming: generator = kernel of H
    G7 = np.array([[1, 0, 0, 0, 0, 1, 1], [0, 1, 0, 0, 1, 0, 1], [0, 0, 1, 0, 1, 1, 0],
                   [0, 0, 0, 1, 1, 1, 1]], np.uint8)
    assert not ((G7 @ H.T) % 2).any()
    out.append(("hamming7", G7, 4, 7))
    out.append(("rm_1_5", C.reed_muller_generator(1, 5), 6, 16))
    out.append(("rm_2_5", C.reed_muller_generator(2, 5), 4, 8))
    out.append(("rm_1_6", C.reed_muller_generator(1, 6), 7, 32))
    out.append(("rep_11", np.ones((1, 11), np.uint8), 3, 11))
    out.append(("sys_40_20", systematic(rng, 20, 40), 4, 10))
    out.append(("sys_96_32", systematic(rng, 32, 96), 4, 24))
    out.append(("sys_130_24", systematic(rng, 24, 130), 3, 50))
    out.append(("sys_200_40", systematic(rng, 40, 200), 3, 80))
    G = rng.integers(0, 2, size=(12, 70), dtype=np.uint8)
    G[3] = 0
    G[7] = G[2]
    G[9] = G[0] ^ G[1]
    out.append(("dependent_12_70", G, 5, 30))
    out.append(("dense_10_64", rng.integers(0, 2, size=(10, 64), dtype=np.uint8), 10, 64))
    out.append(("keep0", systematic(rng, 8, 20), 3, 0))
    out.append(("p_over_m", systematic(rng, 5, 17), 9, 9))
    out.append(("one_col", rng.integers(0, 2, size=(6, 1), dtype=np.uint8), 3, 1))
    return out


def collect_goldens():
    from oracle.refbind import Ref
    ref = Ref()
    arrays = {}
    for name, G, p, keep in collect_cases():
        rows, combos = ref.collect(G, p, keep)
        arrays[f"{name}__G"] = np.asarray(G, np.uint8)
        arrays[f"{name}__meta"] = np.array([p, keep, combos, rows.shape[0], G.shape[1]],
                                           dtype=np.int64)
        arrays[f"{name}__rows"] = np.packbits(rows, axis=1) if rows.size else \
            np.zeros((0, (G.shape[1] + 7) // 8), np.uint8)
        print(name, G.shape, p, keep, "->", rows.shape[0], "rows,", combos, "combos", flush=True)
    np.savez_compressed(HERE / "collect.npz", **arrays)


def mitm_goldens(max_parts=3e7):
    """The reference's own method "mitm" on every golden case whose meet-in-the-middle
    search stays small (parts of the larger half up to its BZ distance)."""
    from math import comb
    from oracle.refbind import Ref
    ref = Ref()
    results = json.loads((HERE / "golden.json").read_text())
    arrays = np.load(HERE / "golden.npz")
    out = {}
    for name, res in sorted(results.items()):
        mats = tuple(arrays[f"{name}__{i}"] for i in range(res["nmats"]))
        kind = res["kind"]
        n = mats[0].shape[1]
        sym = kind == "stabilizer"
        coords = n // 2 if sym else n
        d = res.get("distance")
        if kind == "opweight":
            d = max(res["z_weight"], res["x_weight"])
        half = coords - coords // 2
        parts = sum(comb(half, w) * (3 ** w if sym else 1) for w in range(0, d + 1))
        if d is None or d < 0 or parts > max_parts:
            continue
        if kind == "classical":
            r = ref.classical(mats[0], method="mitm")
        elif kind == "css":
            r = ref.css(mats[0], mats[1], res.get("which", "M"), method="mitm")
        elif kind == "subsystem":
            r = ref.subsystem(mats[0], mats[1], res.get("which", "M"), method="mitm")
        elif kind == "stabilizer":
            rc, r = ref.stabilizer(mats[0], res.get("which", "M"), method="mitm")
            assert rc == 0
        else:
            r = ref.operator_weight(*mats, method="mitm")
            out[name] = [int(r.z_weight), int(r.x_weight), int(r.proven)]
            print(name, out[name], flush=True)
            continue
        out[name] = [int(r.distance), int(r.lower_bound), int(r.proven), int(r.levels)]
        print(name, out[name], flush=True)
    (HERE / "mitm.json").write_text(json.dumps(out, indent=1, sort_keys=True))


def main():
    sys.path.insert(0, str(ROOT))
    if "--mitm" in sys.argv:
        mitm_goldens()
        return
    if "--batch1024" in sys.argv:
        batch1024()
        return
    if "--collect" in sys.argv:
        collect_goldens()
        return
    arrays = {}
    results = {}
    for name, kind, mats, extra in cases():
        for i, m in enumerate(mats):
            arrays[f"{name}__{i}"] = np.asarray(m, dtype=np.uint8)
        res = run_reference(kind, mats, extra)
        res.update({"kind": kind, "nmats": len(mats), **extra})
        results[name] = res
        print(name, res, flush=True)
    for name in COUNT_CASES:
        tr = count_trace(name)
        if tr and max(lv["K"] for lv in tr) <= COUNT_MAX_K:
            results[name]["no_early_stop_levels"] = tr
    np.savez_compressed(HERE / "golden.npz", **arrays)
    (HERE / "golden.json").write_text(json.dumps(results, indent=1, sort_keys=True))


if __name__ == "__main__":
    main()

"""Host-side logic of the engine, no GPU needed: the library loads and exports the ABI,
the host problem reduction reproduces the reference's information sets bit for bit, the
dispatch rules and error codes, and the workload generators."""
from __future__ import annotations

import ctypes
import hashlib
import os
import re
import subprocess
import sys

import numpy as np
import pytest

from conftest import ROOT


def header_functions():
    text = (ROOT / "include" / "qsf_b200.h").read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(distfind_\w+|qsfb_\w+|codeaut_\w+)\s*\(", text)))


def test_library_exports_every_declared_symbol(native):
    names = header_functions()
    assert len(names) >= 15
    lib = native.lib()
    for n in names:
        assert hasattr(lib, n), n
    out = subprocess.run(["nm", "-D", "--defined-only", str(native.LIB_PATH)],
                         capture_output=True, text=True, check=True).stdout
    exported = set(re.findall(r" T (\w+)", out))
    assert set(names) <= exported
    # every binding in the Python layer points at a declared function
    assert {s[0] for s in native.SIGNATURES} == set(names)


def test_struct_layouts_match_reference_abi(native):
    # cpp/distfind/capi.h:12-19 and :39-45 (byte compatible with the reference ctypes)
    assert ctypes.sizeof(native.DistfindResult) == 4 * 4 + 8 + 16
    assert native.DistfindResult.seconds.offset == 16
    assert ctypes.sizeof(native.DistfindOpResult) == 3 * 4 + 4 + 8 + 16
    assert native.DistfindOpResult.seconds.offset == 16


def _collect_handle(native, G, m, n, p, keep, backend):
    L = native.lib()
    ptr = native._p(G) if G is not None else None
    h = L.codeaut_bz_collect(ptr, m, n, p, keep, backend, 0)
    assert h
    try:
        st = native.QsfbCollectStats()
        assert L.qsfb_collect_stats(h, ctypes.byref(st)) == 0
        return (L.codeaut_bz_ok(h), L.codeaut_bz_count(h), L.codeaut_bz_combos(h),
                L.codeaut_bz_backend(h), st.status)
    finally:
        L.codeaut_bz_free(h)


def test_collect_handle_rules_without_device_work(native):
    """The codeaut_bz_* handle answers these before any device work, as the reference's
    does (cpp/codeaut/bz.cpp:55-97, capi.cpp): empty problems are complete with nothing
    collected and no backend named; a nonpositive keep collects nothing but still counts
    every combination (saturating per level at 2^62); backend 0 (cpu) is not run here."""
    G = np.ones((3, 5), np.uint8)
    assert _collect_handle(native, G, 0, 5, 3, 4, 1) == (1, 0, 0, b"", 0)
    assert _collect_handle(native, G, 3, 0, 3, 4, 1) == (1, 0, 0, b"", 0)
    assert _collect_handle(native, G, 3, 5, 0, 4, 1) == (1, 0, 0, b"", 0)
    assert _collect_handle(native, None, 3, 5, 2, 4, 1)[0] == 0          # null G
    ok, cnt, combos, be, status = _collect_handle(native, G, 3, 5, 2, 4, 0)
    assert (ok, cnt, status) == (0, 0, 5)
    G2 = np.zeros((40, 9), np.uint8)
    ok, cnt, combos, be, status = _collect_handle(native, G2, 40, 9, 6, 0, 1)
    assert (ok, cnt, be, status) == (1, 0, b"cuda", 0)
    assert combos == sum(__import__("math").comb(40, s) for s in range(1, 7))
    # p > m: subset sizes stop at m
    ok, cnt, combos, _, _ = _collect_handle(native, G2[:4], 4, 9, 9, -3, 2)
    assert (ok, combos) == (1, 15)
    # C(4000, 30) > 2^62 for every size from 10 up: each level adds the cap, the sum saturates
    G3 = np.zeros((4000, 2), np.uint8)
    ok, _, combos, _, _ = _collect_handle(native, G3, 4000, 2, 30, 0, 1)
    assert (ok, combos) == (1, 1 << 62)
    assert native.lib().codeaut_backend_available(b"cpu") == 0
    assert native.lib().codeaut_version() == b"0.1.0"


def test_version(native):
    assert native.version() == "0.1.0"


def _prep_cases(golden):
    out = []
    for name in ["cfg_classical_96", "cfg_classical_128", "hamming4", "rep6", "batch_0",
                 "batch_5", "batch_11"]:
        out.append((name, 0, golden.mats(name)))
    for name in ["cfg_css_128", "toric4", "surface5", "steane", "shor", "hgp_2x5",
                 "batch_512", "batch_515", "batch_520", "qrm_1_9"]:
        m = golden.mats(name)
        out.append((name + "_Z", 1, m))
        out.append((name + "_X", 2, m))
    for name in ["bacon_shor3", "bacon_shor4"]:
        m = golden.mats(name)
        out.append((name + "_Z", 3, m))
        out.append((name + "_X", 4, m))
    for name in ["five_qubit", "noncss_1", "noncss_4"]:
        out.append((name, 5, golden.mats(name)))
    return out


def test_host_reduction_bit_exact_vs_reference(native, ref, golden):
    """Information-set generators, ranks, detector, parity and seed bound equal the
    reference's (cpp/distfind/bz.cpp:95-115) bit for bit."""
    if ref is None:
        pytest.skip("reference library not built here")
    for name, kind, mats in _prep_cases(golden):
        a = native.prepare_problem(kind, *mats)
        b = ref.problem_gammas(kind, *mats)
        for k in ("n", "K", "stride", "ranks", "even", "count_all", "seed_upper"):
            assert a[k] == b[k], (name, k, a[k], b[k])
        assert np.array_equal(a["gamma"], b["gamma"]), name
        assert np.array_equal(a["check"], b["check"]), name


def test_host_reduction_matches_oracle(native, orc, golden):
    for name, kind, mats in _prep_cases(golden):
        a = native.prepare_problem(kind, *mats)
        b = orc.prepare(kind, *mats)
        assert a["ranks"] == b["ranks"] or sorted(a["ranks"]) == sorted(b["ranks"]), name
        for k in ("n", "K", "even", "count_all", "seed_upper"):
            assert a[k] == b[k], (name, k)


def test_prepare_sides_host_construction(native, golden):
    """The host construction behind qsfb_prepare_sides equals qsfb_prepare_problem, and its
    packed tables have the documented shapes (rows over ceil(n/32) words, syndromes over
    max(1, ceil(kcheck/32))); without a device the device construction fails with rc 4."""
    lib = native.lib()
    for name, kind, mats in _prep_cases(golden):
        a = native.prepare_sides(kind, *mats, on_device=False)
        b = native.prepare_problem(kind, *mats)
        for k in ("n", "K", "stride", "ranks", "even", "count_all", "seed_upper"):
            assert a[k] == b[k], (name, k)
        assert np.array_equal(a["gamma"], b["gamma"]) and np.array_equal(a["check"], b["check"])
        ng = len(a["ranks"])
        assert a["red"].shape == (ng, a["K"], (a["n"] + 31) // 32), name
        assert a["syn"].shape == (ng, a["K"], max(1, (len(a["check"]) + 31) // 32)), name
        assert not a["device"]
        # the pivot columns of every set are zero in the packed rows: each row's weight is
        # its weight outside the set's pivots
        for g in range(ng):
            rows = a["gamma"][g]
            w_full = np.array([sum(bin(int(x)).count("1") for x in r) for r in rows])
            w_red = np.array([sum(bin(int(x)).count("1") for x in r) for r in a["red"][g]])
            piv = np.zeros(a["K"], np.int64)
            piv[: a["ranks"][g]] = 1
            assert np.array_equal(w_full - piv, w_red), (name, g)
    if lib.qsfb_device_sms() == 0:
        with pytest.raises(RuntimeError, match="rc=4:"):
            native.prepare_sides(0, golden.mats("hamming3")[0], on_device=True)


def test_matroid_partition_cases_bit_exact(native, ref):
    """Classical codes where the greedy peel is suboptimal take the matroid partition
    (cpp/distfind/css.cpp:336-366); the chosen sets must still agree exactly."""
    if ref is None:
        pytest.skip("reference library not built here")
    from qubitserf_b200.workloads import classical_parity_from_rng
    rng = np.random.default_rng(11)
    hit = 0
    for _ in range(60):
        n = int(rng.integers(20, 60))
        k = int(rng.integers(n // 4, n // 2 + 1))
        H = classical_parity_from_rng(rng, n, k)
        # sparsify some columns so the greedy peel leaves rank on the table
        H[:, rng.integers(0, n, n // 5)] = 0
        a = native.prepare_problem(0, H)
        b = ref.problem_gammas(0, H)
        assert a["ranks"] == b["ranks"]
        assert np.array_equal(a["gamma"], b["gamma"])
        hit += len(a["ranks"]) > 1
    assert hit > 10


def test_dispatch_rules_without_device(native, golden):
    """No CPU path: without an sm_100 device every distance call fails with rc 4, and the
    unsupported methods/backends with rc 5, before touching any device.  Method "cc" is
    unsupported where the reference runs its connected-cluster solver (CSS, subsystem); the
    classical path maps it to BZ, as the reference does."""
    lib = native.lib()
    H = golden.mats("hamming3")[0]
    a = native.as_u8(H)
    out = native.DistfindResult()
    p = a.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8))
    hx, hz = (native.as_u8(m) for m in golden.mats("steane"))
    px = hx.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8))
    pz = hz.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8))
    for which in (b"Z", b"M"):
        assert lib.distfind_css_distance(px, hx.shape[0], hx.shape[1], pz, hz.shape[0],
                                         hz.shape[1], b"cc", which, b"gpu", 0, 0,
                                         ctypes.byref(out)) == 5
        assert lib.distfind_subsystem_distance(px, hx.shape[0], hx.shape[1], pz, hz.shape[0],
                                               hz.shape[1], b"cc", which, b"gpu", 0, 0,
                                               ctypes.byref(out)) == 5
    assert lib.distfind_classical_distance(p, a.shape[0], a.shape[1], b"bz", b"cpu", 0, 0,
                                           ctypes.byref(out)) == 5
    assert lib.distfind_classical_distance(None, 1, 1, b"bz", b"gpu", 0, 0,
                                           ctypes.byref(out)) == 1
    S = np.zeros((1, 5), np.uint8)
    assert lib.distfind_stabilizer_distance(
        S.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8)), 1, 5, b"bz", b"M", b"gpu", 0, 0,
        ctypes.byref(out)) == 2
    if lib.qsfb_device_sms() == 0:
        assert lib.distfind_backend_available(b"gpu") == 0
        for method in (b"bz", b"mitm", b"cc"):
            rc = lib.distfind_classical_distance(p, a.shape[0], a.shape[1], method, b"gpu", 0,
                                                 0, ctypes.byref(out))
            assert rc == 4
        with pytest.raises(RuntimeError):
            native.classical_distance_raw(H, "bz", "auto", 0, False)
        counters = (ctypes.c_longlong * 4)()
        assert lib.qsfb_alloc_counters(counters) == 4
    assert lib.qsfb_alloc_counters(None) == 1
    assert lib.distfind_backend_available(b"cpu") == 0
    assert lib.distfind_backend_available(b"metal") == 0


@pytest.mark.parametrize("K,stride,d", [
    (128, 2, 32),    # C(128, 16) lists: binomials saturate at 2^64
    (128, 2, 40),
    (128, 2, 64),
    (100, 2, 50),
    (128, 2, 9),     # lists fit 64-bit sizes but not the 32 MiB array
])
def test_noalloc_size_guard_rejects_before_device(native, K, stride, d):
    """The allocation-free level rejects every level its scratch array cannot hold with rc 8
    before any device call, including levels whose binomials saturate (C(K, a) >= 2^64):
    the pointers passed here are placeholders that must never be dereferenced."""
    lib = native.lib()
    fake = ctypes.c_void_p(256)
    rc = lib.qsfb_enumerate_plan_noalloc(64 * stride, stride, K, d, 1, fake, 0, None,
                                         1 << 30, fake, None, None, None, None)
    assert rc == 8


def test_plan_size_guard_rejects_before_device(native):
    """The allocating raw-plan level checks its sizes before it looks for a device: w beyond
    the 64 columns of the binomial table and C(K, w) >= 2^62 give rc 5, subset lists beyond
    2^36 entries rc 6 (C(64, 60) is small, but its prefix list C(64, 30) is not)."""
    rng = np.random.default_rng(3)
    for K, d, want in [(100, 65, 5), (128, 40, 5), (4097, 2, 5), (64, 60, 6)]:
        stride = 2
        gamma = rng.integers(0, 2**63, (1, K, stride), dtype=np.uint64)
        check = np.zeros((0, stride), np.uint64)
        with pytest.raises(RuntimeError, match=f"rc={want}:"):
            native.enumerate_plan(64 * stride, K, d, gamma, check, 1 << 30)


def test_api_argument_validation():
    from qubitserf_b200 import api
    Hx = np.ones((1, 4), np.uint8)
    with pytest.raises(ValueError, match="auto/cpu/gpu"):
        api.css_distance(Hx, Hx, backend="metal")
    with pytest.raises(ValueError, match="min/z/x"):
        api.css_distance(Hx, Hx, which="q")
    with pytest.raises(ValueError):
        api.stabilizer_distance(np.ones((2, 5), np.uint8))
    z, x = api.parse_operator("IXYZ", 4)
    assert list(z) == [0, 0, 1, 1] and list(x) == [0, 1, 1, 0]


def test_workloads_are_deterministic():
    from qubitserf_b200 import workloads as W
    h = lambda a: hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()[:16]
    H1 = W.single_classical_96()
    assert H1.shape == (64, 96) and h(H1) == h(W.single_classical_96())
    Hx, Hz = W.single_css_128()
    assert Hx.shape == (40, 128) and Hz.shape == (40, 128)
    assert not (W.gf2_matmul(Hx, Hz.T)).any()
    assert W.gf2_rank(Hx) == 40 and W.gf2_rank(Hz) == 40
    b = W.batch_1024(8)
    assert [c.kind for c in b] == ["classical"] * 4 + ["css"] * 4


def _cli(args, stdin=""):
    exe = ROOT / "qubitserf_b200" / "qsfb-distfind"
    p = subprocess.run([str(exe), *args], input=stdin, capture_output=True, text=True,
                       timeout=120)
    return p.returncode, p.stdout, p.stderr


def test_cli_usage_errors_exit_2(tmp_path):
    """qsfb-distfind accepts the reference CLI's inputs (cpp/distfind/cli/
    distfind_cli.cpp:100-188: CSS Pauli strings on stdin, 0/1 matrix files): malformed input
    and usage errors exit 2 with a message on stderr, before any device work."""
    rc, out, _ = _cli(["--help"])
    assert rc == 0 and out.startswith("Usage: qsfb-distfind")
    for args, stdin, msg in [
        (["--frobnicate"], "", "unrecognised argument"),
        (["--zx", "--z"], "XXI\n", "--zx cannot be combined"),
        (["--hx", "a.txt"], "", "--hx and --hz must be given together"),
        ([], "", "no generator lines on stdin"),
        ([], "XXZ\n", "input line 1: not a pure X or pure Z generator"),
        ([], "IXI\nXYI\n", "input line 2: not a pure X or pure Z generator"),
        ([], "XXI\nZZ\n", "input line 2: length 2, the first line has 3"),
        ([], "XQI\n", "input line 1: character 'Q' is not a Pauli letter"),
        (["-o", "XX"], "XXI\n", "operator has length 2, the generators 3"),
        (["-o", "XW"], "XI\n", "operator: character 'W' is not a Pauli letter"),
        (["--threads", "x"], "", "non-negative integer"),
    ]:
        rc, out, err = _cli(args, stdin)
        assert rc == 2 and msg in err and out == "", (args, err)
    bad = tmp_path / "ragged.txt"
    bad.write_text("1 0 1\n\n0 1\n")
    good = tmp_path / "good.txt"
    good.write_text("1 1 0\n")
    rc, _, err = _cli(["--hx", str(bad), "--hz", str(good)])
    assert rc == 2 and "ragged.txt: line 3 has 2 entries, line 1 has 3" in err
    two = tmp_path / "two.txt"
    two.write_text("1 2 0\n")
    rc, _, err = _cli(["--hx", str(two), "--hz", str(good)])
    assert rc == 2 and "two.txt: line 1: entry '2' is not 0 or 1" in err
    glued = tmp_path / "glued.txt"
    glued.write_text("10 1\n")
    rc, _, err = _cli(["--hx", str(glued), "--hz", str(good)])
    assert rc == 2 and "entry '10' is not 0 or 1" in err
    empty = tmp_path / "empty.txt"
    empty.write_text("\n \n")
    rc, _, err = _cli(["--hx", str(empty), "--hz", str(good)])
    assert rc == 2 and "empty.txt: no rows" in err
    narrow = tmp_path / "narrow.txt"
    narrow.write_text("1 1\n")
    rc, _, err = _cli(["--hx", str(good), "--hz", str(narrow)])
    assert rc == 2 and "--hx has 3 columns, --hz 2" in err


def test_cli_without_device_fails_cleanly(native):
    if native.lib().qsfb_device_sms() != 0:
        pytest.skip("a device is present")
    rc, out, err = _cli([], "XXXXIII\nZZZZIII\n")
    assert rc == 1 and out == "" and "rc=4" in err


def test_reference_python_binds_the_drop_in(native):
    """The reference's unmodified Python package (copied beside its libraries under
    oracle/_ref) loads this library through QUBITSERF_LIB and binds every distfind_*
    signature; without a device, backend "gpu" is refused by its own check, "cpu" comes
    back as rc 5 and "auto" as rc 4, both RuntimeError (python/qubitserf/distfind/
    _native.py:132-133, api.py:66-72)."""
    ref_py = ROOT / "oracle" / "_ref" / "python"
    if not (ref_py / "qubitserf" / "distfind" / "api.py").exists():
        pytest.skip("the reference Python package was not copied under oracle/_ref")
    script = (
        "import sys, json, numpy as np\n"
        "sys.path.insert(0, sys.argv[1])\n"
        "from qubitserf import distfind as df\n"
        "from qubitserf.distfind import _native as N\n"
        "H = np.array([[1,1,0,1,1,0,0],[1,0,1,1,0,1,0],[0,1,1,1,0,0,1]], np.uint8)\n"
        "out = {'version': df.version(), 'backends': df.available_backends()}\n"
        "for b in ('gpu', 'cpu', 'auto'):\n"
        "    try:\n"
        "        df.classical_distance(H, backend=b); out[b] = 'ok'\n"
        "    except RuntimeError as e:\n"
        "        out[b] = str(e)\n"
        "print(json.dumps(out))\n")
    env = dict(os.environ, QUBITSERF_LIB=str(native.LIB_PATH))
    p = subprocess.run([sys.executable, "-c", script, str(ref_py)], env=env,
                       capture_output=True, text=True, timeout=120)
    assert p.returncode == 0, p.stderr
    out = __import__("json").loads(p.stdout.strip().splitlines()[-1])
    assert out["version"] == "0.1.0"
    if native.lib().qsfb_device_sms() == 0:
        assert out["backends"] == ["cpu"]
        assert "no GPU backend" in out["gpu"]
        assert "rc=5" in out["cpu"] and "rc=4" in out["auto"]
    else:
        assert "gpu" in out["backends"] and out["gpu"] == "ok" and "rc=5" in out["cpu"]


def test_tuning_table_and_overrides(native, tmp_path):
    """The library reads its launch shapes once: defaults, then a `key value` table
    (QSFB_TUNING, else tuning.txt beside the library), then QSFB_TUNE_<KEY> overrides;
    unknown keys and malformed lines are ignored, values are clamped to their ranges."""
    import json
    table = tmp_path / "t.txt"
    table.write_text("# comment\ntc_shape 0\ntc_job_tiles.large 8  # trailing\n"
                     "cc_jobs_per_warp 9999\nbogus 3\ntc_cost_ratio x\nbatch_chunks 6\n"
                     "batch_first_permille 5000\n")
    code = ("import sys, json; sys.path.insert(0, sys.argv[1]); "
            "from qubitserf_b200 import _native as N; print(json.dumps(N.tuning()))")
    env = dict(os.environ, QSFB_TUNING=str(table), QSFB_TUNE_EXEC_GROUPS="2",
               QSFB_TUNE_TC_JOB_TILES_SMALL="4")
    p = subprocess.run([sys.executable, "-c", code, str(ROOT)], env=env, capture_output=True,
                       text=True, timeout=120)
    assert p.returncode == 0, p.stderr
    t = json.loads(p.stdout.strip().splitlines()[-1])
    assert (t["tc_shape"], t["tc_job_tiles.large"], t["batch_chunks"]) == (0, 8, 6)
    assert t["cc_jobs_per_warp"] == 256 and t["tc_cost_ratio"] == 0.6   # clamped / kept
    assert t["batch_first_permille"] == 1000                              # clamped
    assert (t["exec_groups"], t["tc_job_tiles.small"]) == (2, 4)
    assert str(table) in t["source"] and "QSFB_TUNE_EXEC_GROUPS" in t["source"]
    env = dict(os.environ, QSFB_TUNING=str(tmp_path / "absent.txt"))
    p = subprocess.run([sys.executable, "-c", code, str(ROOT)], env=env, capture_output=True,
                       text=True, timeout=120)
    assert json.loads(p.stdout.strip().splitlines()[-1])["source"] == "defaults"

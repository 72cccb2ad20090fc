"""ctypes binding to libqsfb200.so (the C ABI in include/qsf_b200.h).

The distfind_* part mirrors the reference's python/qubitserf/distfind/_native.py:15-258
(same structs, argtypes and rc -> exception mapping); the qsfb_* part exposes the engine
extras (raw-plan enumeration, host reduction, witness, per-level counts, batch).
The library is loaded in-tree; importing this module never builds anything and raises if
the library is missing.
"""
from __future__ import annotations

import ctypes
import os
from pathlib import Path

import numpy as np

PKG = Path(__file__).resolve().parent
LIB_PATH = Path(os.environ.get("QSFB_LIB", PKG / "libqsfb200.so"))

ERRORS = {
    1: "null pointer",
    2: "not a [z|x] matrix / bad operator length",
    3: "method 'cc' is not supported for non-CSS codes",
    4: "no usable sm_100 device, or a CUDA error",
    5: "unsupported method/backend/size on the B200 engine",
    6: "device memory exhausted",
    7: "output buffer too small",
    8: "beyond the fixed scratch of the no-allocation entry point",
}


class DistfindResult(ctypes.Structure):
    _fields_ = [("distance", ctypes.c_int), ("lower_bound", ctypes.c_int),
                ("proven", ctypes.c_int), ("levels", ctypes.c_int),
                ("seconds", ctypes.c_double), ("backend", ctypes.c_char * 16)]


class DistfindOpResult(ctypes.Structure):
    _fields_ = [("z_weight", ctypes.c_int), ("x_weight", ctypes.c_int),
                ("proven", ctypes.c_int), ("seconds", ctypes.c_double),
                ("backend", ctypes.c_char * 16)]


class QsfbReport(ctypes.Structure):
    _fields_ = [("distance", ctypes.c_int), ("lower_bound", ctypes.c_int),
                ("proven", ctypes.c_int), ("levels", ctypes.c_int),
                ("witness_ok", ctypes.c_int), ("witness_bits", ctypes.c_int),
                ("witness_side", ctypes.c_int), ("kernel_launches", ctypes.c_int),
                ("seconds", ctypes.c_double), ("device_ms", ctypes.c_double),
                ("codewords", ctypes.c_ulonglong)]


class QsfbQuery(ctypes.Structure):
    _fields_ = [("kind", ctypes.c_int), ("which", ctypes.c_char),
                ("A", ctypes.POINTER(ctypes.c_uint8)), ("a_rows", ctypes.c_int),
                ("a_cols", ctypes.c_int), ("B", ctypes.POINTER(ctypes.c_uint8)),
                ("b_rows", ctypes.c_int), ("b_cols", ctypes.c_int),
                ("z_op", ctypes.POINTER(ctypes.c_uint8)), ("x_op", ctypes.POINTER(ctypes.c_uint8))]


class QsfbAnswer(ctypes.Structure):
    _fields_ = [("distance", ctypes.c_int), ("z_weight", ctypes.c_int),
                ("x_weight", ctypes.c_int), ("lower_bound", ctypes.c_int),
                ("proven", ctypes.c_int), ("levels", ctypes.c_int),
                ("witness_ok", ctypes.c_int)]


class QsfbBatchStats(ctypes.Structure):
    _fields_ = [("seconds", ctypes.c_double), ("prepare_seconds", ctypes.c_double),
                ("host_setup_seconds", ctypes.c_double), ("device_seed_seconds", ctypes.c_double),
                ("device_ms", ctypes.c_double), ("device_span_ms", ctypes.c_double),
                ("pair_ms", ctypes.c_double), ("codewords", ctypes.c_ulonglong),
                ("popc_issued", ctypes.c_ulonglong), ("zero_codewords", ctypes.c_ulonglong),
                ("rounds", ctypes.c_int), ("kernel_launches", ctypes.c_int),
                ("certificates", ctypes.c_int), ("device_bytes", ctypes.c_longlong),
                ("gen_ms", ctypes.c_double), ("host_plan_seconds", ctypes.c_double),
                ("host_apply_seconds", ctypes.c_double), ("tc_codewords", ctypes.c_ulonglong),
                ("tc_ms", ctypes.c_double), ("device_sets_seconds", ctypes.c_double),
                ("tc_operand_bytes", ctypes.c_ulonglong),
                ("list_bytes_written", ctypes.c_ulonglong)]


class QsfbTiming(ctypes.Structure):
    _fields_ = [("submit_s", ctypes.c_double), ("ready_s", ctypes.c_double),
                ("admit_s", ctypes.c_double), ("done_s", ctypes.c_double),
                ("latency_s", ctypes.c_double)]


class QsfbServeStats(ctypes.Structure):
    _fields_ = [("submitted", ctypes.c_longlong), ("completed", ctypes.c_longlong),
                ("active", ctypes.c_int), ("pending", ctypes.c_int),
                ("busy_s", ctypes.c_double), ("codewords", ctypes.c_ulonglong),
                ("rounds", ctypes.c_int), ("peak_footprint_bytes", ctypes.c_longlong),
                ("elapsed_s", ctypes.c_double)]


class QsfbCollectStats(ctypes.Structure):
    _fields_ = [("combos", ctypes.c_int64), ("hits", ctypes.c_int64), ("passes", ctypes.c_int64),
                ("probe_words", ctypes.c_int32), ("filter", ctypes.c_int32),
                ("pivots", ctypes.c_int32),
                ("launches", ctypes.c_int32), ("reruns", ctypes.c_int32),
                ("gen_ms", ctypes.c_double), ("pairs_ms", ctypes.c_double),
                ("seconds", ctypes.c_double), ("status", ctypes.c_int32)]


# (name, restype, argtypes) of every exported function; tests check the export list.
_u8p = ctypes.POINTER(ctypes.c_uint8)
_u64p = ctypes.POINTER(ctypes.c_uint64)
_u32p = ctypes.POINTER(ctypes.c_uint32)
_ip = ctypes.POINTER(ctypes.c_int)
_ullp = ctypes.POINTER(ctypes.c_ulonglong)
_rp = ctypes.POINTER(DistfindResult)
_i, _c, _s, _d = ctypes.c_int, ctypes.c_char, ctypes.c_char_p, ctypes.c_double
SIGNATURES = [
    ("distfind_css_distance", _i, [_u8p, _i, _i, _u8p, _i, _i, _s, _c, _s, _i, _i, _rp]),
    ("distfind_classical_distance", _i, [_u8p, _i, _i, _s, _s, _i, _i, _rp]),
    ("distfind_operator_weight", _i, [_u8p, _i, _i, _u8p, _i, _i, _u8p, _u8p, _i, _s, _s, _i, _i,
                                      ctypes.POINTER(DistfindOpResult)]),
    ("distfind_subsystem_distance", _i, [_u8p, _i, _i, _u8p, _i, _i, _s, _c, _s, _i, _i, _rp]),
    ("distfind_stabilizer_distance", _i, [_u8p, _i, _i, _s, _c, _s, _i, _i, _rp]),
    ("distfind_subsystem_stabilizer_distance", _i, [_u8p, _i, _i, _s, _c, _s, _i, _i, _rp]),
    ("distfind_stabilizer_operator_weight", _i, [_u8p, _i, _i, _u8p, _i, _s, _s, _i, _i, _rp]),
    ("distfind_backend_available", _i, [_s]),
    ("distfind_version", _s, []),
    ("qsfb_enumerate_plan", _i, [_i, _i, _i, _i, _i, _u64p, _i, _u64p, _i, _ip, _ullp, _ip,
                                 _ullp]),
    ("qsfb_prepare_problem", _i, [_i, _u8p, _i, _i, _u8p, _i, _i, _ip, _ip, _i, _u64p,
                                  ctypes.c_longlong, _u64p, ctypes.c_longlong]),
    ("qsfb_prepare_sides", _i, [_i, _u8p, _i, _i, _u8p, _i, _i, _i, _ip, _ip, _i, _u64p,
                                ctypes.c_longlong, _u64p, ctypes.c_longlong, _u32p,
                                ctypes.c_longlong, _u32p, ctypes.c_longlong]),
    ("qsfb_last_report", _i, [ctypes.POINTER(QsfbReport)]),
    ("qsfb_tuning", _i, [ctypes.c_char_p, _i]),
    ("qsfb_last_witness", _i, [_u8p, _i]),
    ("qsfb_last_counts", _i, [_ip, _ip, _ip, _ullp, _i]),
    ("qsfb_batch", _i, [ctypes.POINTER(QsfbQuery), _i, _i, ctypes.POINTER(QsfbAnswer),
                        ctypes.POINTER(QsfbBatchStats)]),
    ("qsfb_batch_prepare", _i, [ctypes.POINTER(QsfbQuery), _i, _i,
                                ctypes.POINTER(ctypes.c_void_p)]),
    ("qsfb_batch_execute", _i, [ctypes.c_void_p, ctypes.POINTER(QsfbAnswer),
                                ctypes.POINTER(QsfbBatchStats)]),
    ("qsfb_batch_free", None, [ctypes.c_void_p]),
    ("qsfb_enumerate_plan_noalloc", _i, [_i, _i, _i, _i, _i, ctypes.c_void_p, _i,
                                         ctypes.c_void_p, _i, ctypes.c_void_p, ctypes.c_void_p,
                                         ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]),
    ("qsfb_server_start", _i, [_i, ctypes.c_longlong, _i, ctypes.POINTER(ctypes.c_void_p)]),
    ("qsfb_server_submit", _i, [ctypes.c_void_p, ctypes.POINTER(QsfbQuery),
                                ctypes.POINTER(ctypes.c_longlong)]),
    ("qsfb_server_wait", _i, [ctypes.c_void_p, ctypes.c_longlong, ctypes.POINTER(QsfbAnswer),
                              ctypes.POINTER(QsfbTiming)]),
    ("qsfb_server_stats", _i, [ctypes.c_void_p, ctypes.POINTER(QsfbServeStats)]),
    ("qsfb_server_stop", _i, [ctypes.c_void_p]),
    ("qsfb_microbench", _i, [_i, ctypes.POINTER(ctypes.c_double)]),
    ("qsfb_flush_l2", _i, []),
    ("qsfb_tc_selftest", _i, [_i, _i, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]),
    ("qsfb_device_name", _s, []),
    ("qsfb_device_sms", _i, []),
    ("qsfb_alloc_counters", _i, [ctypes.POINTER(ctypes.c_longlong)]),
    ("codeaut_bz_collect", ctypes.c_void_p, [_u8p, ctypes.c_int32, ctypes.c_int32,
                                             ctypes.c_int32, ctypes.c_int32, ctypes.c_int32,
                                             ctypes.c_int32]),
    ("codeaut_bz_ok", ctypes.c_int32, [ctypes.c_void_p]),
    ("codeaut_bz_count", ctypes.c_int64, [ctypes.c_void_p]),
    ("codeaut_bz_combos", ctypes.c_int64, [ctypes.c_void_p]),
    ("codeaut_bz_copy_rows", None, [ctypes.c_void_p, _u8p]),
    ("codeaut_bz_backend", _s, [ctypes.c_void_p]),
    ("codeaut_bz_free", None, [ctypes.c_void_p]),
    ("codeaut_backend_available", ctypes.c_int32, [_s]),
    ("codeaut_version", _s, []),
    ("qsfb_collect_stats", _i, [ctypes.c_void_p, ctypes.POINTER(QsfbCollectStats)]),
]

_lib = None


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise RuntimeError(f"{LIB_PATH} is missing: run `python -m qubitserf_b200.build`")
        L = ctypes.CDLL(str(LIB_PATH))
        for name, res, args in SIGNATURES:
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def _check(rc: int, what: str):
    if rc == 3:
        raise ValueError("method 'cc' (connected cluster) is not supported for non-CSS "
                         "codes; use 'bz' or 'mitm'")
    if rc != 0:
        raise RuntimeError(f"{what} failed (rc={rc}: {ERRORS.get(rc, 'error')})")


def as_u8(mat) -> np.ndarray:
    a = np.ascontiguousarray(np.asarray(mat, dtype=np.uint8) & 1)
    if a.ndim != 2:
        raise ValueError("expected a 2D 0/1 matrix")
    return a


def as_u8_vec(v) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(v, dtype=np.uint8) & 1).reshape(-1)


def _p(a):
    return a.ctypes.data_as(_u8p)


def css_distance_raw(Hx, Hz, method, which, backend, threads, verbose):
    ax, az = as_u8(Hx), as_u8(Hz)
    out = DistfindResult()
    rc = lib().distfind_css_distance(_p(ax), ax.shape[0], ax.shape[1], _p(az), az.shape[0],
                                     az.shape[1], method.encode(), which.encode()[:1] or b"M",
                                     backend.encode(), int(threads), 1 if verbose else 0,
                                     ctypes.byref(out))
    _check(rc, "distfind_css_distance")
    return out


def classical_distance_raw(H, method, backend, threads, verbose):
    a = as_u8(H)
    out = DistfindResult()
    rc = lib().distfind_classical_distance(_p(a), a.shape[0], a.shape[1], method.encode(),
                                           backend.encode(), int(threads), 1 if verbose else 0,
                                           ctypes.byref(out))
    _check(rc, "distfind_classical_distance")
    return out


def operator_weight_raw(Gx, Gz, z_op, x_op, method, backend, threads, verbose):
    ax, az = as_u8(Gx), as_u8(Gz)
    z, x = as_u8_vec(z_op), as_u8_vec(x_op)
    n = ax.shape[1]
    if az.shape[1] != n:
        raise ValueError("Gx and Gz must have the same number of columns (n)")
    if z.shape[0] != n or x.shape[0] != n:
        raise ValueError("z_op and x_op must be length n = %d" % n)
    out = DistfindOpResult()
    rc = lib().distfind_operator_weight(_p(ax), ax.shape[0], ax.shape[1], _p(az), az.shape[0],
                                        az.shape[1], _p(z), _p(x), n, method.encode(),
                                        backend.encode(), int(threads), 1 if verbose else 0,
                                        ctypes.byref(out))
    _check(rc, "distfind_operator_weight")
    return out


def subsystem_distance_raw(Gx, Gz, method, which, backend, threads, verbose):
    ax, az = as_u8(Gx), as_u8(Gz)
    out = DistfindResult()
    rc = lib().distfind_subsystem_distance(_p(ax), ax.shape[0], ax.shape[1], _p(az),
                                           az.shape[0], az.shape[1], method.encode(),
                                           which.encode()[:1] or b"M", backend.encode(),
                                           int(threads), 1 if verbose else 0, ctypes.byref(out))
    _check(rc, "distfind_subsystem_distance")
    return out


def stabilizer_distance_raw(S, method, which, backend, threads, verbose):
    a = as_u8(S)
    if a.shape[1] % 2 != 0:
        raise ValueError("symplectic stabilizer matrix must have 2n (even) columns")
    out = DistfindResult()
    rc = lib().distfind_stabilizer_distance(_p(a), a.shape[0], a.shape[1], method.encode(),
                                            which.encode()[:1] or b"M", backend.encode(),
                                            int(threads), 1 if verbose else 0, ctypes.byref(out))
    _check(rc, "distfind_stabilizer_distance")
    return out


def subsystem_stabilizer_distance_raw(G, method, which, backend, threads, verbose):
    a = as_u8(G)
    if a.shape[1] % 2 != 0:
        raise ValueError("symplectic gauge matrix must have 2n (even) columns")
    out = DistfindResult()
    rc = lib().distfind_subsystem_stabilizer_distance(_p(a), a.shape[0], a.shape[1],
                                                      method.encode(),
                                                      which.encode()[:1] or b"M",
                                                      backend.encode(), int(threads),
                                                      1 if verbose else 0, ctypes.byref(out))
    _check(rc, "distfind_subsystem_stabilizer_distance")
    return out


def stabilizer_operator_weight_raw(G, op, method, backend, threads, verbose):
    a = as_u8(G)
    o = as_u8_vec(op)
    if a.shape[1] % 2 != 0:
        raise ValueError("symplectic gauge matrix must have 2n (even) columns")
    if o.shape[0] != a.shape[1]:
        raise ValueError("operator must be a length-2n symplectic [z|x] vector")
    out = DistfindResult()
    rc = lib().distfind_stabilizer_operator_weight(_p(a), a.shape[0], a.shape[1], _p(o),
                                                   o.shape[0], method.encode(), backend.encode(),
                                                   int(threads), 1 if verbose else 0,
                                                   ctypes.byref(out))
    _check(rc, "distfind_stabilizer_operator_weight")
    return out


def backend_available(name: str) -> bool:
    return bool(lib().distfind_backend_available(name.encode()))


def version() -> str:
    return lib().distfind_version().decode()


# ---------------------------------------------------------------- engine extras
def enumerate_plan(n, K, d, gamma, check, current_best):
    """One level on a raw plan (gamma: [ng, K, stride] uint64, check: [kcheck, stride])."""
    stride = (n + 63) // 64
    g = np.ascontiguousarray(gamma, dtype=np.uint64).reshape(-1)
    ng = g.size // (K * stride)
    c = np.ascontiguousarray(check, dtype=np.uint64).reshape(-1)
    kcheck = c.size // stride
    cbuf = c if c.size else np.zeros(1, np.uint64)
    best = ctypes.c_int(0)
    counts = np.zeros(ng, dtype=np.uint64)
    og = ctypes.c_int(-1)
    orank = ctypes.c_ulonglong(0)
    rc = lib().qsfb_enumerate_plan(n, stride, K, d, ng, g.ctypes.data_as(_u64p), kcheck,
                                   cbuf.ctypes.data_as(_u64p), int(current_best),
                                   ctypes.byref(best), counts.ctypes.data_as(_ullp),
                                   ctypes.byref(og), ctypes.byref(orank))
    _check(rc, "qsfb_enumerate_plan")
    return best.value, counts, og.value, orank.value


def prepare_problem(kind, A, B=None):
    a = as_u8(A)
    b = as_u8(B) if B is not None else np.zeros((0, a.shape[1]), np.uint8)
    meta = (ctypes.c_int * 8)()
    ncol = a.shape[1] * 3 // 2 if kind == 5 else a.shape[1]
    stride = (ncol + 63) // 64
    maxg = ncol + 2
    ranks = (ctypes.c_int * maxg)()
    gamma = np.zeros(maxg * ncol * stride + 1, dtype=np.uint64)
    check = np.zeros(ncol * stride + 1, dtype=np.uint64)
    rc = lib().qsfb_prepare_problem(kind, _p(a), a.shape[0], a.shape[1],
                                    _p(b) if b.size else None, b.shape[0], b.shape[1], meta,
                                    ranks, maxg, gamma.ctypes.data_as(_u64p), gamma.size,
                                    check.ctypes.data_as(_u64p), check.size)
    _check(rc, "qsfb_prepare_problem")
    n, K, ng, kcheck, even, count_all, seed_upper, stride = list(meta)
    return {"n": n, "K": K, "stride": stride, "ranks": [ranks[i] for i in range(ng)],
            "gamma": gamma[: ng * K * stride].reshape(ng, K, stride).copy(),
            "check": check[: kcheck * stride].reshape(kcheck, stride).copy(),
            "even": bool(even), "count_all": bool(count_all), "seed_upper": seed_upper}


def prepare_sides(kind, A, B=None, on_device=True):
    """The subproblem's information sets built on the device (on_device) or the host, with
    the packed non-pivot rows and detector syndromes the pair sweeps read."""
    a = as_u8(A)
    b = as_u8(B) if B is not None else np.zeros((0, a.shape[1]), np.uint8)
    meta = (ctypes.c_int * 12)()
    ncol = a.shape[1] * 3 // 2 if kind == 5 else a.shape[1]
    stride = (ncol + 63) // 64
    w32 = (ncol + 31) // 32
    maxg = ncol + 2
    ranks = (ctypes.c_int * maxg)()
    gamma = np.zeros(maxg * ncol * stride + 1, dtype=np.uint64)
    check = np.zeros(ncol * stride + 1, dtype=np.uint64)
    red = np.zeros(maxg * ncol * w32 + 1, dtype=np.uint32)
    syn = np.zeros(maxg * ncol * max(1, (ncol + 31) // 32) + 1, dtype=np.uint32)
    rc = lib().qsfb_prepare_sides(kind, _p(a), a.shape[0], a.shape[1],
                                  _p(b) if b.size else None, b.shape[0], b.shape[1],
                                  1 if on_device else 0, meta, ranks, maxg,
                                  gamma.ctypes.data_as(_u64p), gamma.size,
                                  check.ctypes.data_as(_u64p), check.size,
                                  red.ctypes.data_as(_u32p), red.size,
                                  syn.ctypes.data_as(_u32p), syn.size)
    _check(rc, "qsfb_prepare_sides")
    n, K, ng, kcheck, even, count_all, seed_upper, stride, W32, SWP, on_dev, classes = list(meta)
    return {"n": n, "K": K, "stride": stride, "ranks": [ranks[i] for i in range(ng)],
            "gamma": gamma[: ng * K * stride].reshape(ng, K, stride).copy(),
            "check": check[: kcheck * stride].reshape(kcheck, stride).copy(),
            "red": red[: ng * K * W32].reshape(ng, K, W32).copy(),
            "syn": syn[: ng * K * SWP].reshape(ng, K, SWP).copy(),
            "even": bool(even), "count_all": bool(count_all), "seed_upper": seed_upper,
            "device": bool(on_dev), "classes": bool(classes)}


def tuning() -> dict:
    """The launch shapes in effect and their source (the tuning table, or defaults)."""
    buf = ctypes.create_string_buffer(4096)
    _check(lib().qsfb_tuning(buf, len(buf)), "qsfb_tuning")
    out = {}
    for line in buf.value.decode().splitlines():
        key, _, val = line.partition(" ")
        try:
            out[key] = int(val)
        except ValueError:
            try:
                out[key] = float(val)
            except ValueError:
                out[key] = val
    return out


def last_report() -> QsfbReport:
    r = QsfbReport()
    lib().qsfb_last_report(ctypes.byref(r))
    return r


def last_witness():
    n = lib().qsfb_last_witness(None, 0)
    if n < 0:
        return None
    buf = np.zeros(n, dtype=np.uint8)
    lib().qsfb_last_witness(_p(buf), n)
    return buf


def last_counts():
    n = lib().qsfb_last_counts(None, None, None, None, 0)
    side = (ctypes.c_int * max(n, 1))()
    w = (ctypes.c_int * max(n, 1))()
    g = (ctypes.c_int * max(n, 1))()
    cnt = (ctypes.c_ulonglong * max(n, 1))()
    lib().qsfb_last_counts(side, w, g, cnt, n)
    return [(side[i], w[i], g[i], int(cnt[i])) for i in range(n)]


class Batch:
    """Queries prepared once (contiguous uint8 host matrices) and certified together with
    qsfb_batch.  Each item: ("classical", H) | ("css", Hx, Hz[, which]) |
    ("opweight", Gx, Gz, z, x)."""

    KINDS = {"classical": 0, "css": 1, "opweight": 2}

    def __init__(self, items):
        self._keep = []
        self.n = len(items)
        self.q = (QsfbQuery * max(1, self.n))()
        self.host_bytes = 0
        for i, it in enumerate(items):
            kind = it[0]
            Q = self.q[i]
            Q.kind = self.KINDS[kind]
            A = as_u8(it[1])
            self._keep.append(A)
            Q.A, Q.a_rows, Q.a_cols = _p(A), A.shape[0], A.shape[1]
            self.host_bytes += A.size
            Q.which = b"M"
            if kind in ("css", "opweight"):
                B = as_u8(it[2])
                self._keep.append(B)
                Q.B, Q.b_rows, Q.b_cols = _p(B), B.shape[0], B.shape[1]
                self.host_bytes += B.size
            if kind == "css" and len(it) > 3:
                Q.which = it[3].encode()[:1]
            if kind == "opweight":
                z, x = as_u8_vec(it[3]), as_u8_vec(it[4])
                self._keep += [z, x]
                Q.z_op, Q.x_op = _p(z), _p(x)
                self.host_bytes += z.size + x.size
        self.out = (QsfbAnswer * max(1, self.n))()

    def run(self, host_threads=0):
        """One-shot certification from the host matrices (prepare + execute + free)."""
        st = QsfbBatchStats()
        rc = lib().qsfb_batch(self.q, self.n, int(host_threads), self.out, ctypes.byref(st))
        _check(rc, "qsfb_batch")
        return [self.out[i] for i in range(self.n)], st

    def prepare(self, host_threads=0):
        """Host setup + upload; returns a handle for execute()/free()."""
        h = ctypes.c_void_p()
        rc = lib().qsfb_batch_prepare(self.q, self.n, int(host_threads), ctypes.byref(h))
        _check(rc, "qsfb_batch_prepare")
        return h

    def execute(self, handle):
        st = QsfbBatchStats()
        rc = lib().qsfb_batch_execute(handle, self.out, ctypes.byref(st))
        _check(rc, "qsfb_batch_execute")
        return [self.out[i] for i in range(self.n)], st

    @staticmethod
    def free(handle):
        lib().qsfb_batch_free(handle)


def batch_items(codes):
    """workloads.CodeSpec list -> Batch items (CSS codes with which='min')."""
    items = []
    for cs in codes:
        if cs.kind == "classical":
            items.append(("classical", cs.mats[0]))
        elif cs.kind == "css":
            items.append(("css", cs.mats[0], cs.mats[1], "M"))
        else:
            items.append(("opweight",) + tuple(cs.mats))
    return items


def make_query(item):
    """One QsfbQuery (plus the arrays it points into) from a Batch-style item."""
    b = Batch([item])
    return b.q[0], b._keep


class Server:
    """Continuous-batching server (qsfb_server_*): submit() returns a ticket at once,
    wait() blocks for that ticket's answer and timing."""

    def __init__(self, intake_threads=0, mem_budget_bytes=0, max_active=0):
        self.h = ctypes.c_void_p()
        _check(lib().qsfb_server_start(int(intake_threads), int(mem_budget_bytes),
                                       int(max_active), ctypes.byref(self.h)), "qsfb_server_start")

    def submit(self, item):
        q, keep = make_query(item)
        t = ctypes.c_longlong()
        _check(lib().qsfb_server_submit(self.h, ctypes.byref(q), ctypes.byref(t)),
               "qsfb_server_submit")
        del keep   # the server copied the matrices
        return t.value

    def wait(self, ticket):
        a = QsfbAnswer()
        tm = QsfbTiming()
        _check(lib().qsfb_server_wait(self.h, ticket, ctypes.byref(a), ctypes.byref(tm)),
               "qsfb_server_wait")
        return a, tm

    def stats(self):
        st = QsfbServeStats()
        lib().qsfb_server_stats(self.h, ctypes.byref(st))
        return st

    def stop(self):
        if self.h:
            rc = lib().qsfb_server_stop(self.h)
            self.h = ctypes.c_void_p()
            _check(rc, "qsfb_server_stop")


def microbench(which):
    """Measured device-wide ops/s: 0 = POPC (XU pipe), 1 = LOP3 (ALU pipe)."""
    v = ctypes.c_double()
    _check(lib().qsfb_microbench(int(which), ctypes.byref(v)), "qsfb_microbench")
    return v.value


def alloc_counters():
    """Driver-level allocations so far: (device allocations, their seconds, pinned staging
    allocations, their seconds)."""
    v = (ctypes.c_longlong * 4)()
    _check(lib().qsfb_alloc_counters(v), "qsfb_alloc_counters")
    return v[0], v[1] * 1e-9, v[2], v[3] * 1e-9


def tc_selftest(ksteps, A, B, packed=False):
    """D = A[:, :32k] @ B[:, :32k].T (int32, 256 x 128) through the tensor-core sweep's own
    copy / MMA / TMEM path; A is 256 x 64 and B 128 x 64 int8.  packed: read back as the
    sweep does (16-bit halves).  ksteps = -1 is the timeout drill (raises RuntimeError with
    rc 4)."""
    A = np.ascontiguousarray(A, dtype=np.int8)
    B = np.ascontiguousarray(B, dtype=np.int8)
    if A.shape != (256, 64) or B.shape != (128, 64):
        raise ValueError("tc_selftest: A must be 256 x 64 and B 128 x 64 int8")
    D = np.zeros((256, 128), dtype=np.int32)
    _check(lib().qsfb_tc_selftest(int(ksteps), int(bool(packed)), A.ctypes.data, B.ctypes.data,
                                  D.ctypes.data), "qsfb_tc_selftest")
    return D


_COLLECT_BACKEND = {"cpu": 0, "gpu": 1, "auto": 2}


def collect(G, p, keep_weight, backend="gpu", threads=0, stats=False):
    """Every distinct codeword of weight 1..keep_weight that is the XOR of a size-1..p subset
    of the rows of G, as the reference's ``_collect_one_native`` returns them
    (python/qubitserf/codeaut/lowweight.py:53-78): ``(rows uint8[count, n], combos)``, rows
    sorted by their packed 64-bit words.  Raises RuntimeError when the handle is not ok
    (backend "cpu", sizes beyond the engine's, no device).  stats=True appends the
    QsfbCollectStats of the run."""
    L = lib()
    G = as_u8(G)
    m, n = G.shape
    be = _COLLECT_BACKEND.get(backend, backend)
    h = L.codeaut_bz_collect(_p(G) if G.size else None, m, n, int(p), int(keep_weight),
                             int(be), int(threads))
    if not h:
        raise RuntimeError("codeaut_bz_collect failed (no handle)")
    try:
        st = QsfbCollectStats()
        L.qsfb_collect_stats(h, ctypes.byref(st))
        if not L.codeaut_bz_ok(h):
            raise RuntimeError(f"codeaut_bz_collect failed (rc={st.status}: "
                               f"{ERRORS.get(st.status, 'error')})")
        cnt = int(L.codeaut_bz_count(h))
        combos = int(L.codeaut_bz_combos(h))
        rows = np.zeros((max(cnt, 1), n), dtype=np.uint8)
        if cnt:
            L.codeaut_bz_copy_rows(h, _p(rows))
        rows = rows[:cnt]
    finally:
        L.codeaut_bz_free(h)
    return (rows, combos, st) if stats else (rows, combos)

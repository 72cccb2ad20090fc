"""ctypes binding to the checkers under oracle/ (TEST INFRASTRUCTURE ONLY).

* ``Ref``    -- the reference's own CPU library, built from its sources into
  ``oracle/_ref/libqubitserf.so`` by ``oracle/Makefile``; its ``distfind_*`` ABI is the
  one in the reference's ``cpp/distfind/capi.h:12-111``, plus the two shim entry points of
  ``oracle/ref_shim.cpp``.
* ``RefCuda`` -- the same sources with the reference's own CUDA backend
  (``cpp/qsf/cuda/backend_cuda.cu``) compiled for sm_100a, as its CMake build does when a
  CUDA toolkit is present (``CMakeLists.txt:86-90``): ``oracle/_ref/libqubitserf_cuda.so``,
  called with ``backend="gpu"``.  It is the plain per-code GPU path that the batched
  engine is compared with.
* ``Oracle`` -- the C restatement ``oracle/libbzoracle.so`` (``oracle/bz_oracle.c``).

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s baseline legs import this
module, and only as the checker or the timed comparator.  The product library never loads
any of these files.
"""
from __future__ import annotations

import ctypes
import os
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
REF_LIB = HERE / "_ref" / "libqubitserf.so"
REF_CUDA_LIB = HERE / "_ref" / "libqubitserf_cuda.so"
ORACLE_LIB = HERE / "libbzoracle.so"

WEIGHT_NONE = 1 << 30


class DistfindResult(ctypes.Structure):
    _fields_ = [("distance", ctypes.c_int), ("lower_bound", ctypes.c_int),
                ("proven", ctypes.c_int), ("levels", ctypes.c_int),
                ("seconds", ctypes.c_double), ("backend", ctypes.c_char * 16)]


class DistfindOpResult(ctypes.Structure):
    _fields_ = [("z_weight", ctypes.c_int), ("x_weight", ctypes.c_int),
                ("proven", ctypes.c_int), ("seconds", ctypes.c_double),
                ("backend", ctypes.c_char * 16)]


def u8(a):
    a = np.ascontiguousarray(np.asarray(a, dtype=np.uint8) & 1)
    return a


def _p(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8))


def _u64p(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64))


def unpack_rows(packed, n):
    """0/1 rows of n columns from rows of little-endian 64-bit words (bit j of word w is
    column 64 w + j)."""
    packed = np.ascontiguousarray(packed, dtype=np.uint64)
    if packed.shape[0] == 0:
        return np.zeros((0, n), dtype=np.uint8)
    bits = np.unpackbits(packed.view(np.uint8).reshape(packed.shape[0], -1), axis=1,
                         bitorder="little")
    return bits[:, :n].copy()


def ref_available() -> bool:
    return REF_LIB.exists()


class Ref:
    """The reference library on its CPU backend."""

    backend = b"cpu"

    def __init__(self, path: Path = REF_LIB):
        self.lib = ctypes.CDLL(str(path), mode=os.RTLD_LOCAL)
        L = self.lib
        u8p = ctypes.POINTER(ctypes.c_uint8)
        rp = ctypes.POINTER(DistfindResult)
        L.distfind_classical_distance.argtypes = [u8p, ctypes.c_int, ctypes.c_int,
                                                  ctypes.c_char_p, ctypes.c_char_p,
                                                  ctypes.c_int, ctypes.c_int, rp]
        L.distfind_css_distance.argtypes = [u8p, ctypes.c_int, ctypes.c_int, u8p, ctypes.c_int,
                                            ctypes.c_int, ctypes.c_char_p, ctypes.c_char,
                                            ctypes.c_char_p, ctypes.c_int, ctypes.c_int, rp]
        L.distfind_subsystem_distance.argtypes = L.distfind_css_distance.argtypes
        L.distfind_operator_weight.argtypes = [u8p, ctypes.c_int, ctypes.c_int, u8p,
                                               ctypes.c_int, ctypes.c_int, u8p, u8p,
                                               ctypes.c_int, ctypes.c_char_p, ctypes.c_char_p,
                                               ctypes.c_int, ctypes.c_int,
                                               ctypes.POINTER(DistfindOpResult)]
        L.distfind_stabilizer_distance.argtypes = [u8p, ctypes.c_int, ctypes.c_int,
                                                   ctypes.c_char_p, ctypes.c_char,
                                                   ctypes.c_char_p, ctypes.c_int,
                                                   ctypes.c_int, rp]
        L.distfind_subsystem_stabilizer_distance.argtypes = L.distfind_stabilizer_distance.argtypes
        L.distfind_stabilizer_operator_weight.argtypes = [u8p, ctypes.c_int, ctypes.c_int, u8p,
                                                          ctypes.c_int, ctypes.c_char_p,
                                                          ctypes.c_char_p, ctypes.c_int,
                                                          ctypes.c_int, rp]
        L.ref_enumerate.restype = ctypes.c_int
        L.ref_enumerate.argtypes = [ctypes.c_int] * 5 + [ctypes.POINTER(ctypes.c_uint64),
                                                         ctypes.c_int,
                                                         ctypes.POINTER(ctypes.c_uint64),
                                                         ctypes.c_int, ctypes.c_int]
        L.ref_problem_gammas.argtypes = [ctypes.c_int, u8p, ctypes.c_int, ctypes.c_int, u8p,
                                         ctypes.c_int, ctypes.c_int,
                                         ctypes.POINTER(ctypes.c_int),
                                         ctypes.POINTER(ctypes.c_int), ctypes.c_int,
                                         ctypes.POINTER(ctypes.c_uint64), ctypes.c_longlong,
                                         ctypes.POINTER(ctypes.c_uint64), ctypes.c_longlong]

    def classical(self, H, threads=0, method="bz"):
        a = u8(H)
        out = DistfindResult()
        rc = self.lib.distfind_classical_distance(_p(a), a.shape[0], a.shape[1], method.encode(), self.backend,
                                                  threads, 0, ctypes.byref(out))
        assert rc == 0
        return out

    def css(self, Hx, Hz, which="M", threads=0, method="bz"):
        ax, az = u8(Hx), u8(Hz)
        out = DistfindResult()
        rc = self.lib.distfind_css_distance(_p(ax), ax.shape[0], ax.shape[1], _p(az),
                                            az.shape[0], az.shape[1], method.encode(), which.encode(),
                                            self.backend, threads, 0, ctypes.byref(out))
        assert rc == 0
        return out

    def subsystem(self, Gx, Gz, which="M", threads=0, method="bz"):
        ax, az = u8(Gx), u8(Gz)
        out = DistfindResult()
        rc = self.lib.distfind_subsystem_distance(_p(ax), ax.shape[0], ax.shape[1], _p(az),
                                                  az.shape[0], az.shape[1], method.encode(),
                                                  which.encode(), self.backend, threads, 0,
                                                  ctypes.byref(out))
        assert rc == 0
        return out

    def operator_weight(self, Gx, Gz, z, x, threads=0, method="bz"):
        ax, az = u8(Gx), u8(Gz)
        zz, xx = u8(z).reshape(-1), u8(x).reshape(-1)
        out = DistfindOpResult()
        rc = self.lib.distfind_operator_weight(_p(ax), ax.shape[0], ax.shape[1], _p(az),
                                               az.shape[0], az.shape[1], _p(zz), _p(xx),
                                               ax.shape[1], method.encode(), self.backend, threads, 0,
                                               ctypes.byref(out))
        assert rc == 0
        return out

    def stabilizer(self, S, which="M", threads=0, method="bz"):
        a = u8(S)
        out = DistfindResult()
        rc = self.lib.distfind_stabilizer_distance(_p(a), a.shape[0], a.shape[1], method.encode(),
                                                   which.encode(), self.backend, threads, 0,
                                                   ctypes.byref(out))
        return rc, out

    def subsystem_stabilizer(self, G, which="M", threads=0, method="bz"):
        a = u8(G)
        out = DistfindResult()
        rc = self.lib.distfind_subsystem_stabilizer_distance(_p(a), a.shape[0], a.shape[1],
                                                             method.encode(), which.encode(), self.backend,
                                                             threads, 0, ctypes.byref(out))
        return rc, out

    def pauli_operator_weight(self, G, op, threads=0, method="bz"):
        a = u8(G)
        o = u8(op).reshape(-1)
        out = DistfindResult()
        rc = self.lib.distfind_stabilizer_operator_weight(_p(a), a.shape[0], a.shape[1], _p(o),
                                                          o.shape[0], method.encode(), self.backend, threads, 0,
                                                          ctypes.byref(out))
        return rc, out

    def enumerate(self, n, stride, K, d, gamma, check, current_best, threads=0):
        g = np.ascontiguousarray(gamma, dtype=np.uint64)
        c = np.ascontiguousarray(check, dtype=np.uint64)
        ng = g.size // (K * stride)
        kcheck = c.size // stride
        if c.size == 0:
            c = np.zeros(1, dtype=np.uint64)
        return self.lib.ref_enumerate(n, stride, K, d, ng, _u64p(g), kcheck, _u64p(c),
                                      int(current_best), threads)

    def problem_gammas(self, kind, A, B=None):
        """Return dict(n, K, ranks, gamma[ng,K,stride], check[kcheck,stride], even,
        count_all, seed_upper) exactly as the reference's bz_distance sees them."""
        a = u8(A)
        b = u8(B) if B is not None else np.zeros((0, a.shape[1]), np.uint8)
        meta = (ctypes.c_int * 8)()
        n_est = a.shape[1] * (3 if kind == 5 else 1) // (2 if kind == 5 else 1) + 64
        stride_est = (n_est + 63) // 64 + 1
        maxg = max(4, n_est + 2)
        ranks = (ctypes.c_int * maxg)()
        K_est = n_est
        gamma = np.zeros(maxg * K_est * stride_est, dtype=np.uint64)
        check = np.zeros(K_est * stride_est + 1, dtype=np.uint64)
        rc = self.lib.ref_problem_gammas(kind, _p(a), a.shape[0], a.shape[1],
                                         _p(b) if b.size else None, b.shape[0], b.shape[1],
                                         meta, ranks, maxg, _u64p(gamma), gamma.size,
                                         _u64p(check), check.size)
        assert rc == 0, "buffer too small"
        n, K, ng, kcheck, even, count_all, seed_upper, stride = list(meta)
        return {
            "n": n, "K": K, "stride": stride, "ranks": [ranks[i] for i in range(ng)],
            "gamma": gamma[: ng * K * stride].reshape(ng, K, stride).copy(),
            "check": check[: kcheck * stride].reshape(kcheck, stride).copy(),
            "even": bool(even), "count_all": bool(count_all), "seed_upper": seed_upper,
        }


    def collect(self, G, p, keep, threads=0):
        """The reference's codeaut low-weight collector (``codeaut_bz_collect``,
        cpp/codeaut/bz.cpp:55-117) on its CPU backend: ``(rows uint8[count, n], combos)``."""
        L = self.lib
        vp = ctypes.c_void_p
        L.codeaut_bz_collect.restype = vp
        L.codeaut_bz_collect.argtypes = [ctypes.POINTER(ctypes.c_uint8)] + [ctypes.c_int32] * 6
        for name, rt in (("codeaut_bz_ok", ctypes.c_int32), ("codeaut_bz_count", ctypes.c_int64),
                         ("codeaut_bz_combos", ctypes.c_int64)):
            getattr(L, name).restype = rt
            getattr(L, name).argtypes = [vp]
        L.codeaut_bz_copy_rows.restype = None
        L.codeaut_bz_copy_rows.argtypes = [vp, ctypes.POINTER(ctypes.c_uint8)]
        L.codeaut_bz_free.restype = None
        L.codeaut_bz_free.argtypes = [vp]
        g = u8(G)
        m, n = g.shape
        h = L.codeaut_bz_collect(_p(g), m, n, int(p), int(keep), 0, int(threads))
        try:
            assert L.codeaut_bz_ok(h) == 1
            cnt = int(L.codeaut_bz_count(h))
            rows = np.zeros((max(cnt, 1), n), dtype=np.uint8)
            if cnt:
                L.codeaut_bz_copy_rows(h, _p(rows))
            return rows[:cnt], int(L.codeaut_bz_combos(h))
        finally:
            L.codeaut_bz_free(h)

class RefCuda(Ref):
    """The reference library built with its CUDA backend, called with backend "gpu": its
    levels of at least 2^18 codewords run on ``bz_enumerate`` (``backend_cuda.cu:133-205``),
    smaller ones on its CPU backend (``backend_cuda.cu:518-521``)."""

    backend = b"gpu"

    def __init__(self, path: Path = REF_CUDA_LIB):
        super().__init__(path)
        self.lib.distfind_backend_available.argtypes = [ctypes.c_char_p]
        self.lib.distfind_backend_available.restype = ctypes.c_int

    def available(self) -> bool:
        return self.lib.distfind_backend_available(b"gpu") == 1


class OrcResult(ctypes.Structure):
    _fields_ = [("distance", ctypes.c_int), ("lower_bound", ctypes.c_int),
                ("proven", ctypes.c_int), ("levels", ctypes.c_int),
                ("codewords", ctypes.c_ulonglong)]


class OrcOptions(ctypes.Structure):
    _fields_ = [("no_early_stop", ctypes.c_int), ("seed_trials", ctypes.c_int),
                ("cap", ctypes.c_int), ("levels_w", ctypes.POINTER(ctypes.c_int)),
                ("levels_active", ctypes.POINTER(ctypes.c_int)),
                ("levels_side", ctypes.POINTER(ctypes.c_int)), ("mitm", ctypes.c_int)]


class Oracle:
    """The C restatement (oracle/bz_oracle.c).  Results carry distance, lower_bound,
    proven, levels and the summed level work; ``trace`` (when requested) lists
    (side, w, active) of every enumerated level."""

    def __init__(self, path: Path = ORACLE_LIB):
        self.lib = ctypes.CDLL(str(path), mode=os.RTLD_LOCAL)
        L = self.lib
        u8p = ctypes.POINTER(ctypes.c_uint8)
        op = ctypes.POINTER(OrcOptions)
        rp = ctypes.POINTER(OrcResult)
        i = ctypes.c_int
        L.orc_enumerate.restype = i
        L.orc_enumerate.argtypes = [i, i, i, i, i, ctypes.POINTER(ctypes.c_uint64), i,
                                    ctypes.POINTER(ctypes.c_uint64), i,
                                    ctypes.POINTER(ctypes.c_ulonglong), ctypes.POINTER(i),
                                    ctypes.POINTER(ctypes.c_ulonglong)]
        L.orc_enumerate_fast.restype = i
        L.orc_enumerate_fast.argtypes = [i, i, i, i, i, ctypes.POINTER(ctypes.c_uint64), i,
                                         ctypes.POINTER(ctypes.c_uint64), i]
        L.orc_classical_distance.argtypes = [u8p, i, i, op, rp]
        L.orc_css_distance.argtypes = [u8p, i, i, u8p, i, i, ctypes.c_char, op, rp]
        L.orc_subsystem_distance.argtypes = [u8p, i, i, u8p, i, i, ctypes.c_char, op, rp]
        L.orc_operator_weight.argtypes = [u8p, i, i, u8p, i, i, u8p, u8p, op,
                                          ctypes.POINTER(i), ctypes.POINTER(i)]
        L.orc_stabilizer_distance.argtypes = [u8p, i, i, i, ctypes.c_char, op, rp]
        L.orc_pauli_operator_weight.argtypes = [u8p, i, i, u8p, op, rp]
        L.orc_prepare.argtypes = [i, u8p, i, i, u8p, i, i, ctypes.POINTER(i),
                                  ctypes.POINTER(i), i]

    @staticmethod
    def _opts(no_early_stop=False, seed_trials=0, trace_cap=0, method="bz"):
        o = OrcOptions()
        o.mitm = 1 if method == "mitm" else 0
        o.no_early_stop = 1 if no_early_stop else 0
        o.seed_trials = seed_trials
        bufs = None
        if trace_cap:
            bufs = [(ctypes.c_int * trace_cap)() for _ in range(3)]
            o.cap = trace_cap
            o.levels_w, o.levels_active, o.levels_side = [
                ctypes.cast(b, ctypes.POINTER(ctypes.c_int)) for b in bufs]
        return o, bufs

    @staticmethod
    def _trace(res, bufs):
        if bufs is None:
            return None
        n = min(res.levels * 2 + 2, len(bufs[0]))
        out = []
        for k in range(len(bufs[0])):
            if bufs[0][k] == 0:
                break
            out.append((bufs[2][k], bufs[0][k], bufs[1][k]))
        return out

    def enumerate(self, n, K, d, gamma, check, current_best):
        stride = (n + 63) // 64
        g = np.ascontiguousarray(gamma, dtype=np.uint64).reshape(-1)
        c = np.ascontiguousarray(check, dtype=np.uint64).reshape(-1)
        ng = g.size // (K * stride)
        kc = c.size // stride
        cb = c if c.size else np.zeros(1, np.uint64)
        counts = np.zeros(ng, dtype=np.uint64)
        ag = ctypes.c_int(-1)
        ar = ctypes.c_ulonglong(0)
        best = self.lib.orc_enumerate(n, stride, K, d, ng, _u64p(g), kc, _u64p(cb),
                                      int(current_best),
                                      counts.ctypes.data_as(ctypes.POINTER(ctypes.c_ulonglong)),
                                      ctypes.byref(ag), ctypes.byref(ar))
        return best, counts, ag.value, ar.value

    def enumerate_fast(self, n, K, d, gamma, check, current_best):
        stride = (n + 63) // 64
        g = np.ascontiguousarray(gamma, dtype=np.uint64).reshape(-1)
        c = np.ascontiguousarray(check, dtype=np.uint64).reshape(-1)
        ng = g.size // (K * stride)
        kc = c.size // stride
        cb = c if c.size else np.zeros(1, np.uint64)
        return self.lib.orc_enumerate_fast(n, stride, K, d, ng, _u64p(g), kc, _u64p(cb),
                                           int(current_best))

    def classical(self, H, **kw):
        a = u8(H)
        o, bufs = self._opts(**kw)
        r = OrcResult()
        self.lib.orc_classical_distance(_p(a), a.shape[0], a.shape[1], ctypes.byref(o),
                                        ctypes.byref(r))
        r.trace = self._trace(r, bufs)
        return r

    def css(self, Hx, Hz, which="M", **kw):
        ax, az = u8(Hx), u8(Hz)
        o, bufs = self._opts(**kw)
        r = OrcResult()
        self.lib.orc_css_distance(_p(ax), ax.shape[0], ax.shape[1], _p(az), az.shape[0],
                                  az.shape[1], which.encode(), ctypes.byref(o), ctypes.byref(r))
        r.trace = self._trace(r, bufs)
        return r

    def subsystem(self, Gx, Gz, which="M", **kw):
        ax, az = u8(Gx), u8(Gz)
        o, bufs = self._opts(**kw)
        r = OrcResult()
        self.lib.orc_subsystem_distance(_p(ax), ax.shape[0], ax.shape[1], _p(az), az.shape[0],
                                        az.shape[1], which.encode(), ctypes.byref(o),
                                        ctypes.byref(r))
        return r

    def operator_weight(self, Gx, Gz, z, x, **kw):
        ax, az = u8(Gx), u8(Gz)
        zz, xx = u8(z).reshape(-1), u8(x).reshape(-1)
        o, _ = self._opts(**kw)
        zw, xw = ctypes.c_int(0), ctypes.c_int(0)
        self.lib.orc_operator_weight(_p(ax), ax.shape[0], ax.shape[1], _p(az), az.shape[0],
                                     az.shape[1], _p(zz), _p(xx), ctypes.byref(o),
                                     ctypes.byref(zw), ctypes.byref(xw))
        return zw.value, xw.value

    def stabilizer(self, S, which="M", subsystem=False, **kw):
        a = u8(S)
        o, _ = self._opts(**kw)
        r = OrcResult()
        self.lib.orc_stabilizer_distance(_p(a), a.shape[0], a.shape[1], 1 if subsystem else 0,
                                         which.encode(), ctypes.byref(o), ctypes.byref(r))
        return r

    def pauli_operator_weight(self, G, op, **kw):
        a = u8(G)
        v = u8(op).reshape(-1)
        o, _ = self._opts(**kw)
        r = OrcResult()
        self.lib.orc_pauli_operator_weight(_p(a), a.shape[0], a.shape[1], _p(v),
                                           ctypes.byref(o), ctypes.byref(r))
        return r

    def prepare(self, kind, A, B=None):
        a = u8(A)
        b = u8(B) if B is not None else np.zeros((0, a.shape[1]), np.uint8)
        meta = (ctypes.c_int * 8)()
        ranks = (ctypes.c_int * (3 * a.shape[1] + 4))()
        self.lib.orc_prepare(kind, _p(a), a.shape[0], a.shape[1], _p(b) if b.size else None,
                             b.shape[0], b.shape[1], meta, ranks, len(ranks))
        m = list(meta)
        return {"n": m[0], "K": m[1], "ranks": [ranks[i] for i in range(m[2])],
                "kcheck": m[3], "even": bool(m[4]), "count_all": bool(m[5]),
                "seed_upper": m[6]}

    def collect(self, G, p, keep):
        """The C restatement of the codeaut collector: ``(rows uint8[count, n], combos)``."""
        L = self.lib
        pp = ctypes.POINTER(ctypes.c_uint64)
        L.orc_collect.restype = ctypes.c_longlong
        L.orc_collect.argtypes = [ctypes.POINTER(ctypes.c_uint8), ctypes.c_int, ctypes.c_int,
                                  ctypes.c_int, ctypes.c_int, ctypes.POINTER(pp),
                                  ctypes.POINTER(ctypes.c_longlong)]
        L.orc_free.restype = None
        L.orc_free.argtypes = [ctypes.c_void_p]
        g = u8(G)
        m, n = g.shape
        out = pp()
        combos = ctypes.c_longlong(0)
        cnt = L.orc_collect(_p(g) if g.size else None, m, n, int(p), int(keep),
                            ctypes.byref(out), ctypes.byref(combos))
        assert cnt >= 0
        s = (n + 63) // 64
        try:
            packed = (np.ctypeslib.as_array(out, shape=(cnt * s,)).copy() if cnt
                      else np.zeros(0, np.uint64))
        finally:
            L.orc_free(ctypes.cast(out, ctypes.c_void_p))
        return unpack_rows(packed.reshape(cnt, s), n), int(combos.value)

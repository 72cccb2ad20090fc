"""Distance API of the B200 engine, mirroring the reference's
python/qubitserf/distfind/api.py:75-251 (same names, keyword arguments, return values and
exceptions).  Every call runs on the GPU; ``backend`` accepts "auto"/"gpu" ("cpu" raises:
this engine has no CPU path); ``method`` "bz" runs Brouwer-Zimmermann, "mitm" the
meet-in-the-middle syndrome join, "cc" (connected cluster) raises where the reference would
run its cc solver and falls back as the reference does elsewhere.
"""
from __future__ import annotations

import numpy as np

from . import _native

_WHICH = {"min": "M", "m": "M", "z": "Z", "x": "X"}
_BACKENDS = {"auto", "cpu", "gpu"}


def parse_operator(s: str, n: int):
    """Pauli string -> (z_vec, x_vec); I . _ space are identity, Y sets both supports."""
    s = s.strip().rstrip("\r")
    if len(s) != n:
        raise ValueError("operator has length %d, expected n = %d" % (len(s), n))
    z = np.zeros(n, dtype=np.uint8)
    x = np.zeros(n, dtype=np.uint8)
    for j, ch in enumerate(s):
        if ch in "I._ ":
            continue
        if ch in "Xx":
            x[j] = 1
        elif ch in "Zz":
            z[j] = 1
        elif ch in "Yy":
            x[j] = 1
            z[j] = 1
        else:
            raise ValueError("operator has an unrecognised character %r" % ch)
    return z, x


def _as_css(Hx, Hz):
    if Hz is not None:
        return np.asarray(Hx), np.asarray(Hz)
    if isinstance(Hx, (tuple, list)) and len(Hx) == 2:
        return np.asarray(Hx[0]), np.asarray(Hx[1])
    for a, b in (("Hx", "Hz"),):
        if hasattr(Hx, a) and hasattr(Hx, b):
            return np.asarray(getattr(Hx, a)), np.asarray(getattr(Hx, b))
    raise TypeError("expected (Hx, Hz) or a CSS code object")


def _as_symplectic(S):
    a = np.ascontiguousarray(np.asarray(S, dtype=np.uint8) & 1)
    if a.ndim != 2 or a.shape[1] % 2 != 0:
        raise ValueError("expected a 2D symplectic matrix with 2n (even) columns "
                         "in [z | x] order")
    return a


def _parse_operator(operator, n):
    if isinstance(operator, str):
        return parse_operator(operator, n)
    if isinstance(operator, (tuple, list)) and len(operator) == 2:
        z = np.asarray(operator[0], dtype=np.uint8).reshape(-1) & 1
        x = np.asarray(operator[1], dtype=np.uint8).reshape(-1) & 1
        if z.shape[0] != n or x.shape[0] != n:
            raise ValueError("(z_vec, x_vec) must each have length n = %d" % n)
        return z, x
    a = np.asarray(operator, dtype=np.uint8).reshape(-1) & 1
    if a.shape[0] != 2 * n:
        raise ValueError("symplectic operator must have length 2n = %d" % (2 * n))
    return a[:n].copy(), a[n:].copy()


def _normalize_backend(backend) -> str:
    b = "auto" if backend is None else str(backend).lower()
    if b not in _BACKENDS:
        raise ValueError("backend must be one of auto/cpu/gpu")
    if b == "gpu" and not _native.backend_available("gpu"):
        raise RuntimeError("no GPU backend is available on this machine")
    return b


def _which(which):
    w = _WHICH.get(str(which).lower())
    if w is None:
        raise ValueError("which must be one of min/z/x")
    return w


def css_distance(Hx, Hz=None, *, method="bz", which="min", backend="auto", threads=0,
                 verbose=False) -> int:
    Hx, Hz = _as_css(Hx, Hz)
    w = _which(which)
    b = _normalize_backend(backend)
    return int(_native.css_distance_raw(Hx, Hz, method, w, b, threads, verbose).distance)


def subsystem_css_distance(Gx, Gz=None, *, method="bz", which="min", backend="auto", threads=0,
                           verbose=False) -> int:
    Gx, Gz = _as_css(Gx, Gz)
    w = _which(which)
    b = _normalize_backend(backend)
    return int(_native.subsystem_distance_raw(Gx, Gz, method, w, b, threads, verbose).distance)


def operator_weight(Gx, Gz, operator, *, method="bz", backend="auto", threads=0,
                    verbose=False) -> int:
    Gx, Gz = _as_css(Gx, Gz)
    n = Gx.shape[1]
    if Gz.shape[1] != n:
        raise ValueError("Gx and Gz must have the same number of columns (n)")
    z, x = _parse_operator(operator, n)
    b = _normalize_backend(backend)
    r = _native.operator_weight_raw(Gx, Gz, z, x, method, b, threads, verbose)
    return max(int(r.z_weight), int(r.x_weight))


def stabilizer_distance(S, *, method="bz", which="min", backend="auto", threads=0,
                        verbose=False) -> int:
    S = _as_symplectic(S)
    w = _which(which)
    b = _normalize_backend(backend)
    return int(_native.stabilizer_distance_raw(S, method, w, b, threads, verbose).distance)


def subsystem_stabilizer_distance(G, *, method="bz", which="min", backend="auto", threads=0,
                                  verbose=False) -> int:
    G = _as_symplectic(G)
    w = _which(which)
    b = _normalize_backend(backend)
    return int(_native.subsystem_stabilizer_distance_raw(G, method, w, b, threads,
                                                         verbose).distance)


def pauli_operator_weight(G, operator, *, method="bz", backend="auto", threads=0,
                          verbose=False) -> int:
    G = _as_symplectic(G)
    n = G.shape[1] // 2
    if isinstance(operator, str):
        z, x = parse_operator(operator, n)
        op = np.concatenate([z, x]).astype(np.uint8)
    else:
        z, x = _parse_operator(operator, n)
        op = np.concatenate([z, x]).astype(np.uint8)
    b = _normalize_backend(backend)
    return int(_native.stabilizer_operator_weight_raw(G, op, method, b, threads,
                                                      verbose).distance)


def classical_distance(H, *, method="bz", backend="auto", threads=0, verbose=False) -> int:
    b = _normalize_backend(backend)
    return int(_native.classical_distance_raw(H, method, b, threads, verbose).distance)


def available_backends():
    out = []
    if _native.backend_available("gpu"):
        out.append("gpu")
    return out


def version() -> str:
    return _native.version()

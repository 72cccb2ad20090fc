"""Seeded synthetic inputs for the BZ distance engine.

All codes are random binary matrices drawn with ``numpy.random.default_rng(seed)`` and
Bernoulli(1/2) entries (``rng.integers(0, 2, size, dtype=uint8)``).  There is no public
benchmark suite behind them; the shapes follow the five workloads the engine is measured
on:

* ``single_classical_96``   -- a [96, 32] code, G = [I_32 | R], seed 0, passed as H = [R^T | I_64].
* ``single_css_128``        -- CSS n=128: Hx 40x128 (full rank), Hz = C . N with N a basis of
  ker(Hx) and C 40x88 random, rank 40 (so Hx Hz^T = 0, k = 48), seed 1.
* ``single_classical_128``  -- a [128, 40] code, seed 2.
* ``batch_1024``            -- 1024 uneven codes, seed 3: 512 classical (n in [48,128],
  k in [n/4, n/2]) then 512 CSS (n in [40,128], rank(Hx), rank(Hz) in [n/5, n/3]).
* ``serving_stream``        -- a Poisson request stream, seed 4 (40% classical, 40% CSS,
  20% CSS operator weight).

The GF(2) helpers here are plain row-reduction over uint8 arrays (canonical RREF
nullspace basis: one vector per free column, pivot coordinates from the RREF column).
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np


# --------------------------------------------------------------------------- GF(2) helpers
def gf2_rref(M):
    """Reduced row-echelon form over GF(2); returns (R, pivot_columns)."""
    R = (np.asarray(M, dtype=np.uint8) & 1).copy()
    rows, cols = R.shape
    piv = []
    r = 0
    for c in range(cols):
        if r == rows:
            break
        nz = np.nonzero(R[r:, c])[0]
        if nz.size == 0:
            continue
        s = r + int(nz[0])
        if s != r:
            R[[r, s]] = R[[s, r]]
        hit = np.nonzero(R[:, c])[0]
        hit = hit[hit != r]
        if hit.size:
            R[hit] ^= R[r]
        piv.append(c)
        r += 1
    return R, piv


def gf2_rank(M) -> int:
    M = np.asarray(M)
    if M.size == 0:
        return 0
    return len(gf2_rref(M)[1])


def gf2_nullspace(M):
    """Canonical basis of {y : M y^T = 0} as rows (one per free column, ascending)."""
    M = np.asarray(M, dtype=np.uint8)
    n = M.shape[1]
    if M.shape[0] == 0:
        return np.eye(n, dtype=np.uint8)
    R, piv = gf2_rref(M)
    pset = set(piv)
    free = [c for c in range(n) if c not in pset]
    out = np.zeros((len(free), n), dtype=np.uint8)
    for i, f in enumerate(free):
        out[i, f] = 1
        for ri, pc in enumerate(piv):
            if R[ri, f]:
                out[i, pc] = 1
    return out


def gf2_matmul(A, B):
    return (np.asarray(A, dtype=np.int64) @ np.asarray(B, dtype=np.int64) % 2).astype(np.uint8)


# --------------------------------------------------------------------------- code builders
def classical_parity_from_rng(rng, n: int, k: int):
    """H = [R^T | I_{n-k}] for the systematic generator G = [I_k | R], R k x (n-k)."""
    R = rng.integers(0, 2, (k, n - k), dtype=np.uint8)
    return np.concatenate([R.T, np.eye(n - k, dtype=np.uint8)], axis=1).astype(np.uint8)


def css_from_rng(rng, n: int, rx: int, rz: int):
    """Random CSS pair: Hx rx x n resampled to full rank, Hz = C . ker(Hx) with rank rz."""
    while True:
        Hx = rng.integers(0, 2, (rx, n), dtype=np.uint8)
        if gf2_rank(Hx) == rx:
            break
    N = gf2_nullspace(Hx)
    while True:
        C = rng.integers(0, 2, (rz, N.shape[0]), dtype=np.uint8)
        Hz = gf2_matmul(C, N)
        if gf2_rank(Hz) == rz:
            break
    return Hx, Hz


def single_classical_96():
    rng = np.random.default_rng(0)
    return classical_parity_from_rng(rng, 96, 32)


def single_css_128():
    rng = np.random.default_rng(1)
    return css_from_rng(rng, 128, 40, 40)


def single_classical_128():
    rng = np.random.default_rng(2)
    return classical_parity_from_rng(rng, 128, 40)


@dataclass
class CodeSpec:
    """One code of a batch: ``kind`` is 'classical' (H) or 'css' (Hx, Hz, which='min')."""
    kind: str
    mats: tuple
    n: int
    meta: dict = field(default_factory=dict)


def batch_1024(num: int = 1024, seed: int = 3):
    """The 1024-code uneven batch: first half classical, second half CSS."""
    rng = np.random.default_rng(seed)
    half = num // 2
    out = []
    for _ in range(half):
        n = int(rng.integers(48, 129))
        k = int(rng.integers(n // 4, n // 2 + 1))
        H = classical_parity_from_rng(rng, n, k)
        out.append(CodeSpec("classical", (H,), n, {"k": k}))
    for _ in range(num - half):
        n = int(rng.integers(40, 129))
        rx = int(rng.integers(n // 5, n // 3 + 1))
        rz = int(rng.integers(n // 5, n // 3 + 1))
        Hx, Hz = css_from_rng(rng, n, rx, rz)
        out.append(CodeSpec("css", (Hx, Hz), n, {"rx": rx, "rz": rz}))
    return out


@dataclass
class Request:
    """One serving request: arrival time (s), kind and matrices."""
    t: float
    kind: str          # 'classical' | 'css' | 'opweight'
    mats: tuple
    n: int


def serving_stream(rate: float, num: int = 20000, seed: int = 4, pool: int = 256):
    """Poisson arrivals at ``rate`` req/s.  Mix 40% classical / 40% CSS / 20% operator weight.

    Classical: n log-uniform in [32,128], k = round(U(0.25,0.5) n).  CSS: n log-uniform in
    [40,128], ranks uniform in [n/5, n/3].  Operator weight: a CSS code from a pool of
    ``pool`` pre-drawn codes with Bernoulli(1/2) z and x vectors.
    """
    rng = np.random.default_rng(seed)
    css_pool = []
    for _ in range(pool):
        n = int(round(math.exp(rng.uniform(math.log(40), math.log(128)))))
        rx = int(rng.integers(n // 5, n // 3 + 1))
        rz = int(rng.integers(n // 5, n // 3 + 1))
        css_pool.append(css_from_rng(rng, n, rx, rz))
    t = 0.0
    reqs = []
    for _ in range(num):
        t += float(rng.exponential(1.0 / rate))
        u = float(rng.uniform())
        if u < 0.4:
            n = int(round(math.exp(rng.uniform(math.log(32), math.log(128)))))
            k = max(1, int(round(rng.uniform(0.25, 0.5) * n)))
            reqs.append(Request(t, "classical", (classical_parity_from_rng(rng, n, k),), n))
        elif u < 0.8:
            n = int(round(math.exp(rng.uniform(math.log(40), math.log(128)))))
            rx = int(rng.integers(n // 5, n // 3 + 1))
            rz = int(rng.integers(n // 5, n // 3 + 1))
            Hx, Hz = css_from_rng(rng, n, rx, rz)
            reqs.append(Request(t, "css", (Hx, Hz), n))
        else:
            Hx, Hz = css_pool[int(rng.integers(0, pool))]
            n = Hx.shape[1]
            z = rng.integers(0, 2, n, dtype=np.uint8)
            x = rng.integers(0, 2, n, dtype=np.uint8)
            reqs.append(Request(t, "opweight", (Hx, Hz, z, x), n))
    return reqs


def collect_generator(n: int = 128, k: int = 64, seed: int = 13):
    """Input of the low-weight collector benchmark: a random k x n generator in systematic
    form on a random column set, as the reference's codeaut layer hands its information-set
    generators to codeaut_bz_collect (python/qubitserf/codeaut/lowweight.py:117-126)."""
    rng = np.random.default_rng(seed)
    A = rng.integers(0, 2, size=(k, n - k), dtype=np.uint8)
    G = np.concatenate([np.eye(k, dtype=np.uint8), A], axis=1)
    return np.ascontiguousarray(G[:, rng.permutation(n)])


def toric_code(L: int):
    """(Hx, Hz) of the [[2 L^2, 2, L]] toric code: the hypergraph product of the L x L check
    matrix of the cyclic repetition code with itself (edges of an L x L torus; X checks on
    vertices, Z checks on faces)."""
    H = np.zeros((L, L), dtype=np.uint8)
    for i in range(L):
        H[i, i] = H[i, (i + 1) % L] = 1
    I = np.eye(L, dtype=np.uint8)
    Hx = np.concatenate([np.kron(H, I), np.kron(I, H.T)], axis=1) % 2
    Hz = np.concatenate([np.kron(I, H), np.kron(H.T, I)], axis=1) % 2
    return Hx.astype(np.uint8), Hz.astype(np.uint8)

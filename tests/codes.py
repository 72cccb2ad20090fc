"""Standard code families used as test inputs (constructed here from their definitions):
repetition / Hamming parity checks, Steane, Shor, hypergraph products (toric, planar
surface), Reed-Muller, Bacon-Shor gauge groups, and small non-CSS stabilizer codes.
All return uint8 0/1 matrices."""
from __future__ import annotations

from itertools import combinations

import numpy as np


def repetition_parity(n):
    H = np.zeros((n - 1, n), np.uint8)
    for i in range(n - 1):
        H[i, i] = H[i, i + 1] = 1
    return H


def cyclic_repetition_parity(n):
    H = np.zeros((n, n), np.uint8)
    for i in range(n):
        H[i, i] = H[i, (i + 1) % n] = 1
    return H


def hamming_parity(r):
    n = (1 << r) - 1
    return np.array([[(j >> b) & 1 for j in range(1, n + 1)] for b in range(r)], np.uint8)


def steane():
    H = hamming_parity(3)
    return H.copy(), H.copy()


def shor():
    # X checks compare adjacent blocks of three; Z checks compare neighbours in a block.
    Hx = np.zeros((2, 9), np.uint8)
    Hx[0, 0:6] = 1
    Hx[1, 3:9] = 1
    Hz = np.zeros((6, 9), np.uint8)
    for b in range(3):
        for i in range(2):
            Hz[2 * b + i, 3 * b + i] = Hz[2 * b + i, 3 * b + i + 1] = 1
    return Hx, Hz


def hypergraph_product(H1, H2):
    m1, n1 = H1.shape
    m2, n2 = H2.shape
    Hx = np.concatenate([np.kron(H1, np.eye(n2, dtype=np.uint8)),
                         np.kron(np.eye(m1, dtype=np.uint8), H2.T)], axis=1) % 2
    Hz = np.concatenate([np.kron(np.eye(n1, dtype=np.uint8), H2),
                         np.kron(H1.T, np.eye(m2, dtype=np.uint8))], axis=1) % 2
    return Hx.astype(np.uint8), Hz.astype(np.uint8)


def toric(L):
    H = cyclic_repetition_parity(L)
    return hypergraph_product(H, H)


def surface(L):
    H = repetition_parity(L)
    return hypergraph_product(H, H)


def reed_muller_generator(r, m):
    n = 1 << m
    pts = np.array([[(i >> b) & 1 for b in range(m)] for i in range(n)], np.uint8)
    rows = []
    for deg in range(r + 1):
        for S in combinations(range(m), deg):
            row = np.ones(n, np.uint8)
            for b in S:
                row = row * pts[:, b]
            rows.append(row)
    return np.array(rows, np.uint8)


def quantum_reed_muller(r, m):
    G = reed_muller_generator(r, m)
    return G.copy(), G.copy()


def bacon_shor(d):
    """Gauge generators on a d x d grid: XX on horizontal pairs, ZZ on vertical pairs."""
    n = d * d
    gx, gz = [], []
    for r in range(d):
        for c in range(d - 1):
            v = np.zeros(n, np.uint8)
            v[r * d + c] = v[r * d + c + 1] = 1
            gx.append(v)
    for c in range(d):
        for r in range(d - 1):
            v = np.zeros(n, np.uint8)
            v[r * d + c] = v[(r + 1) * d + c] = 1
            gz.append(v)
    return np.array(gx), np.array(gz)


def pauli_rows(strings):
    """Symplectic [z|x] matrix from Pauli strings."""
    n = len(strings[0])
    S = np.zeros((len(strings), 2 * n), np.uint8)
    for i, s in enumerate(strings):
        for j, ch in enumerate(s):
            if ch in "ZY":
                S[i, j] = 1
            if ch in "XY":
                S[i, n + j] = 1
    return S


def five_qubit():
    """[[5,1,3]]: cyclic shifts of XZZXI."""
    return pauli_rows(["XZZXI", "IXZZX", "XIXZZ", "ZXIXZ"])


def random_isotropic(rng, n, m, tries=200):
    """Random commuting (isotropic) symplectic generators, not necessarily CSS."""
    rows = []
    for _ in range(tries):
        if len(rows) == m:
            break
        v = rng.integers(0, 2, 2 * n, dtype=np.uint8)
        ok = True
        for r in rows:
            if (int(np.dot(r[:n], v[n:])) + int(np.dot(r[n:], v[:n]))) % 2:
                ok = False
                break
        if ok and v.any():
            rows.append(v)
    return np.array(rows, np.uint8) if rows else np.zeros((0, 2 * n), np.uint8)


def random_css(rng, n, m):
    """Hx m x n random; Hz from the orthogonal complement (Hx Hz^T = 0)."""
    from qubitserf_b200.workloads import gf2_nullspace, gf2_matmul
    Hx = rng.integers(0, 2, (m, n), dtype=np.uint8)
    N = gf2_nullspace(Hx)
    if N.shape[0] == 0:
        return Hx, np.zeros((0, n), np.uint8)
    C = rng.integers(0, 2, (max(1, N.shape[0] // 2), N.shape[0]), dtype=np.uint8)
    return Hx, gf2_matmul(C, N)

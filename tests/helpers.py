"""Matrices of the reference's own Cholesky tests (crates/solver/src/cholesky.rs:1573-2207),
rebuilt here so the oracle and the GPU path are checked on the cases the reference pins."""
from __future__ import annotations

import numpy as np

from fieldcraft_b200 import problems
from fieldcraft_b200.cholesky import Csr

MASK = (1 << 64) - 1


class Lcg:
    """The tests' generator: state = state * 6364136223846793005 + 1442695040888963407 (mod 2^64)."""

    def __init__(self, seed: int):
        self.state = seed

    def step(self) -> int:
        self.state = (self.state * 6364136223846793005 + 1442695040888963407) & MASK
        return self.state

    def unit(self) -> float:
        """(state >> 11) / 2^53 - 0.5 (cholesky.rs:1631-1635)."""
        return (self.step() >> 11) / float(1 << 53) - 0.5

    def high(self) -> int:
        """state >> 33 (cholesky.rs:2025-2028, :2156-2159)."""
        return self.step() >> 33


def trapezoid(m: int, w: int) -> int:
    return sum(max(m - c, 0) for c in range(w))


def offset(m: int, c: int) -> int:
    return c * m - c * max(c - 1, 0) // 2


def rows_to_csr(rows) -> Csr:
    """Rows of (column, value) pairs, each sorted by column, to Csr."""
    ptr, idx, val = [0], [], []
    for row in rows:
        row = sorted(row, key=lambda e: e[0])
        idx.extend(c for c, _ in row)
        val.extend(v for _, v in row)
        ptr.append(len(idx))
    return Csr(len(rows), np.array(ptr, np.int64), np.array(idx, np.int32), np.array(val, np.float64))


def grid_7x5(shift: bool = True) -> np.ndarray:
    """The 2D Laplacian-like 7 x 5 grid with diagonal 4.5 (cholesky.rs:1689-1706); the pure
    Laplacian when `shift` is false (:1713-1718)."""
    w, h = 7, 5
    n = w * h
    a = np.zeros((n, n))
    for i in range(w):
        for j in range(h):
            k = i * h + j
            a[k, k] = 4.5
            if i + 1 < w:
                a[k, k + h] = a[k + h, k] = -1.0
            if j + 1 < h:
                a[k, k + 1] = a[k + 1, k] = -1.0
    if not shift:
        for k in range(n):
            a[k, k] = -sum(a[k, j] for j in range(n) if j != k)
    return a


def panels_matrix() -> Csr:
    """Two 8 x 8 x 6 grids of 3 coupled unknowns per point, a dense 400-wide separator and a
    separate 5 x 5 block (cholesky.rs:1746-1810)."""
    nx, ny, nz = 8, 8, 6
    point = lambda i, j, k: i + nx * (j + ny * k)
    per = 3 * nx * ny * nz
    sep = 400
    n = 2 * per + sep + 5
    rows = [[] for _ in range(n)]

    def pair(a, b, v):
        rows[a].append((b, v))
        rows[b].append((a, v))

    for base in (0, per):
        for k in range(nz):
            for j in range(ny):
                for i in range(nx):
                    p = base + 3 * point(i, j, k)
                    for a in range(3):
                        rows[p + a].append((p + a, 7.0))
                        for b in range(a + 1, 3):
                            pair(p + a, p + b, 0.25)
                    nxt = []
                    if i + 1 < nx:
                        nxt.append(point(i + 1, j, k))
                    if j + 1 < ny:
                        nxt.append(point(i, j + 1, k))
                    if k + 1 < nz:
                        nxt.append(point(i, j, k + 1))
                    for q in nxt:
                        for a in range(3):
                            pair(p + a, base + 3 * q + a, -1.0)
    s0 = 2 * per
    for a in range(sep):
        rows[s0 + a].append((s0 + a, 20.0))
        for b in range(a + 1, sep):
            pair(s0 + a, s0 + b, 0.5 / (1.0 + (b - a)) ** 2)
        pair(s0 + a, (7 * a) % per, -0.1)
        pair(s0 + a, per + (11 * a) % per, -0.1)
    d0 = s0 + sep
    for a in range(5):
        rows[d0 + a].append((d0 + a, 10.0))
        for b in range(a + 1, 5):
            pair(d0 + a, d0 + b, 1.0 / (1.0 + (a + b)))
    return rows_to_csr(rows)


def blocks40() -> np.ndarray:
    """40 nodes of three unknowns, each coupled with three random others (LCG seed 7,
    cholesky.rs:2021-2043)."""
    nodes, B = 40, 3
    g = Lcg(7)
    dense = np.zeros((B * nodes, B * nodes))

    def couple(a, b):
        for i in range(B):
            for j in range(B):
                v = 100.0 if (a == b and i == j) else 0.5
                dense[B * a + i, B * b + j] = v
                dense[B * b + j, B * a + i] = v

    for a in range(nodes):
        couple(a, a)
        for _ in range(3):
            b = g.high() % nodes
            couple(max(a, b), min(a, b))
    return dense


def solid_stiffness(n: int = 5, roller: bool = False) -> Csr:
    """A block of n^3 unit hex8 elements held at its base, E = 1000, nu = 0.3, in the
    fill-reducing order (cholesky.rs:2067-2124); with `roller`, the corner node (n, n, n) is
    held in x too, which removes its first equation."""
    i, j, k = problems.node_grid(n, n, n)
    p = problems.box(n, n, n, float(n), float(n), float(n), 1000.0, 0.3, k == 0)
    csr = p.csr
    if not roller:
        return csr
    corner = n + (n + 1) * (n + (n + 1) * n)
    e = int(p.eq[3 * corner])
    dense_rows = []
    for r in range(csr.n):
        if r == e:
            continue
        lo, hi = csr.ptr[r], csr.ptr[r + 1]
        row = []
        for c, v in zip(csr.idx[lo:hi], csr.val[lo:hi]):
            if c == e:
                continue
            row.append((int(c) - (c > e), float(v)))
        dense_rows.append(row)
    return rows_to_csr(dense_rows)


def band_matrix():
    """A band with a few entries far off it, by full rows (LCG seed 99, cholesky.rs:2151-2172)."""
    n = 3 * 1024 + 17
    g = Lcg(99)
    rows = [[] for _ in range(n)]
    for i in range(n):
        rows[i].append((i, 10.0 + i))
        cand = [max(i - 1, 0), max(i - 7, 0), g.high() % (i + 1)]
        for j in cand:
            if j < i and not any(c == j for c, _ in rows[i]):
                v = 1.0 + (g.high() % 100) / 100.0
                rows[i].append((j, v))
                rows[j].append((i, v))
    return rows, rows_to_csr(rows)


def sin_solution(n: int) -> np.ndarray:
    """x_i = sin(0.37 i) (cholesky.rs:1676)."""
    return np.sin(np.arange(n, dtype=np.float64) * 0.37)


def shifted_grid(n, sigma: float):
    """A 3D grid Laplacian, 3 uncoupled unknowns per point, shifted by sigma, and the count of its
    eigenvalues below sigma (crates/solver/src/ldlt.rs:594-635): rows built point by point, each
    point's diagonal then its couplings to the next point along x, y and z."""
    nx, ny, nz = n
    point = lambda i, j, k: i + nx * (j + ny * k)  # noqa: E731
    rows = [[] for _ in range(3 * nx * ny * nz)]
    for k in range(nz):
        for j in range(ny):
            for i in range(nx):
                p = 3 * point(i, j, k)
                for a in range(3):
                    rows[p + a].append((p + a, 6.0 - sigma))
                nxt = [point(i + 1, j, k) if i + 1 < nx else None, point(i, j + 1, k) if j + 1 < ny else None,
                       point(i, j, k + 1) if k + 1 < nz else None]
                for q in nxt:
                    if q is None:
                        continue
                    for a in range(3):
                        rows[p + a].append((3 * q + a, -1.0))
                        rows[3 * q + a].append((p + a, -1.0))
    axis = lambda m: [2.0 - 2.0 * np.cos(np.pi * t / (m + 1.0)) for t in range(1, m + 1)]  # noqa: E731
    below = 3 * sum(1 for a in axis(nx) for b in axis(ny) for c in axis(nz) if a + b + c < sigma)
    return rows_to_csr(rows), below


def saddle(nk: int, nb: int) -> Csr:
    """[[K, B], [B^T, 0]] in one dense supernode, the zero-diagonal columns first
    (crates/solver/src/ldlt.rs:656-688)."""
    n = nk + nb
    rows = [[] for _ in range(n)]
    for i in range(nk):
        for j in range(nk):
            rows[i].append((j, 0.5 if i == j else 0.05 / (1.0 + (i + j))))
    for c in range(nb):
        for i in range(nk):
            v = float((i * 7 + c * 3) % 5) - 2.0 + (3.0 if i == c else 0.0)
            rows[i].append((nk + c, v))
            rows[nk + c].append((i, v))
        for d in range(nb):
            rows[nk + c].append((nk + d, 0.0))
    order = list(range(nk, n)) + list(range(nk))
    inverse = [order.index(i) for i in range(n)]
    permuted = [None] * n
    for i, row in enumerate(rows):
        permuted[inverse[i]] = [(inverse[c], v) for c, v in row]
    return rows_to_csr(permuted)


def exact_solution(n: int) -> np.ndarray:
    """x_i = ((37 i mod 101) - 50) / 50: exact in binary on every platform
    (crates/solver/src/ldlt.rs:791-792)."""
    i = np.arange(n, dtype=np.int64)
    return ((i * 37 % 101).astype(np.float64) - 50.0) / 50.0


def fingerprint(values) -> int:
    """FNV-1a over the bit patterns of FP64 values (crates/solver/src/ldlt.rs:755-758)."""
    h = 0xCBF29CE484222325
    for b in np.ascontiguousarray(values, np.float64).view(np.uint64).tolist():
        h = ((h ^ b) * 0x100000001B3) & MASK
    return h


def hex_pattern(n: int, sigma: float, nested_dissection) -> Csr:
    """The stiffness pattern of a hex8 mesh on an n^3 grid of nodes (27 neighbours, 3 unknowns a
    node), ordered by `nested_dissection(xyz, adjacency)`, diagonally dominant and shifted by
    sigma (crates/solver/src/ldlt.rs:979-1020)."""
    node = lambda i, j, k: i + n * (j + n * k)  # noqa: E731
    nodes = n ** 3
    xyz = np.array([[v % n, (v // n) % n, v // (n * n)] for v in range(nodes)], np.float64)
    adjacency = [[] for _ in range(nodes)]
    for k in range(n):
        for j in range(n):
            for i in range(n):
                for t in range(27):
                    x, y, z = i + t % 3, j + (t // 3) % 3, k + t // 9
                    if 1 <= x <= n and 1 <= y <= n and 1 <= z <= n:
                        adjacency[node(i, j, k)].append(node(x - 1, y - 1, z - 1))
    order = nested_dissection(xyz, adjacency)
    place = np.zeros(nodes, np.int64)
    place[np.asarray(order)] = np.arange(nodes)
    rows = [[] for _ in range(3 * nodes)]
    for v, adj in enumerate(adjacency):
        for w in adj:
            for a in range(3):
                for b in range(3):
                    if v == w:
                        value = 30.0 - sigma if a == b else 0.5
                    elif a == b:
                        value = -1.0
                    else:
                        value = 0.01 * ((v + w) % 3)
                    rows[3 * place[v] + a].append((3 * place[w] + b, value))
    return rows_to_csr(rows)

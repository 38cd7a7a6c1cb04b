"""Shift-invert block Lanczos for the lowest modes of K phi = lambda M phi (crates/solver/src/eigen.rs:
155-466), the caller that solves many right-hand sides with one factor: every block of Lanczos
vectors is one `solve_many` of (K - sigma M) on the GPU.

The spectral transformation: with sigma below the wanted eigenvalues, (K - sigma M)^-1 M is
symmetric in the M inner product with eigenvalues theta = 1 / (lambda - sigma), so the lowest
lambda become the largest, well separated theta. A block of vectors finds eigenvalues repeated up to
the block size; every new block is orthogonalised against all earlier ones twice (classical
Gram-Schmidt in the M inner product); a Ritz pair has converged when its residual bound
||B_{j+1} s|| is below tolerance * theta. The start block comes from the reference's seeded
xorshift64* generator, so results are reproducible.

The projected matrix's dense eigenproblem (at most a few hundred rows) is numpy's; the solves are
the operator's (`ShiftInvert`: the GPU factor's `solve_many`).
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

MASK = (1 << 64) - 1


class Random:
    """xorshift64* (eigen.rs:155-173): uniform in [-1, 1)."""

    def __init__(self, seed: int):
        self.state = max(seed & MASK, 1)

    def uniform(self) -> float:
        s = self.state
        s ^= s >> 12
        s ^= (s << 25) & MASK
        s ^= s >> 27
        self.state = s
        v = (s * 0x2545F4914F6CDD1D) & MASK
        return (v >> 11) / float(1 << 52) - 1.0

    def vector(self, n: int) -> np.ndarray:
        return np.array([self.uniform() for _ in range(n)])


@dataclass
class Wanted:
    """Modes to return with lambda in [min, max] (eigen.rs:175-184)."""
    count: int
    min: float = -np.inf
    max: float = np.inf


@dataclass
class Eigenpairs:
    values: list = field(default_factory=list)     # lambda ascending
    vectors: list = field(default_factory=list)    # M-orthonormal, the largest component positive
    negative: list = field(default_factory=list)   # converged eigenvalues of negative Ritz values
    basis: int = 0                                 # Lanczos vectors used


class NotConverged(RuntimeError):
    pass


class Operator:
    """What the iteration needs (eigen.rs:186-215): n, y = M x, x <- (K - sigma M)^-1 x for a block."""

    n: int

    def mass(self, x: np.ndarray) -> np.ndarray:
        raise NotImplementedError

    def solve_many(self, xs: np.ndarray) -> np.ndarray:
        """xs [n, k] -> (K - sigma M)^-1 xs."""
        raise NotImplementedError

    def operand(self, x: np.ndarray, mx: np.ndarray) -> np.ndarray:
        return mx.copy()

    def eigenvalue(self, shift: float, theta: float) -> float:
        return shift + 1.0 / theta


def orthonormalize(op: Operator, w, q, mq, rng: Random):
    """A block orthonormalised against the basis and itself in the M inner product (classical
    Gram-Schmidt, twice); a vanishing column is replaced by a fresh random direction whose
    coefficient stays zero (eigen.rs:225-279). Returns (vectors, M products, r[j][i])."""
    n, k = op.n, len(w)
    r = np.zeros((k, k))
    out, mout = [], []
    for i, v in enumerate(w):
        v = np.array(v, dtype=np.float64)
        fresh = False
        for _attempt in range(4):
            before = np.sqrt(max(float(v @ op.mass(v)), 0.0))
            for _ in range(2):
                for qj, mqj in zip(q, mq):
                    v -= float(mqj @ v) * qj
                for j, (qj, mqj) in enumerate(zip(out, mout)):
                    c = float(mqj @ v)
                    v -= c * qj
                    if not fresh:
                        r[j, i] += c
            mv = op.mass(v)
            norm = np.sqrt(max(float(v @ mv), 0.0))
            if norm > 1e-8 * before and norm > 0.0:
                if not fresh:
                    r[i, i] = norm
                out.append(v / norm)
                mout.append(mv / norm)
                break
            fresh = True
            v = rng.vector(n)
    return out, mout, r


def lanczos(op: Operator, shift: float, wanted: Wanted, block: int, max_basis: int, tolerance: float) -> Eigenpairs:
    """Shift-invert block Lanczos with full reorthogonalisation (eigen.rs:281-466)."""
    n = op.n
    if n == 0:
        raise ValueError("there are no free degrees of freedom")
    b = min(max(block, 1), n)
    max_basis = max(min(max_basis, n), b)
    rng = Random(0x9E3779B97F4A7C15)
    q, mq = [], []
    t = np.zeros((0, 0))
    start = [rng.vector(n) for _ in range(b)]
    cur, mcur, _ = orthonormalize(op, start, q, mq, rng)
    if len(cur) < b:
        raise NotConverged("could not build a Lanczos start block")
    prev_b = None
    next_check = max(wanted.count + b, 2 * b)
    while True:
        j0 = len(q)
        # W = Op Q_j: the block's solves at once
        ys = np.stack([op.operand(c, mc) for c, mc in zip(cur, mcur)], axis=1)
        wblock = op.solve_many(ys)
        w = [wblock[:, j].copy() for j in range(wblock.shape[1])]
        a = np.array([[float(mqi @ wj) for wj in w] for mqi in mcur])
        for i in range(b):
            for j in range(i + 1, b):
                s = 0.5 * (a[i, j] + a[j, i])
                a[i, j] = a[j, i] = s
        q.extend(cur)
        mq.extend(mcur)
        m = len(q)
        grown = np.zeros((m, m))
        grown[:t.shape[0], :t.shape[1]] = t
        t = grown
        t[j0:j0 + b, j0:j0 + b] = a
        if prev_b is not None:
            t[j0:j0 + b, j0 - b:j0] = prev_b
            t[j0 - b:j0, j0:j0 + b] = prev_b.T
        full = m >= max_basis or m + b > n
        if full:
            nxt, mnxt, bnext = [], [], np.zeros((b, b))
        else:
            nxt, mnxt, bnext = orthonormalize(op, w, q, mq, rng)
        if m >= next_check or full or len(nxt) < b:
            next_check = m + max(m // 4, b)
            theta, s = np.linalg.eigh(t)
            idx = sorted(range(m), key=lambda x: (-theta[x], x))
            done, accepted, found = False, [], 0
            for i in idx:
                th = theta[i]
                if not th > 0.0:
                    break
                res2 = 0.0 if full else float(np.sum((bnext @ s[m - b:m, i]) ** 2))
                if np.sqrt(res2) > tolerance * th:
                    break
                lam = op.eigenvalue(shift, th)
                if lam > wanted.max:
                    done = True
                    break
                if lam >= wanted.min:
                    accepted.append(i)
                    found += 1
                    if found == wanted.count:
                        done = True
                        break
            if full and not done:
                if m >= n:
                    done = True
                else:
                    raise NotConverged(f"found {found} of {wanted.count} modes after {m} Lanczos vectors (the cap)")
            if done:
                negative = []
                for i in reversed(idx):
                    th = theta[i]
                    if not th < 0.0:
                        break
                    res2 = 0.0 if full else float(np.sum((bnext @ s[m - b:m, i]) ** 2))
                    if np.sqrt(res2) > tolerance * abs(th):
                        break
                    negative.append(op.eigenvalue(shift, th))
                qm = np.stack(q, axis=1)
                values, vectors = [], []
                for i in accepted:
                    values.append(op.eigenvalue(shift, theta[i]))
                    x = qm @ s[:, i]
                    norm = np.sqrt(max(float(x @ op.mass(x)), 0.0))
                    if norm > 0.0:
                        x = x / norm
                    big = x[np.argmax(np.abs(x))]
                    vectors.append(-x if big < 0.0 else x)
                return Eigenpairs(values, vectors, negative, m)
        if full:
            raise NotConverged("the Lanczos basis is exhausted")
        cur, mcur = nxt, mnxt
        if len(cur) < b:
            raise NotConverged("the Lanczos block lost rank")
        prev_b = bnext


class ShiftInvert(Operator):
    """(K - sigma M)^-1 on the GPU: K and M by rows (both triangles, M's pattern within K's or
    diagonal as a vector), factored once by the path's Cholesky (sigma below the spectrum) or LDL^T
    (`indefinite`); each Lanczos block is one solve_many of the factor."""

    def __init__(self, k, m, sigma: float, max_entries: int = 2**62, indefinite: bool = False, device: int = 0):
        from .cholesky import Csr, Factor, LdltFactor, UpperColumns
        self.n = k.n
        self.k, self.m = k, m
        rows = np.repeat(np.arange(k.n), np.diff(k.ptr))
        shifted = k.val.copy()
        if isinstance(m, np.ndarray):
            shifted[k.idx == rows] -= sigma * m[rows[k.idx == rows]]
            self._mass = lambda x: m * x  # noqa: E731
        else:
            mk = {}
            mrows = np.repeat(np.arange(m.n), np.diff(m.ptr))
            for r, c, v in zip(mrows, m.idx, m.val):
                mk[(int(r), int(c))] = v
            for e, (r, c) in enumerate(zip(rows, k.idx)):
                shifted[e] -= sigma * mk.get((int(r), int(c)), 0.0)
            mrow = mrows

            def mass(x):
                y = np.zeros(m.n)
                np.add.at(y, mrow, m.val * x[m.idx])
                return y
            self._mass = mass
        up = UpperColumns.from_symmetric(Csr(k.n, k.ptr, k.idx, shifted))
        self.factor = (LdltFactor if indefinite else Factor).new(up, max_entries, device=device)

    def mass(self, x):
        return self._mass(x)

    def solve_many(self, xs):
        out = np.asfortranarray(xs, dtype=np.float64).copy(order="F")
        self.factor.solve_many(out)
        return out

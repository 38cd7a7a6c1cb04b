"""The LDL^T solve's structure (fieldcraft_b200/csrc/host/ldlt_fold.cpp): the factor's pivot
orders folded into the supernodal structure so that the Cholesky solve runs on it unchanged.
Checked against a restatement of each output, and by solving on the folded structure (the
oracle's factor with its rows below moved as the fold says, D out of a unit lower L, D^-1 between
the passes): the solution is the oracle's LDL^T solve's (ldlt.rs:404-413) to rounding. (Not bit
for bit: the backward pass sums a supernode's rows below in their new order.)"""
import ctypes as C

import numpy as np
import pytest

import helpers as H
from fieldcraft_b200 import _lib
from oracle import oracle


def fold(s, order):
    n, ns = s.info("n"), s.info("ns")
    first, rptr = s.array("first"), s.array("rptr")
    rows = s.array("rows").astype(np.int32)
    perm, sparent = s.array("perm"), s.array("sparent")
    below = int(sum((rptr[k + 1] - rptr[k]) - (first[k + 1] - first[k]) for k in range(ns)))
    roots_below = int(sum((rptr[k + 1] - rptr[k]) - (first[k + 1] - first[k]) for k in range(ns) if sparent[k] < 0))
    out_perm = np.zeros(n, np.int64)
    out_rows = np.zeros(rows.size, np.int32)
    out_from = np.zeros(max(below, 1), np.int32)
    out_rel = np.zeros(max(below - roots_below, 1), np.int32)
    order32 = np.ascontiguousarray(order, np.int32)  # kept alive across the call
    lib = _lib.load()
    lib.fc_test_ldlt_fold.restype = C.c_int
    p = lambda a: C.c_void_p(a.ctypes.data)  # noqa: E731
    rc = lib.fc_test_ldlt_fold(C.c_int64(n), C.c_int64(ns), p(first), p(rptr), p(rows), p(perm), p(sparent),
                               p(order32), p(out_perm), p(out_rows), p(out_from), p(out_rel))
    assert rc == 0
    return out_perm, out_rows, out_from[:below], out_rel[:below - roots_below]


def cases():
    mixed_rows = [[] for _ in range(7)]
    for i, row in enumerate([[0.0, 0.1, 3.0], [0.1, 5.0, 0.2], [3.0, 0.2, 0.5]]):
        mixed_rows[i].extend((j, v) for j, v in enumerate(row))
    for i in range(3, 6):
        mixed_rows[i].extend((j, 4.0 if i == j else 0.25) for j in range(3, 6))
    for i in range(6):
        mixed_rows[i].append((6, 0.15))
        mixed_rows[6].append((i, 0.15))
    mixed_rows[6].append((6, 8.0))
    order = [3, 0, 4, 1, 5, 2, 6]
    inverse = [order.index(i) for i in range(7)]
    mixed = H.rows_to_csr([[(inverse[j], v) for j, v in mixed_rows[i]] for i in order])
    return {"mixed": mixed, "grid": H.shifted_grid([7, 6, 5], 3.3)[0], "saddle": H.saddle(8, 3),
            "wide": H.shifted_grid([14, 12, 10], 2.7)[0]}


@pytest.mark.parametrize("name", list(cases()))
def test_fold_and_solve_on_the_folded_structure(name):
    a = cases()[name]
    ptr, idx, val = oracle.upper_from_symmetric(a.n, a.ptr, a.idx, a.val)
    s = oracle.Sym(a.n, ptr, idx)
    f = oracle.Ldlt(s, val)
    piv, order = f.pivots()
    n, ns = a.n, s.info("ns")
    first, rptr, rows, perm = s.array("first"), s.array("rptr"), s.array("rows"), s.array("perm")
    sparent = s.array("sparent")
    new_perm, new_rows, frm, rel = fold(s, order)
    # a restatement of each output
    pos = np.zeros(n, np.int64)
    for k in range(ns):
        f0, w = first[k], first[k + 1] - first[k]
        pos[f0 + order[f0:f0 + w]] = f0 + np.arange(w)
    assert np.array_equal(new_perm[pos], perm)
    at_from, at_rel = 0, 0
    for k in range(ns):
        f0, w, m = first[k], first[k + 1] - first[k], rptr[k + 1] - rptr[k]
        r = new_rows[rptr[k]:rptr[k + 1]]
        assert np.array_equal(r[:w], f0 + np.arange(w))
        old_below = pos[rows[rptr[k] + w:rptr[k + 1]]]
        assert np.all(np.diff(r[w:]) > 0) and np.array_equal(r[w:], old_below[frm[at_from:at_from + m - w]])
        at_from += m - w
        if sparent[k] >= 0:
            pr = list(new_rows[rptr[sparent[k]]:rptr[sparent[k] + 1]])
            assert list(rel[at_rel:at_rel + m - w]) == [pr.index(x) for x in r[w:]]
            at_rel += m - w
    # the solve on the folded structure
    values = f.values()
    L, D, E = [], np.zeros(n), np.zeros(n)
    at, at_from = 0, 0
    for k in range(ns):
        f0, w, m = first[k], first[k + 1] - first[k], rptr[k + 1] - rptr[k]
        F = np.zeros((m, w))
        for c in range(w):
            F[c:, c] = values[at:at + m - c]
            at += m - c
        for c in range(w):
            D[f0 + c] = F[c, c]
            F[c, c] = 1.0
            if piv[f0 + c] == 1:
                E[f0 + c] = F[c + 1, c]
                F[c + 1, c] = 0.0
        F[w:] = F[w:][frm[at_from:at_from + m - w]]
        at_from += m - w
        L.append(F)
    x_true = np.sin((np.arange(n) + 0.5) * 0.37)
    b = oracle.spmv(a.n, a.ptr, a.idx, a.val, x_true)
    want = f.solve(b.copy())
    y = b[new_perm].copy()
    for k in range(ns):  # forward, unit lower
        f0, w, m = first[k], first[k + 1] - first[k], rptr[k + 1] - rptr[k]
        r = new_rows[rptr[k]:rptr[k + 1]]
        for q in range(w):
            for i in range(q + 1, m):
                y[r[i]] -= L[k][i, q] * y[f0 + q]
    c = 0
    while c < n:  # D^-1
        if piv[c] == 1:
            d11, d21, d22 = D[c], E[c], D[c + 1]
            det = d11 * d22 - d21 * d21
            p, q = y[c], y[c + 1]
            y[c], y[c + 1] = (d22 * p - d21 * q) / det, (d11 * q - d21 * p) / det
            c += 2
        else:
            y[c] = y[c] / D[c]
            c += 1
    for k in reversed(range(ns)):  # backward
        f0, w, m = first[k], first[k + 1] - first[k], rptr[k + 1] - rptr[k]
        r = new_rows[rptr[k]:rptr[k + 1]]
        for q in reversed(range(w)):
            acc = y[f0 + q]
            for i in range(q + 1, m):
                acc -= L[k][i, q] * y[r[i]]
            y[f0 + q] = acc
    got = np.empty(n)
    got[new_perm] = y
    assert np.max(np.abs(got - want)) <= 1e-10 * np.max(np.abs(want))  # the path's accuracy bar
    assert np.max(np.abs(got - x_true)) < 1e-9


@pytest.mark.parametrize("seed", range(4))
def test_fold_on_random_sparse_indefinite_matrices(seed):
    """Random sparse symmetric matrices with small and negative diagonals (2 x 2 pivots, many
    supernodes, interchanges): the folded structure's solve is the oracle's to the path's bar."""
    rng = np.random.default_rng(seed)
    n = 150
    rows = [[] for _ in range(n)]
    for i in range(n):
        rows[i].append((i, float(rng.choice([0.05, -3.0, 4.0, 8.0]))))
    for _ in range(3 * n):
        i, j = rng.integers(0, n, 2)
        if i != j:
            v = float(rng.standard_normal())
            rows[i].append((int(j), v))
            rows[j].append((int(i), v))
    merged = []
    for r in rows:
        acc = {}
        for c, v in r:
            acc[c] = acc.get(c, 0.0) + v
        merged.append(sorted(acc.items()))
    a = H.rows_to_csr(merged)
    ptr, idx, val = oracle.upper_from_symmetric(a.n, a.ptr, a.idx, a.val)
    s = oracle.Sym(a.n, ptr, idx)
    try:
        f = oracle.Ldlt(s, val)
    except oracle.OracleError:
        pytest.skip("singular within a supernode")
    piv, order = f.pivots()
    new_perm, new_rows, frm, rel = fold(s, order)
    first, rptr = s.array("first"), s.array("rptr")
    values = f.values()
    ns = s.info("ns")
    L, D, E = [], np.zeros(n), np.zeros(n)
    at, at_from = 0, 0
    for k in range(ns):
        f0, w, m = first[k], first[k + 1] - first[k], rptr[k + 1] - rptr[k]
        F = np.zeros((m, w))
        for c in range(w):
            F[c:, c] = values[at:at + m - c]
            at += m - c
        for c in range(w):
            D[f0 + c] = F[c, c]
            F[c, c] = 1.0
            if piv[f0 + c] == 1:
                E[f0 + c] = F[c + 1, c]
                F[c + 1, c] = 0.0
        F[w:] = F[w:][frm[at_from:at_from + m - w]]
        at_from += m - w
        L.append(F)
    b = rng.standard_normal(n)
    want = f.solve(b.copy())
    y = b[new_perm].copy()
    for k in range(ns):
        f0, w, m = first[k], first[k + 1] - first[k], rptr[k + 1] - rptr[k]
        r = new_rows[rptr[k]:rptr[k + 1]]
        for q in range(w):
            y[r[q + 1:m]] -= L[k][q + 1:m, q] * y[f0 + q]
    c = 0
    while c < n:
        if piv[c] == 1:
            d11, d21, d22 = D[c], E[c], D[c + 1]
            det = d11 * d22 - d21 * d21
            p_, q_ = y[c], y[c + 1]
            y[c], y[c + 1] = (d22 * p_ - d21 * q_) / det, (d11 * q_ - d21 * p_) / det
            c += 2
        else:
            y[c] /= D[c]
            c += 1
    for k in reversed(range(ns)):
        f0, w, m = first[k], first[k + 1] - first[k], rptr[k + 1] - rptr[k]
        r = new_rows[rptr[k]:rptr[k + 1]]
        for q in reversed(range(w)):
            y[f0 + q] -= float(L[k][q + 1:m, q] @ y[r[q + 1:m]])
    got = np.empty(n)
    got[new_perm] = y
    assert np.max(np.abs(got - want)) <= 1e-10 * np.max(np.abs(want))

"""The device LDL^T panel (fieldcraft_b200/csrc/cuda/ldlt_panel.cuh) run on host threads by
tests/native/ldlt_emulation.cpp, against the oracle's LDL^T (crates/solver/src/ldlt.rs): the
same source the kernel compiles, so its pivots, interchanges, 1 x 1 and 2 x 2 stores, the
update coefficients W and its synchronisation are checked without a GPU. Fronts whose factor
depends only on A (dense single-supernode matrices, and leaf supernodes of sparse ones) must
come out bit for bit the oracle's on any number of threads."""
import numpy as np
import pytest

import helpers as H
from native import emulation as E
from oracle import oracle

SINGULAR = 2


def dense_csr(A):
    n = A.shape[0]
    return H.rows_to_csr([[(j, A[i, j]) for j in range(n) if A[i, j] != 0 or i == j] for i in range(n)])


def indefinite(n, seed, zero_every=3):
    rng = np.random.default_rng(seed)
    B = rng.standard_normal((n, n))
    A = B + B.T
    A[np.arange(1, n, zero_every), np.arange(1, n, zero_every)] = 0.0  # zero diagonals: 2 x 2 pivots
    return A


def oracle_ldlt(a):
    ptr, idx, val = oracle.upper_from_symmetric(a.n, a.ptr, a.idx, a.val)
    s = oracle.Sym(a.n, ptr, idx)
    return s, oracle.Ldlt(s, val)


def bits(x):
    return np.ascontiguousarray(x, np.float64).view(np.uint64)


@pytest.mark.parametrize("n", [1, 2, 11, 63, 64, 65, 129, 200])
@pytest.mark.parametrize("threads", [1, 5, 32])
def test_dense_fronts_are_the_oracles_bit_for_bit(n, threads):
    """One supernode (a dense matrix), panels of 64 with the update of the later columns between
    them: values, pivots, order and the count of 2 x 2 pivots as the oracle's."""
    A = indefinite(n, seed=n)
    s, f = oracle_ldlt(dense_csr(A))
    assert s.info("ns") == 1 and np.array_equal(s.array("perm"), np.arange(n))
    rc, F, piv, order, twos = E.factor_front(np.tril(A), n, np.max(np.abs(A), axis=0), threads)
    assert rc == -1
    opiv, oorder = f.pivots()
    assert np.array_equal(piv, opiv) and np.array_equal(order, oorder)
    assert twos == f.two_by_two()
    assert np.array_equal(bits(E.packed(F, n)), bits(f.values()))


@pytest.mark.parametrize("seed", range(6))
def test_no_thread_reads_what_another_moved(seed):
    """Random delays after every barrier (seeded) change which thread runs ahead; a thread that
    wrote what another had yet to read would change a bit or a branch."""
    A = indefinite(96, seed=100 + seed, zero_every=2)
    s, f = oracle_ldlt(dense_csr(A))
    rc, F, piv, order, _ = E.factor_front(np.tril(A), 96, np.max(np.abs(A), axis=0), threads=6, jitter=seed + 1)
    assert rc == -1
    assert np.array_equal(order, f.pivots()[1])
    assert np.array_equal(bits(E.packed(F, 96)), bits(f.values()))


def test_saddle_point_front():
    """ldlt.rs:656-698: zero diagonals first, so the search must pivot past them in 2 x 2 pairs."""
    a = H.saddle(8, 3)
    s, f = oracle_ldlt(a)
    A = np.zeros((a.n, a.n))
    for i in range(a.n):
        A[i, a.idx[a.ptr[i]:a.ptr[i + 1]]] = a.val[a.ptr[i]:a.ptr[i + 1]]
    perm = s.array("perm")
    Ap = A[np.ix_(perm, perm)]
    assert s.info("ns") == 1
    rc, F, piv, order, twos = E.factor_front(np.tril(Ap), a.n, np.max(np.abs(A), axis=0)[perm], threads=4)
    assert rc == -1 and twos == f.two_by_two() == 3
    assert np.array_equal(bits(E.packed(F, a.n)), bits(f.values()))


def leaf_fronts(a, s):
    """The leaf supernodes' fronts (no descendant updates): A's entries of their columns at
    their rows, in the analysis' order; with the largest |A| of each column."""
    perm = s.array("perm")
    first, rptr, rows, uptr = s.array("first"), s.array("rptr"), s.array("rows"), s.array("uptr")
    n = a.n
    A = np.zeros((n, n))
    for i in range(n):
        A[i, a.idx[a.ptr[i]:a.ptr[i + 1]]] = a.val[a.ptr[i]:a.ptr[i + 1]]
    Ap = A[np.ix_(perm, perm)]
    scale = np.max(np.abs(A), axis=0)[perm]
    trap = [sum(rptr[k + 1] - rptr[k] - c for c in range(first[k + 1] - first[k])) for k in range(len(first) - 1)]
    offs = np.concatenate([[0], np.cumsum(trap)])
    for k in range(len(first) - 1):
        if uptr[k + 1] != uptr[k]:
            continue
        f0, w = first[k], first[k + 1] - first[k]
        rk = rows[rptr[k]:rptr[k + 1]]
        front = np.zeros((len(rk), w))
        for c in range(w):
            front[c:, c] = Ap[rk[c:], f0 + c]
        yield k, front, w, scale[f0:f0 + w], slice(offs[k], offs[k + 1]), slice(f0, f0 + w)


@pytest.mark.parametrize("case", ["grid", "hex", "blocks"])
def test_leaf_fronts_with_rows_below(case):
    """Fronts taller than their columns (rows of later supernodes below the pivots): the
    interchanges move those rows' entries too, and L is stored for them."""
    if case == "grid":
        a = H.shifted_grid([7, 6, 5], 3.3)[0]
    elif case == "hex":
        from test_oracle_ldlt import nested_dissection
        a = H.hex_pattern(5, 22.0, nested_dissection)
    else:
        # two dense indefinite blocks of 100 and 40 columns sharing a 10-column separator
        n1, n2, ns = 100, 40, 10
        n = n1 + n2 + ns
        A = np.zeros((n, n))
        A[:n1, :n1] = indefinite(n1, seed=7)
        A[n1:n1 + n2, n1:n1 + n2] = indefinite(n2, seed=8)
        rng = np.random.default_rng(9)
        C = rng.standard_normal((n1 + n2, ns))
        A[:n1 + n2, n1 + n2:] = C
        A[n1 + n2:, :n1 + n2] = C.T
        A[n1 + n2:, n1 + n2:] = np.eye(ns) * 50.0
        a = dense_csr(A)
    s, f = oracle_ldlt(a)
    values = f.values()
    opiv, oorder = f.pivots()
    checked = 0
    for k, front, w, scale, vslice, cslice in leaf_fronts(a, s):
        rc, F, piv, order, _ = E.factor_front(front, w, scale, threads=4)
        assert rc == -1, k
        assert np.array_equal(piv, opiv[cslice]) and np.array_equal(order, oorder[cslice]), k
        assert np.array_equal(bits(E.packed(F, w)), bits(values[vslice])), k
        checked += 1
    assert checked > 0
    if case == "blocks":
        assert max(front.shape[0] - w for _, front, w, *_ in leaf_fronts(a, s)) > 0


def test_singular_columns_are_the_oracles():
    """A rank-one matrix and a NaN: the column the panel reports is the one the oracle names."""
    v = np.arange(1.0, 8.0)
    for A in [np.outer(v, v), indefinite(9, seed=4)]:
        if A.shape[0] == 9:
            A[4, 6] = A[6, 4] = np.nan
        with pytest.raises(oracle.OracleError) as e:
            oracle_ldlt(dense_csr(A))
        assert e.value.code == SINGULAR
        rc, *_ = E.factor_front(np.tril(A), A.shape[0], np.max(np.abs(A), axis=0), threads=3)
        assert rc == e.value.column


@pytest.mark.parametrize("m,w", [(64, 64), (65, 65), (130, 129), (300, 200), (1000, 257)])
def test_update_tiles_cover_the_later_columns_once(m, w):
    """The GEMM tiles a panel writes for the update of the later own columns: every entry of rows
    [c1, m) x columns [c1, w) on or below the diagonal exactly once, nothing else; a later end
    never needs more tiles than the earliest (the plan reserves that many)."""
    for c0 in range(0, w, 64):
        for c1 in (c0 + 64, c0 + 65):
            if c1 > w:
                continue
            hits = np.zeros((m, w), np.int32)
            for i0, j0, M, N, lower in E.update_tiles(m, w, c1):
                assert 0 < M <= 64 and 0 < N <= 64 and i0 >= j0 and lower == (i0 == j0)
                r = np.arange(i0, i0 + M)[:, None]
                c = np.arange(j0, j0 + N)[None, :]
                hits[i0:i0 + M, j0:j0 + N] += (r >= c) if lower else 1
            want = np.zeros((m, w), np.int32)
            for c in range(c1, w):
                want[c:, c] = 1
            assert np.array_equal(hits, want), (c0, c1)
            assert len(E.update_tiles(m, w, c1)) <= len(E.update_tiles(m, w, c0 + 64))


def test_w21_split_and_d_inverse():
    """After the panels: W21 = L21 D with times_d's operations (the Y of a descendant's product,
    cholesky.rs:531-548), D split from a unit lower L, and D^-1 applied as the solve's block step
    (cholesky.rs:946-974): each bit for bit the restatement below."""
    n1, n2, ns = 100, 40, 10
    n = n1 + n2 + ns
    A = np.zeros((n, n))
    A[:n1, :n1] = indefinite(n1, seed=7)
    A[n1:n1 + n2, n1:n1 + n2] = indefinite(n2, seed=8)
    Cc = np.random.default_rng(9).standard_normal((n1 + n2, ns))
    A[:n1 + n2, n1 + n2:] = Cc
    A[n1 + n2:, :n1 + n2] = Cc.T
    A[n1 + n2:, n1 + n2:] = np.eye(ns) * 50.0
    a = dense_csr(A)
    s, f = oracle_ldlt(a)
    k, front, w, scale, _, _ = max(leaf_fronts(a, s), key=lambda t: t[2])
    m = front.shape[0]
    assert m > w
    rc, F, piv, order, twos = E.factor_front(front, w, scale, threads=4)
    assert rc == -1 and twos > 0
    L = F.copy()
    w21, d, e = E.after_factor(F, w, piv, threads=5)
    # W21 by times_d on each row below
    want = np.zeros((m - w, w))
    for r in range(w, m):
        c = 0
        while c < w:
            if piv[c] == 1:
                x, y = L[r, c], L[r, c + 1]
                d11, d21, d22 = L[c, c], L[c + 1, c], L[c + 1, c + 1]
                want[r - w, c] = x * d11 + y * d21
                want[r - w, c + 1] = x * d21 + y * d22
                c += 2
            else:
                want[r - w, c] = L[r, c] * L[c, c]
                c += 1
    assert np.array_equal(bits(w21), bits(want))
    assert np.array_equal(d, np.diag(L)[:w])
    assert np.array_equal(e[piv == 1], L[np.flatnonzero(piv == 1) + 1, np.flatnonzero(piv == 1)])
    assert np.all(np.diag(F)[:w] == 1.0) and np.all(F[np.flatnonzero(piv == 1) + 1, np.flatnonzero(piv == 1)] == 0.0)
    # D^-1 on 3 right-hand sides
    y = np.random.default_rng(1).standard_normal((w, 3))
    got = E.apply_d_inverse(d, e, piv, y.copy())
    ref = y.copy()
    c = 0
    while c < w:
        if piv[c] == 1:
            d11, d21, d22 = d[c], e[c], d[c + 1]
            det = d11 * d22 - d21 * d21
            p, q = y[c].copy(), y[c + 1].copy()
            ref[c] = (d22 * p - d21 * q) / det
            ref[c + 1] = (d11 * q - d21 * p) / det
            c += 2
        else:
            ref[c] = y[c] / d[c]
            c += 1
    assert np.array_equal(bits(got), bits(ref))


@pytest.mark.parametrize("nb", [1, 2, 17, 64])
def test_unit_lower_inverse(nb):
    """The solve's 64 x 64 diagonal-block inverses of the unit lower L: each column by forward
    substitution in k order (bit for bit the loop below), and L X = I to rounding."""
    rng = np.random.default_rng(nb)
    L = np.tril(rng.standard_normal((nb, nb)) * 0.3, -1) + np.diag(rng.standard_normal(nb) * 7)  # diagonal ignored
    X = E.unit_lower_inverse(L, threads=5)
    want = np.zeros((nb, nb))
    for j in range(nb):
        want[j, j] = 1.0
        for i in range(j + 1, nb):
            s = 0.0
            for k in range(j, i):
                s = s + L[i, k] * want[k, j]
            want[i, j] = -s
    assert np.array_equal(bits(X), bits(want))
    Lu = np.tril(L, -1) + np.eye(nb)
    assert np.max(np.abs(Lu @ X - np.eye(nb))) < 1e-12


def test_rows_below_permuted():
    """A front's rows below its own columns reordered in place, every own column the same way."""
    rng = np.random.default_rng(2)
    m, w = 200, 70
    F = rng.standard_normal((m, w))
    frm = rng.permutation(m - w)
    G = E.permute_rows_below(F, w, frm, threads=7)
    assert np.array_equal(G[:w], F[:w])
    assert np.array_equal(G[w:], F[w:][frm])

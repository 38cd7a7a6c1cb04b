"""The oracle (oracle/chol_oracle.cpp) against every known answer the reference's own Cholesky
tests hold (crates/solver/src/cholesky.rs:1573-2207). The reference is Rust and cannot be built
here; these pins are what ties the CPU restatement to it."""
import ctypes as C

import numpy as np
import pytest

import helpers as H
from fieldcraft_b200.cholesky import Csr, UpperColumns
from oracle import oracle


def upper_of(csr: Csr):
    return oracle.upper_from_symmetric(csr.n, csr.ptr, csr.idx, csr.val)


def factor(csr: Csr, max_entries=2**64 - 1, cancel=None):
    ptr, idx, val = upper_of(csr)
    s = oracle.Sym(csr.n, ptr, idx, max_entries)
    return s, oracle.Fac(s, val, cancel)


def check_solve(csr: Csr, f, tol):
    """cholesky.rs:1675-1684: x = sin(0.37 i), b = A x, solve, max error below tol."""
    x = H.sin_solution(csr.n)
    b = oracle.spmv(csr.n, csr.ptr, csr.idx, csr.val, x)
    got = f.solve(b.copy())
    err = np.max(np.abs(got - x)) if csr.n else 0.0
    assert err < tol, err


def test_postorder_lists_children_first():
    # cholesky.rs:2200-2206
    N = -1
    assert oracle.postorder([2, 2, 4, 4, N, N]).tolist() == [0, 1, 2, 3, 4, 5]
    assert oracle.postorder([4, 3, 3, 4, N]).tolist() == [0, 1, 2, 3, 4]
    assert oracle.postorder([N, 0]).tolist() == [1, 0]
    assert oracle.postorder([3, N, 1, N]).tolist() == [2, 1, 0, 3]


def test_factor_and_solve_a_sparse_spd_matrix():
    # cholesky.rs:1686-1738
    a = H.grid_7x5()
    csr = Csr.from_dense(a)
    _, f = factor(csr)
    check_solve(csr, f, 1e-13)
    ptr, idx, _ = upper_of(csr)
    with pytest.raises(oracle.OracleError) as e:
        oracle.Sym(csr.n, ptr, idx, 10)
    assert e.value.code == 3  # TooLarge, refused before the numeric phase
    sing = Csr.from_dense(H.grid_7x5(shift=False))
    with pytest.raises(oracle.OracleError) as e:
        factor(sing)
    assert e.value.code == 1 and e.value.column == 34  # NotPositiveDefinite { column: n - 1 }
    flag = C.c_int32(1)
    with pytest.raises(oracle.OracleError) as e:
        factor(csr, cancel=flag)
    assert e.value.code == 6  # Cancelled
    empty = Csr(0, np.zeros(1, np.int64), np.zeros(0, np.int32), np.zeros(0))
    s, f = factor(empty, 10)
    assert s.info("entries") == 0
    one = Csr.from_dense([[4.0]])
    s, f = factor(one, 10)
    assert f.solve(np.array([2.0])).tolist() == [0.5]


@pytest.mark.parametrize("threads", [1, 2, 7])
def test_supernodes_panels_and_threads(threads):
    # cholesky.rs:1746-1905: a supernode spans panels, residual 1e-12, solve_many bit for bit
    # the single solves, the factor the same bit for bit on 1, 2 and 7 threads.
    csr = H.panels_matrix()
    oracle.set_threads(1)
    s1, one = factor(csr)
    ref = one.values()
    first = s1.array("first")
    assert np.diff(first).max() > 2 * 64
    check_solve(csr, one, 1e-12)
    rhs = [np.sin((np.arange(csr.n) * 7 + s * 13) * 0.11) for s in range(5)]
    alone = [one.solve(b.copy()) for b in rhs]
    together = one.solve(np.asfortranarray(np.stack(rhs, axis=1)))
    assert all(np.array_equal(together[:, j].view(np.uint64), alone[j].view(np.uint64)) for j in range(5))
    uptr = s1.array("uptr")
    assert np.diff(uptr).max() > 8
    assert s1.info("tasks") > 0 and s1.info("top") > 0
    oracle.set_threads(threads)
    try:
        _, other = factor(csr)
        assert np.array_equal(other.values().view(np.uint64), ref.view(np.uint64))
    finally:
        oracle.set_threads(1)


def test_micro_tiled_products_are_the_column_sums_bit_for_bit():
    # cholesky.rs:1625-1660 (the cases of :1637, LCG seed 11), without pivots.
    g = H.Lcg(11)
    for (m, w, k0, kw, p, mu, wu) in [(5, 3, 0, 3, 3, 2, 1), (40, 12, 0, 7, 7, 33, 5), (90, 20, 2, 9, 11, 79, 13),
                                      (200, 70, 0, 64, 64, 136, 6), (300, 90, 5, 30, 40, 260, 50)]:
        data = np.array([g.unit() for _ in range(H.trapezoid(m, w))])
        got = oracle.products(m, data, k0, kw, p, mu, wu, tiled=True)
        exp = oracle.products(m, data, k0, kw, p, mu, wu, tiled=False)
        assert got is not None and np.array_equal(got.view(np.uint64), exp.view(np.uint64))


def _tile_layout(tiles_full, mu, wu):
    # products' tiles hold cols = min(wu, i0 + h) columns each (the first cols * 64 entries).
    out = []
    for t, tile in enumerate(tiles_full):
        i0 = 64 * t
        h = min(64, mu - i0)
        out.append(tile[: min(wu, i0 + h) * 64])
    return np.concatenate(out)


def test_a_large_update_is_subtracted_bit_for_bit():
    # cholesky.rs:1911-1943: every entry takes the one subtraction of the naive loop.
    m, w, mu, wu = 400, 300, 400, 300
    tiles = [np.sin((t * 7919 + np.arange(wu * 64)) * 1e-3) for t in range((mu + 63) // 64)]
    start = np.cos(np.arange(H.trapezoid(m, w)) * 0.5)
    naive = start.copy()
    for c in range(wu):
        for i in range(c, mu):
            naive[H.offset(m, c) + i - c] -= tiles[i // 64][c * 64 + i % 64]
    for threads in (1, 5):
        oracle.set_threads(threads)
        rc, own = oracle.subtract(start.copy(), m, _tile_layout(tiles, mu, wu), mu, wu, np.arange(mu))
        assert rc == 0 and np.array_equal(own.view(np.uint64), naive.view(np.uint64))
    oracle.set_threads(1)


def test_an_update_outside_its_supernode_is_an_error():
    # cholesky.rs:1979-1990
    m, w = 4, 2
    tiles = np.ones(2 * 64)
    rc, own = oracle.subtract(np.zeros(H.trapezoid(m, w)), m, tiles, 2, 2, np.arange(2))
    assert rc == 0 and int(np.sum(own == -1.0)) == 3
    for rel in ([1, 0], [4, 5], [2, 3]):
        rc, _ = oracle.subtract(np.zeros(H.trapezoid(m, w)), m, tiles, 2, 2, np.array(rel))
        assert rc != 0


def test_a_tile_past_its_panel_is_an_error():
    # cholesky.rs:1949-1956
    data = np.full(64, 1.5)
    assert oracle.products(64, data, 0, 1, 0, 64, 1, tiled=True) is not None
    assert oracle.products(64, data, 0, 1, 0, 128, 1, tiled=True) is None
    assert oracle.products(64, data, 0, 1, 0, 100, 1, tiled=True) is None


def test_the_structure_of_uniform_blocks_is_the_structure_by_columns():
    # cholesky.rs:2021-2062
    dense = H.blocks40()
    csr = Csr.from_dense(dense)
    ptr, idx, _ = upper_of(csr)
    p1, c1, blocks = oracle.tree_counts(csr.n, ptr, idx)
    p2, c2, _ = oracle.tree_counts(csr.n, ptr, idx, by_columns=True)
    assert blocks and np.array_equal(p1, p2) and np.array_equal(c1, c2)
    _, f = factor(csr)
    check_solve(csr, f, 1e-10)
    a, b = 3 * 39, 1
    other = dense.copy()
    other[a, b] = other[b, a] = 0.5 if dense[a, b] == 0.0 else 0.0
    ptr, idx, _ = upper_of(Csr.from_dense(other))
    p1, c1, blocks = oracle.tree_counts(csr.n, ptr, idx)
    p2, c2, _ = oracle.tree_counts(csr.n, ptr, idx, by_columns=True)
    assert not blocks and np.array_equal(p1, p2) and np.array_equal(c1, c2)
    shorter = Csr.from_dense(dense[:-1, :-1])
    ptr, idx, _ = upper_of(shorter)
    assert not oracle.tree_counts(shorter.n, ptr, idx)[2]


def test_a_solid_models_stiffness_is_analysed_by_blocks():
    # cholesky.rs:2126-2145
    n = 5
    held = H.solid_stiffness(n)
    assert held.n == 3 * n * (n + 1) * (n + 1)
    ptr, idx, _ = upper_of(held)
    p1, c1, blocks = oracle.tree_counts(held.n, ptr, idx)
    p2, c2, _ = oracle.tree_counts(held.n, ptr, idx, by_columns=True)
    assert blocks and np.array_equal(p1, p2) and np.array_equal(c1, c2)
    _, f = factor(held)
    check_solve(held, f, 1e-9)
    rolling = H.solid_stiffness(n, roller=True)
    assert rolling.n == held.n - 1
    ptr, idx, _ = upper_of(rolling)
    p1, c1, blocks = oracle.tree_counts(rolling.n, ptr, idx)
    p2, c2, _ = oracle.tree_counts(rolling.n, ptr, idx, by_columns=True)
    assert not blocks and np.array_equal(p1, p2) and np.array_equal(c1, c2)
    _, f = factor(rolling)
    check_solve(rolling, f, 1e-9)


def test_the_matrix_is_copied_and_reordered_whole():
    # cholesky.rs:2151-2198
    rows, csr = H.band_matrix()
    n = csr.n
    ptr, idx, val = upper_of(csr)
    for k in range(n):
        exp = sorted((c, v) for c, v in rows[k] if c <= k)
        got = list(zip(idx[ptr[k]:ptr[k + 1]].tolist(), val[ptr[k]:ptr[k + 1]].tolist()))
        assert got == exp, k
    # the product's conversion agrees entry for entry
    up = UpperColumns.from_symmetric(csr)
    assert np.array_equal(up.ptr, ptr) and np.array_equal(up.idx, idx) and np.array_equal(up.val, val)
    inverse = np.arange(n)[::-1].copy()
    lptr, lidx, slot, crow, ccol = oracle.pattern(n, ptr, idx, inverse)
    for j in range(n):
        r = lidx[lptr[j]:lptr[j + 1]]
        assert np.all(np.diff(r) > 0) and r[0] == j
        exp = sorted(n - 1 - c for c, _ in rows[n - 1 - j] if c <= n - 1 - j)
        assert r.tolist() == exp
    for e in range(len(slot)):
        at = slot[e]
        assert lptr[ccol[e]] <= at < lptr[ccol[e] + 1] and lidx[at] == crow[e]


def test_cholesky_solution_keeps_the_frozen_bits():
    """crates/solver/src/ldlt.rs:774-849 (`f64_factors_keep_their_bits`, "shifted grid, definite"):
    the reference froze the FNV-1a fingerprint of the Cholesky solution of the 5x5x5 grid shifted
    by -0.5 for the exact right-hand side A x. The oracle's analysis, factor, solve and product
    reproduce it bit for bit."""
    a, below = H.shifted_grid([5, 5, 5], -0.5)
    assert below == 0
    _, f = factor(a)
    b = oracle.spmv(a.n, a.ptr, a.idx, a.val, H.exact_solution(a.n))
    assert H.fingerprint(f.solve(b.copy())) == 15069623423640047316

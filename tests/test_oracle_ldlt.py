"""The oracle's symmetric indefinite factor (oracle/chol_oracle.cpp, the LDL^T section) against
the reference's own LDL^T tests (crates/solver/src/ldlt.rs:563-1020): the bounded Bunch-Kaufman
pivots inside supernodes on the Cholesky factor's structure. The frozen fingerprints pin it bit
for bit: factor values, solutions, inertia and the count of 2 x 2 pivots."""
import numpy as np
import pytest

import helpers as H
from fieldcraft_b200 import _lib
from fieldcraft_b200.cholesky import Csr
from oracle import oracle

SINGULAR, TOO_LARGE, NOT_POSITIVE_DEFINITE = 2, 3, 1
PANEL = 64


def analysed(a: Csr, max_entries=2**64 - 1):
    ptr, idx, val = oracle.upper_from_symmetric(a.n, a.ptr, a.idx, a.val)
    return oracle.Sym(a.n, ptr, idx, max_entries), val


def ldlt(a: Csr, max_entries=2**64 - 1):
    s, val = analysed(a, max_entries)
    return s, oracle.Ldlt(s, val)


def cholesky(a: Csr):
    s, val = analysed(a)
    try:
        return oracle.Fac(s, val)
    except oracle.OracleError as e:
        assert e.code == NOT_POSITIVE_DEFINITE
        return None


def residual(a: Csr, solve, seed: float) -> float:
    """ldlt.rs:585-592: x_i = sin(0.37 (i + seed)), b = A x, solve, the largest error."""
    x = np.sin((np.arange(a.n, dtype=np.float64) + seed) * 0.37)
    b = oracle.spmv(a.n, a.ptr, a.idx, a.val, x)
    got = solve(b.copy())
    return float(np.max(np.abs(got - x))) if a.n else 0.0


def nested_dissection(xyz, adjacency):
    lib = _lib.load()
    ptr = np.zeros(len(adjacency) + 1, np.int64)
    ptr[1:] = np.cumsum([len(r) for r in adjacency])
    idx = np.array([c for r in adjacency for c in r], np.int32)
    out = np.zeros(len(adjacency), np.int64)
    xyz = np.ascontiguousarray(xyz, np.float64)
    assert lib.fc_nested_dissection(len(adjacency), _lib.ptr(xyz), _lib.ptr(ptr), _lib.ptr(idx), _lib.ptr(out)) == 0
    return out


def blocks(s: oracle.Sym, f: oracle.Ldlt):
    """Per supernode (pivots, order, rows, width)."""
    first, rptr = s.array("first"), s.array("rptr")
    piv, order = f.pivots()
    return [(piv[first[k]:first[k + 1]], order[first[k]:first[k + 1]], rptr[k + 1] - rptr[k], first[k + 1] - first[k])
            for k in range(len(first) - 1)]


FROZEN = [
    # ldlt.rs:810-849: (negative, 2 x 2 pivots, factor fingerprint, solution fingerprint)
    ("shifted grid, definite", lambda: H.shifted_grid([5, 5, 5], -0.5)[0],
     (0, 0, 12318096910519023990, 10217835541271929398)),
    ("shifted grid, indefinite", lambda: H.shifted_grid([7, 6, 5], 3.3)[0],
     (78, 9, 17838274908630861643, 4015666017640459628)),
    ("saddle point, 2 x 2 pivots", lambda: H.saddle(8, 3), (3, 3, 4028760691601933113, 11718422723752440401)),
    ("hex stiffness, indefinite", lambda: H.hex_pattern(6, 22.0, nested_dissection),
     (45, 40, 2687260628477475718, 8749587493275634787)),
]


@pytest.mark.parametrize("name,make,frozen", FROZEN, ids=[c[0] for c in FROZEN])
def test_ldlt_factors_keep_the_frozen_bits(name, make, frozen):
    """ldlt.rs:774-849 (`f64_factors_keep_their_bits`): the exact right-hand side A x with
    x_i = ((37 i mod 101) - 50) / 50; the FNV-1a fingerprints of every supernode's values and of
    the solution, the negative pivots and the 2 x 2 pivots, as the reference froze them."""
    a = make()
    _, f = ldlt(a)
    b = oracle.spmv(a.n, a.ptr, a.idx, a.val, H.exact_solution(a.n))
    x = f.solve(b.copy())
    assert (f.inertia()[1], f.two_by_two(), H.fingerprint(f.values()), H.fingerprint(x)) == frozen


def test_indefinite_systems_solve_with_their_inertia():
    """ldlt.rs:637-656: the shifted grid's inertia is the count of its eigenvalues below sigma;
    a definite matrix gets no negative pivot and Cholesky's fill."""
    for sigma in [0.0, 0.9, 3.3, 7.1]:
        a, below = H.shifted_grid([7, 6, 5], sigma)
        _, f = ldlt(a)
        assert f.inertia() == (a.n - below, below), sigma
        assert residual(a, f.solve, sigma) < 1e-10, sigma
    a, _ = H.shifted_grid([5, 5, 5], -0.5)
    s, f = ldlt(a)
    assert f.inertia()[1] == 0
    assert f.values().size == oracle.Fac(*analysed(a)).values().size
    assert residual(a, f.solve, 1.0) < 1e-12


def test_two_by_two_pivots_for_zero_diagonals():
    """ldlt.rs:690-698: a saddle point in one supernode needs 2 x 2 pivots; inertia (8, 3)."""
    a = H.saddle(8, 3)
    _, f = ldlt(a)
    assert f.inertia() == (8, 3)
    assert f.two_by_two() > 0
    assert residual(a, f.solve, 0.5) < 1e-12


def test_singular_and_hostile_matrices_are_located_errors():
    """ldlt.rs:700-734: a Laplacian with the constant in its null space is Singular at a column;
    a NaN is Singular; the cap is checked before the numeric phase; empty and 1 x 1 matrices."""
    n = 12
    rows = []
    for i in range(n):
        r = [(j, -1.0) for j in (i - 1, i + 1) if 0 <= j < n]
        r.append((i, float(len(r))))
        rows.append(r)
    with pytest.raises(oracle.OracleError) as e:
        ldlt(H.rows_to_csr(rows))
    assert e.value.code == SINGULAR and 0 <= e.value.column < n
    bad = [list(r) for r in rows]
    bad[5][0] = (bad[5][0][0], float("nan"))
    bad[4] = [(c, float("nan") if c == 5 else v) for c, v in bad[4]]
    with pytest.raises(oracle.OracleError) as e:
        ldlt(H.rows_to_csr(bad))
    assert e.value.code == SINGULAR
    a, _ = H.shifted_grid([3, 3, 3], 2.0)
    with pytest.raises(oracle.OracleError) as e:
        ldlt(a, max_entries=10)
    assert e.value.code == TOO_LARGE
    empty = Csr(0, np.zeros(1, np.int64), np.zeros(0, np.int32), np.zeros(0))
    _, f = ldlt(empty, 10)
    assert f.solve(np.zeros(0)).size == 0
    _, f = ldlt(H.rows_to_csr([[(0, -4.0)]]), 10)
    assert f.solve(np.array([2.0]))[0] == -0.5
    assert f.inertia() == (0, 1)


def test_same_factor_on_any_number_of_threads():
    """ldlt.rs:736-754: wide supernodes spanning panels; the factor and the pivot orders bit for
    bit the same on 1, 2 and 7 threads."""
    a, below = H.shifted_grid([14, 12, 10], 2.7)
    before = oracle.load().or_get_threads()
    try:
        oracle.set_threads(1)
        s, one = ldlt(a)
        assert one.inertia()[1] == below
        assert max(w for _, _, _, w in blocks(s, one)) > 2 * PANEL
        ref_values, ref_order = one.values(), one.pivots()[1]
        for threads in [2, 7]:
            oracle.set_threads(threads)
            _, other = ldlt(a)
            assert np.array_equal(other.values().view(np.uint64), ref_values.view(np.uint64)), threads
            assert np.array_equal(other.pivots()[1], ref_order), threads
    finally:
        oracle.set_threads(before)
    assert residual(a, one.solve, 0.1) < 1e-9


def test_several_right_hand_sides_solve_as_each_alone():
    """ldlt.rs:851-884: 1, 2 and 6 right-hand sides solved together give each one's solve bit
    for bit, through pivoted supernodes, local interchanges and 2 x 2 pivots, with LDL^T and
    Cholesky."""
    cases = [H.rows_to_csr([[(0, 4.0)]]), H.shifted_grid([4, 3, 3], -0.5)[0], H.shifted_grid([4, 3, 3], 2.7)[0],
             H.shifted_grid([5, 4, 3], 7.1)[0]]
    for case, a in enumerate(cases):
        factors = [ldlt(a)[1]]
        c = cholesky(a)
        if c is not None:
            factors.append(c)
        for f in factors:
            for k in [1, 2, 6]:
                i = np.arange(a.n, dtype=np.float64)
                rhs = np.stack([np.cos((i * 5 + s * 3) * 0.37) for s in range(k)], axis=1)
                alone = np.stack([f.solve(rhs[:, s].copy()) for s in range(k)], axis=1)
                together = f.solve(np.asfortranarray(rhs.copy()))
                assert np.array_equal(together.view(np.uint64), alone.view(np.uint64)), (case, k)


def test_solve_across_pivoted_supernodes():
    """ldlt.rs:886-957: two dense blocks sharing a separator, interleaved so the postorder is
    not the identity, the first needing a local interchange and a 2 x 2 pivot; then solves of
    seven matrices to 1e-10, bit for bit when repeated, and Cholesky's where it exists."""
    rows = [[] for _ in range(7)]
    for i, row in enumerate([[0.0, 0.1, 3.0], [0.1, 5.0, 0.2], [3.0, 0.2, 0.5]]):
        rows[i].extend((j, v) for j, v in enumerate(row))
    for i in range(3, 6):
        rows[i].extend((j, 4.0 if i == j else 0.25) for j in range(3, 6))
    for i in range(6):
        rows[i].append((6, 0.15))
        rows[6].append((i, 0.15))
    rows[6].append((6, 8.0))
    order = [3, 0, 4, 1, 5, 2, 6]
    inverse = [order.index(i) for i in range(7)]
    mixed = H.rows_to_csr([[(inverse[j], v) for j, v in rows[i]] for i in order])
    s, f = ldlt(mixed)
    perm = s.array("perm")
    assert np.any(perm != np.arange(7))
    bl = blocks(s, f)
    assert len(bl) > 1
    assert any(0 in piv and 1 in piv and np.any(order != np.arange(len(order))) and m > w for piv, order, m, w in bl)
    empty = Csr(0, np.zeros(1, np.int64), np.zeros(0, np.int32), np.zeros(0))
    cases = [empty, H.rows_to_csr([[(0, 4.0)]]), H.rows_to_csr([[(0, -4.0)]]), mixed,
             H.shifted_grid([4, 3, 3], -0.5)[0], H.shifted_grid([4, 3, 3], 2.7)[0], H.shifted_grid([4, 3, 3], 7.1)[0]]
    for case, a in enumerate(cases):
        _, lf = ldlt(a)
        chol = cholesky(a)
        for seed in [0.0, 0.5, 3.25]:
            expected = np.sin((np.arange(a.n, dtype=np.float64) + seed) * 0.37)
            rhs = oracle.spmv(a.n, a.ptr, a.idx, a.val, expected)
            actual = lf.solve(rhs.copy())
            assert np.all(np.abs(actual - expected) < 1e-10), case
            assert np.array_equal(lf.solve(rhs.copy()).view(np.uint64), actual.view(np.uint64))
            if chol is not None:
                assert np.all(np.abs(chol.solve(rhs.copy()) - expected) < 1e-10), case


def test_auto_selection_and_refinement():
    """ldlt.rs:959-978: Kind::Auto keeps Cholesky for a definite matrix and takes LDL^T for an
    indefinite one (one analysis serves both); refinement brings the solution to 1e-12."""
    spd, _ = H.shifted_grid([4, 4, 4], -1.0)
    assert cholesky(spd) is not None
    ind, below = H.shifted_grid([4, 4, 4], 4.4)
    s, val = analysed(ind)
    with pytest.raises(oracle.OracleError) as e:
        oracle.Fac(s, val)
    assert e.value.code == NOT_POSITIVE_DEFINITE
    f = oracle.Ldlt(s, val)
    assert f.inertia()[1] == below
    x = np.cos(np.arange(ind.n, dtype=np.float64))
    b = oracle.spmv(ind.n, ind.ptr, ind.idx, ind.val, x)
    got = oracle.solve_refined(ind.n, ind.ptr, ind.idx, ind.val, f, b, 3)
    assert np.all(np.abs(got - x) < 1e-12)


def test_shifted_stiffness_block():
    """A hex8 stiffness matrix shifted past its lowest eigenvalues (the workload of
    `bench.py --ldlt`): the pivots inside supernodes solve it to the path's 1e-10 with negative
    eigenvalues and 2 x 2 pivots present."""
    from fieldcraft_b200 import problems
    from fieldcraft_b200.cholesky import UpperColumns
    p = problems.lognormal_block(12, nrhs=3, seed=2024)
    csr = p.csr
    rows = np.repeat(np.arange(csr.n), np.diff(csr.ptr))
    on = csr.idx == rows
    val = csr.val.copy()
    val[on] -= 0.02 * float(np.mean(csr.val[on]))
    a = Csr(csr.n, csr.ptr, csr.idx, val)
    up = UpperColumns.from_symmetric(a)
    s = oracle.Sym(a.n, up.ptr, up.idx)
    f = oracle.Ldlt(s, up.val)
    assert f.inertia()[1] > 0 and f.two_by_two() > 0
    x = f.solve(p.rhs.copy(order="F"))
    for j in range(3):
        r = oracle.spmv(a.n, a.ptr, a.idx, a.val, x[:, j]) - p.rhs[:, j]
        assert np.linalg.norm(r) <= 1e-10 * np.linalg.norm(p.rhs[:, j])

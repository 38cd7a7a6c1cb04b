"""The batch's host side (fieldcraft_b200/batch.py): many systems laid end to end as one
block-diagonal matrix. The analysis of the batch keeps every supernode inside one system, and its
solution is each system's own, bit for bit (the oracle, the reference's algorithm: the systems'
operations never mix)."""
import numpy as np

from fieldcraft_b200 import problems
from fieldcraft_b200.batch import block_diagonal, factor_cost
from oracle import oracle


def test_block_diagonal_solves_as_its_systems():
    boxes = [problems.box(nx, ny, nz, float(nx), float(ny), float(nz), 210e3 * (1 + 0.1 * k), 0.3,
                          problems.node_grid(nx, ny, nz)[2] == 0)
             for k, (nx, ny, nz) in enumerate([(3, 2, 2), (5, 3, 2), (2, 2, 4)])]
    parts = [b.upper() for b in boxes]
    batch = block_diagonal(parts)
    assert batch.n == sum(p.n for p in parts)
    s = oracle.Sym(batch.n, batch.ptr, batch.idx)
    first = s.array("first")
    perm = s.array("perm")
    bounds = np.cumsum([0] + [p.n for p in parts])
    system = np.searchsorted(bounds, perm, side="right") - 1  # the system of each factor column
    for k in range(len(first) - 1):
        assert len(set(system[first[k]:first[k + 1]].tolist())) == 1, k
    f = oracle.Fac(s, batch.val)
    rng = np.random.default_rng(0)
    b = rng.standard_normal(batch.n)
    x = f.solve(b.copy())
    for i, p in enumerate(parts):
        sp = oracle.Sym(p.n, p.ptr, p.idx)
        xi = oracle.Fac(sp, p.val).solve(b[bounds[i]:bounds[i + 1]].copy())
        assert np.array_equal(x[bounds[i]:bounds[i + 1]].view(np.uint64), xi.view(np.uint64)), i


def test_factor_cost_is_the_sum_of_squared_column_counts():
    p = problems.box(4, 3, 3, 4.0, 3.0, 3.0, 210e3, 0.3, problems.node_grid(4, 3, 3)[2] == 0).upper()
    s = oracle.Sym(p.n, p.ptr, p.idx)
    first, rptr = s.array("first"), s.array("rptr")
    want = 0.0
    for k in range(len(first) - 1):
        m, w = rptr[k + 1] - rptr[k], first[k + 1] - first[k]
        want += sum(float(m - c) ** 2 for c in range(w))
    assert factor_cost(p) == want


def test_batch_abi_is_the_block_diagonal_analysis():
    """fc_chol_batch_analyse gives the analysis of diag(A_0, A_1, ...) array for array, with each
    system's first unknown; fc_chol_batch_locate maps a batch column back to (system, column)."""
    import ctypes as C

    from fieldcraft_b200 import Symbolic, _lib, problems
    from fieldcraft_b200.batch import block_diagonal
    boxes = list(problems.uneven_boxes(count=7, lo=2, hi=6, nrhs=1, seed=13))
    parts = [b.upper() for b in boxes]
    sym, offsets = Symbolic.batch(parts, 2**62)
    ref = Symbolic(block_diagonal(parts), 2**62)
    a, b = sym.arrays(), ref.arrays()
    assert a.keys() == b.keys()
    for k in a:
        assert np.array_equal(np.asarray(a[k]), np.asarray(b[k])), k
    assert offsets.tolist() == [0] + np.cumsum([p.n for p in parts]).tolist()
    lib = _lib.load()
    for col in (0, offsets[3] - 1, offsets[3], offsets[-1] - 1):
        s, loc = C.c_int32(0), C.c_int64(0)
        assert lib.fc_chol_batch_locate(len(parts), _lib.ptr(offsets), int(col), C.byref(s), C.byref(loc)) == 0
        assert offsets[s.value] + loc.value == col and 0 <= loc.value < parts[s.value].n
    assert lib.fc_chol_batch_locate(len(parts), _lib.ptr(offsets), int(offsets[-1]), C.byref(s), C.byref(loc)) != 0
    # the whole batch refused before any numeric memory, as one system would be
    from fieldcraft_b200 import TooLarge
    import pytest
    with pytest.raises(TooLarge):
        Symbolic.batch(parts, 10)

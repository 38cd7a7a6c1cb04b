"""The oracle's own input builder (oracle/fem_oracle.cpp, oracle/workloads.py) against the
library's (fieldcraft_b200/csrc/host/fem.cpp, fieldcraft_b200/problems.py): two restatements of
the reference's node graph, fill-reducing order (crates/solver/src/ordering.rs), hex8 stiffness
(crates/fem/src/element.rs) and assembly (crates/solver/src/analysis.rs:199-234,
sparse.rs:178-226), which must give the same K_ff, node order, equation numbering and loads bit
for bit. The CPU reference arm builds its inputs this way, without the library."""
import numpy as np
import pytest

from fieldcraft_b200 import problems
from oracle import oracle, workloads


def same(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return a.shape == b.shape and a.dtype == b.dtype and a.tobytes() == b.tobytes()


def check(w, p):
    assert w.n == p.n
    assert same(w.ptr.astype(np.int64), p.csr.ptr.astype(np.int64))
    assert same(w.idx, p.csr.idx)
    assert same(w.val, p.csr.val)
    assert same(w.order, p.order)
    assert same(w.eq, p.eq)
    if p.rhs is not None:
        assert same(np.asfortranarray(w.rhs), np.asfortranarray(p.rhs))


def test_cantilever():
    check(workloads.cantilever(), problems.cantilever())


@pytest.mark.parametrize("n_el", [3, 8, 17])
def test_lognormal_block(n_el):
    check(workloads.lognormal_block(n_el, nrhs=3, seed=9), problems.lognormal_block(n_el, nrhs=3, seed=9))


def test_random_field_block():
    check(workloads.field_block(10, nrhs=2), problems.field_block(10, nrhs=2))


def test_plate():
    check(workloads.plate(20, 16, 3, nrhs=2), problems.plate(20, 16, 3, nrhs=2))


def test_uneven_boxes():
    for w, p in zip(workloads.uneven_boxes(count=6, lo=2, hi=9, nrhs=2, seed=4),
                    problems.uneven_boxes(count=6, lo=2, hi=9, nrhs=2, seed=4)):
        check(w, p)


def test_a_wall_takes_the_graph_order():
    """ordering.rs:380-395 in spirit: on a thin wall the graph dissection's separators are the
    smaller, and both builders keep the order with the smaller fill (the same one)."""
    nx, ny, nz = 40, 1, 12
    i, j, k = workloads.node_grid(nx, ny, nz)
    w = workloads.box(nx, ny, nz, 40.0, 1.0, 12.0, 1000.0, 0.3, k == 0)
    p = problems.box(nx, ny, nz, 40.0, 1.0, 12.0, 1000.0, 0.3, k == 0)
    check(w, p)


def test_refuses_a_bad_material():
    i, j, k = workloads.node_grid(2, 2, 2)
    with pytest.raises(oracle.OracleError):
        workloads.box(2, 2, 2, 2.0, 2.0, 2.0, -1.0, 0.3, k == 0)

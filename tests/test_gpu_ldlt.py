"""The device LDL^T factor (FC_PRECISION_LDLT) against the oracle's (crates/solver/src/ldlt.rs):
inertia exactly, the factor's values within 1e-11 of the largest entry where the pivots are the
same (1e-9 where element growth amplifies rounding; see VALUES_TOL), the pivots themselves the
same in most supernodes (the updates run on the FP64 tensor pipe with fused multiply-adds, so an
exact tie in the rook search, common on a uniform grid, may break the other way: another, equally
valid factor), solutions within 1e-10 of the oracle's and
solve_many bit for bit the single solves, values unchanged by a solve, singular columns named.
The panel's source is also checked bit for bit on the CPU (tests/test_ldlt_panel_emulated.py) and
the solve's structure by tests/test_ldlt_fold.py."""
import numpy as np
import pytest

import helpers as H
from fieldcraft_b200 import Kind, LdltFactor, NotPositiveDefinite, Singular, Symmetric, UpperColumns
from oracle import oracle

pytestmark = pytest.mark.gpu


def both(a):
    up = UpperColumns.from_symmetric(a)
    g = LdltFactor.new(up, 2**62)
    s = oracle.Sym(up.n, up.ptr, up.idx)
    return g, oracle.Ldlt(s, up.val)


CASES = {
    "grid indefinite": lambda: H.shifted_grid([7, 6, 5], 3.3)[0],
    "saddle": lambda: H.saddle(8, 3),
    "grid definite": lambda: H.shifted_grid([5, 5, 5], -0.5)[0],
    "grid wide": lambda: H.shifted_grid([14, 12, 10], 2.7)[0],
}


# Values where the pivots agree: to rounding on the definite grid, the saddle point and the
# indefinite grid. The wide indefinite grid has supernodes of one column, which cannot pivot (rows
# below are never candidates): their small 1 x 1 pivots give multipliers up to 6 761, which carry
# the rounding of the cancellation that made each pivot (the tensor pipe's fused multiply-adds
# against the oracle's separate ones) to their ancestors, amplified; there the values agree to
# 1e-9 of the largest entry (measured 4.5e-10) and the solutions still to 1e-10 (below).
VALUES_TOL = {"grid indefinite": 1e-11, "saddle": 1e-11, "grid definite": 1e-11, "grid wide": 1e-9}


def supernode_of_entries(o, n):
    """Per value of the reference layout (supernode by supernode, each its trapezoid by columns),
    the supernode it belongs to; and per column, its supernode."""
    first, rptr = o.sym.array("first"), o.sym.array("rptr")
    ent, col = [], []
    for s in range(first.size - 1):
        w, m = int(first[s + 1] - first[s]), int(rptr[s + 1] - rptr[s])
        ent.append(np.full(w * m - w * (w - 1) // 2, s))
        col.append(np.full(w, s))
    return np.concatenate(ent), np.concatenate(col)


@pytest.mark.parametrize("name", list(CASES))
def test_factor_and_inertia_match_the_oracle(cuda, name):
    """Inertia exactly. Where a supernode took the oracle's pivots (kinds and orders), its values
    within VALUES_TOL of the largest entry. A uniform grid's matrix has many exactly equal magnitudes,
    and the tensor-pipe updates round differently from the oracle's, so the rook search may break
    a tie the other way in some supernodes: such a factor is another valid one (its solves are
    checked against the oracle's below); most supernodes must still agree."""
    a = CASES[name]()
    g, o = both(a)
    assert (g.inertia().positive, g.inertia().negative) == o.inertia()
    gv, ov = g.values(), o.values()
    assert gv.shape == ov.shape
    gp, go = g.pivots()
    op, oo = o.pivots()
    ent_sn, col_sn = supernode_of_entries(o, a.n)
    ns = int(col_sn.max()) + 1 if col_sn.size else 0
    differs = np.zeros(ns, bool)
    np.logical_or.at(differs, col_sn, (gp != op) | (go != oo))
    same = ~differs[ent_sn]
    assert differs.mean() <= 0.25, differs.mean()
    if same.any():
        assert np.max(np.abs(gv[same] - ov[same])) <= VALUES_TOL[name] * np.max(np.abs(ov))


@pytest.mark.parametrize("name", list(CASES))
def test_solves_match_the_oracle(cuda, name):
    a = CASES[name]()
    g, o = both(a)
    before = g.values()
    rng = np.random.default_rng(5)
    B = np.asfortranarray(rng.standard_normal((a.n, 7)))
    want = o.solve(B.copy(order="F"))
    got = B.copy(order="F")
    g.solve_many(got)
    assert np.max(np.abs(got - want)) <= 1e-10 * np.max(np.abs(want))
    alone = np.stack([np.ascontiguousarray(B[:, j]) for j in range(7)], axis=1)
    for j in range(7):
        x = np.ascontiguousarray(B[:, j])
        g.solve(x)
        alone[:, j] = x
    assert np.array_equal(alone.view(np.uint64), got.view(np.uint64))
    assert np.array_equal(g.values(), before)  # the solve's row moves are undone in the values


def test_singular_columns_and_refused_solves(cuda):
    n = 12
    rows = []
    for i in range(n):
        r = [(j, -1.0) for j in (i - 1, i + 1) if 0 <= j < n]
        r.append((i, float(len(r))))
        rows.append(r)
    with pytest.raises(Singular) as e:
        both(H.rows_to_csr(rows))
    assert 0 <= e.value.column < n
    g, _ = both(H.saddle(8, 3))
    with pytest.raises(ValueError):
        g.option(g.SOLVE_SCHEDULE, 1)  # the persistent solve is the Cholesky factor's only


def test_auto_selection_and_refinement(cuda):
    """ldlt.rs:959-978: Kind.AUTO keeps Cholesky for a definite matrix and takes LDL^T for an
    indefinite one; refinement brings the solution to 1e-12; Kind.DEFINITE refuses the indefinite."""
    spd, _ = H.shifted_grid([4, 4, 4], -1.0)
    assert Symmetric.new(UpperColumns.from_symmetric(spd), 2**62, Kind.AUTO).is_cholesky()
    ind, below = H.shifted_grid([4, 4, 4], 4.4)
    s = Symmetric.new(UpperColumns.from_symmetric(ind), 2**62, Kind.AUTO)
    assert not s.is_cholesky() and s.inertia().negative == below
    x = np.cos(np.arange(ind.n, dtype=np.float64))
    b = oracle.spmv(ind.n, ind.ptr, ind.idx, ind.val, x)
    s.solve_refined(ind, b, 3)
    assert np.all(np.abs(b - x) < 1e-12)
    with pytest.raises(NotPositiveDefinite):
        Symmetric.new(UpperColumns.from_symmetric(ind), 2**62, Kind.DEFINITE)


def test_plain_refinement_on_the_device(cuda):
    """fc_chol_refine_solve_device with the LDL^T factor: plain refinement (FC_OPTION_REFINEMENT = 1)
    reaches 1e-12 on an indefinite grid; conjugate gradients (the default) is refused, since it
    needs a positive definite preconditioner."""
    torch = cuda
    a, _ = H.shifted_grid([7, 6, 5], 3.3)
    g, _ = both(a)
    csr = tuple(torch.from_numpy(v).cuda() for v in (a.ptr, a.idx, a.val))
    x_true = np.sin(np.arange(a.n) * 0.37)
    b = torch.from_numpy(oracle.spmv(a.n, a.ptr, a.idx, a.val, x_true)).cuda().reshape(1, a.n)
    x = torch.zeros_like(b)
    with pytest.raises(ValueError):
        g.refine_solve_device(csr, b, x, 1, a.n, tol=1e-12, max_iter=10)
    g.option(g.REFINEMENT, 1)
    rel, its = g.refine_solve_device(csr, b, x, 1, a.n, tol=1e-12, max_iter=10)
    assert rel[0] <= 1e-12 and its >= 1
    assert np.max(np.abs(x.cpu().numpy()[0] - x_true)) < 1e-9

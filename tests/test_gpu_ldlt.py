"""The device LDL^T factor (FC_PRECISION_LDLT) against the oracle's (crates/solver/src/ldlt.rs):
inertia exactly, the factor's values within 1e-11 of the largest entry where the pivots are the
same (the updates run on the FP64 tensor pipe with fused multiply-adds, so a near tie in the rook
search may choose another, equally valid pivot), singular columns named, solves refused.

Skipped until these kernels have run on a GPU: the panel's source is checked bit for bit on the
CPU (tests/test_ldlt_panel_emulated.py); the plan and the launches have not run yet."""
import numpy as np
import pytest

import helpers as H
from fieldcraft_b200 import LdltFactor, Singular, UpperColumns
from oracle import oracle

pytestmark = [pytest.mark.gpu, pytest.mark.skip(reason="the device LDL^T has not run on a GPU yet")]


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


@pytest.mark.parametrize("name", list(CASES))
def test_factor_and_inertia_match_the_oracle(cuda, name):
    a = CASES[name]()
    g, o = both(a)
    assert (g.inertia().positive, g.inertia().negative) == o.inertia()
    gv, ov = g.values(), o.values()
    assert gv.shape == ov.shape
    if g.two_by_two() == o.two_by_two():
        assert np.max(np.abs(gv - ov)) <= 1e-11 * np.max(np.abs(ov))


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
        g.solve(np.ones(g.n))

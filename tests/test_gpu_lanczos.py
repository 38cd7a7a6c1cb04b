"""Shift-invert block Lanczos on the GPU factor (fieldcraft_b200/lanczos.py ShiftInvert): every
Lanczos block one solve_many of the Cholesky factor of K - sigma I; the lowest eigenvalues of a
hex8 stiffness matrix against the dense eigenproblem's, to 1e-8 relative.
The iteration itself is checked on the CPU against the reference's own test
(tests/test_lanczos.py)."""
import numpy as np
import pytest

from fieldcraft_b200 import problems
from fieldcraft_b200.lanczos import ShiftInvert, Wanted, lanczos

pytestmark = pytest.mark.gpu


def test_lowest_modes_of_a_stiffness_matrix(cuda):
    nx, ny, nz = 6, 3, 3
    p = problems.box(nx, ny, nz, 6.0, 3.0, 3.0, 210e3, 0.3, problems.node_grid(nx, ny, nz)[0] == 0)
    k = p.csr
    dense = np.zeros((k.n, k.n))
    for i in range(k.n):
        dense[i, k.idx[k.ptr[i]:k.ptr[i + 1]]] = k.val[k.ptr[i]:k.ptr[i + 1]]
    want = np.linalg.eigvalsh(dense)[:8]
    sigma = -0.01 * want[0]
    op = ShiftInvert(k, np.ones(k.n), sigma)
    pairs = lanczos(op, sigma, Wanted(8), 4, 120, 1e-10)
    assert np.allclose(pairs.values, want, rtol=1e-8, atol=0.0)
    for v, lam in zip(pairs.vectors, pairs.values):
        r = dense @ v - lam * v
        assert np.linalg.norm(r) <= 1e-7 * lam * np.linalg.norm(v)

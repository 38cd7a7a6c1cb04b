"""The committed golden fixtures (tests/golden/, made by make_golden.py from the oracle): the hex8
builder and the oracle reproduce them bit for bit on the CPU, and the GPU factor's solutions agree
with them to the parity tolerance."""
from pathlib import Path

import numpy as np
import pytest

from fieldcraft_b200 import Factor, UpperColumns, problems
from oracle import oracle

GOLDEN = Path(__file__).resolve().parent / "golden"
CASES = [("cantilever", problems.cantilever), ("lognormal12", lambda: problems.lognormal_block(12, nrhs=4))]


@pytest.mark.parametrize("name,make", CASES, ids=[c[0] for c in CASES])
def test_oracle_reproduces_the_golden_solution(name, make):
    g = np.load(GOLDEN / f"{name}.npz")
    p = make()
    assert p.n == int(g["n"]) and p.csr.idx.size == int(g["nnz"])
    up = UpperColumns.from_symmetric(p.csr)
    f = oracle.Fac(oracle.Sym(up.n, up.ptr, up.idx), up.val)
    assert f.values().size == int(g["entries"])
    x = f.solve(np.asfortranarray(p.rhs.copy()))
    assert np.array_equal(x.view(np.uint64), np.asarray(g["x"]).view(np.uint64))


@pytest.mark.gpu
@pytest.mark.parametrize("name,make", CASES, ids=[c[0] for c in CASES])
def test_gpu_matches_the_golden_solution(cuda, name, make):
    g = np.load(GOLDEN / f"{name}.npz")
    p = make()
    f = Factor.new(UpperColumns.from_symmetric(p.csr), 2**62)
    assert f.entries() == int(g["entries"])
    x = np.asfortranarray(p.rhs.copy())
    f.solve_many(x)
    exp = np.asarray(g["x"])
    for j in range(x.shape[1]):
        assert np.linalg.norm(x[:, j] - exp[:, j]) <= 1e-10 * np.linalg.norm(exp[:, j])

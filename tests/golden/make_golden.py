"""Writes the golden fixtures of tests/golden/ from the oracle (the reference's CPU algorithm
restated, oracle/chol_oracle.cpp): the cantilever workload (config 1: 40x4x4 hex8, 3 000 DOFs,
1 kN tip load) and the 12^3 lognormal block (4 right-hand sides). Run from the repository root:
    python tests/golden/make_golden.py
Each fixture holds the system's size, the factor's entry count and the oracle's solution."""
from pathlib import Path
import sys

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from fieldcraft_b200 import UpperColumns, problems  # noqa: E402
from oracle import oracle  # noqa: E402


def solve(p):
    up = UpperColumns.from_symmetric(p.csr)
    s = oracle.Sym(up.n, up.ptr, up.idx)
    f = oracle.Fac(s, up.val)
    return f.values().size, f.solve(np.asfortranarray(p.rhs.copy()))


def main():
    out = Path(__file__).resolve().parent
    for name, p in (("cantilever", problems.cantilever()), ("lognormal12", problems.lognormal_block(12, nrhs=4))):
        entries, x = solve(p)
        np.savez_compressed(out / f"{name}.npz", n=p.n, nnz=p.csr.idx.size, entries=entries, x=x)
        print(name, p.n, entries)


if __name__ == "__main__":
    main()

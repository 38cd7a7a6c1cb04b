"""The product's host-side symbolic analysis against the oracle's restatement of Symbolic::new
(cholesky.rs:1212-1378), array for array; and the C ABI: the library loads without a GPU and
exports every entry point include/*.h declares."""
import re
from pathlib import Path

import numpy as np
import pytest

import helpers as H
from fieldcraft_b200 import Symbolic, TooLarge, UpperColumns, _lib, problems
from fieldcraft_b200.cholesky import Csr
from oracle import oracle

ROOT = Path(__file__).resolve().parent.parent
ARRAYS = ["perm", "first", "rptr", "rows", "lptr", "lidx", "slot", "crow", "ccol", "uptr", "uk", "up1", "up2",
          "task_lo", "task_hi", "top"]


def cases():
    yield "grid7x5", Csr.from_dense(H.grid_7x5())
    yield "panels", H.panels_matrix()
    yield "blocks40", Csr.from_dense(H.blocks40())
    yield "solid5", H.solid_stiffness(5)
    yield "solid5-roller", H.solid_stiffness(5, roller=True)
    yield "band", H.band_matrix()[1]
    yield "cantilever", problems.cantilever().csr
    yield "one", Csr.from_dense([[4.0]])


@pytest.mark.parametrize("name,csr", list(cases()), ids=[c[0] for c in cases()])
def test_symbolic_is_the_oracles(name, csr):
    up = UpperColumns.from_symmetric(csr)
    mine = Symbolic(up, 2**62).arrays()
    ref = oracle.Sym(up.n, up.ptr, up.idx)
    assert mine["entries"] == ref.info("entries") and mine["ns"] == ref.info("ns")
    for k in ARRAYS:
        assert np.array_equal(mine[k], ref.array(k)), k


def test_too_large_is_refused_before_the_numeric_phase():
    up = UpperColumns.from_symmetric(Csr.from_dense(H.grid_7x5()))
    with pytest.raises(TooLarge) as e:
        Symbolic(up, 10)
    assert e.value.limit == 10 and e.value.entries > 10


def test_empty_matrix_analyses():
    up = UpperColumns(0, np.zeros(1, np.int64), np.zeros(0, np.int32), np.zeros(0))
    a = Symbolic(up, 10).arrays()
    assert a["ns"] == 0 and a["entries"] == 0


def declared_functions():
    names = []
    for h in sorted((ROOT / "include").glob("*.h")):
        text = h.read_text()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"^\s*(?:const\s+)?[A-Za-z_][A-Za-z0-9_ ]*?[\s\*]+(fc_[A-Za-z0-9_]+)\s*\(", text, re.M):
            names.append(m.group(1))
    return sorted(set(names))


def test_library_exports_every_declared_symbol():
    lib = _lib.load()
    names = declared_functions()
    assert len(names) >= 20
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    # the Python binding covers them all
    assert set(names) <= set(_lib.SIGNATURES), set(names) - set(_lib.SIGNATURES)
    assert lib.fc_version().startswith(b"fieldcraft-b200")


def test_import_round_trips_an_analysis():
    import ctypes as C
    up = UpperColumns.from_symmetric(H.panels_matrix())
    s = Symbolic(up, 2**62)
    lib = _lib.load()
    arrays = _lib.SymbolicArrays()
    assert lib.fc_symbolic_get(s.handle, C.byref(arrays)) == 0
    st = _lib.Status()
    h = C.c_void_p()
    assert lib.fc_symbolic_import(C.byref(arrays), C.byref(h), C.byref(st)) == 0
    back = _lib.SymbolicArrays()
    lib.fc_symbolic_get(h, C.byref(back))
    assert back.ns == arrays.ns and back.entries == arrays.entries
    lib.fc_symbolic_free(h)

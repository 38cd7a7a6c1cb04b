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


def _import_with(arrays, **changes):
    """fc_symbolic_import of a copy of `arrays` with some arrays replaced; returns the status."""
    import ctypes as C
    lib = _lib.load()
    a = _lib.SymbolicArrays()
    C.pointer(a)[0] = arrays
    keep = []
    for name, (values, length) in changes.items():
        dtype = np.int32 if name in ("rows", "upper_idx", "lidx", "crow", "ccol") else np.int64
        v = np.ascontiguousarray(values, dtype)
        keep.append(v)
        setattr(a, name, v.ctypes.data_as(type(getattr(a, name))))
        if length is not None:
            setattr(a, length, int(v.size))
    st = _lib.Status()
    h = C.c_void_p()
    rc = lib.fc_symbolic_import(C.byref(a), C.byref(h), C.byref(st))
    if rc == 0:
        lib.fc_symbolic_free(h)
    return rc, st.message.decode()


def test_import_refuses_inconsistent_arrays():
    """Every array the device plan indexes with is checked before it is used: a corrupted copy
    of a real analysis is refused with FC_INTERNAL and the reason, a negative length with
    FC_INVALID_ARGUMENT, and the unchanged copy is accepted."""
    import ctypes as C
    up = UpperColumns.from_symmetric(H.panels_matrix())
    s = Symbolic(up, 2**62)
    lib = _lib.load()
    arrays = _lib.SymbolicArrays()
    assert lib.fc_symbolic_get(s.handle, C.byref(arrays)) == 0
    a = s.arrays()
    n, ns = a["n"], a["ns"]
    assert ns > 2
    assert _import_with(arrays)[0] == 0

    perm = a["perm"].copy()
    perm[1] = perm[0]
    assert _import_with(arrays, perm=(perm, None)) == (5, "perm is not a permutation")

    rows = a["rows"].copy()
    t = next(t for t in range(ns) if a["rptr"][t + 1] - a["rptr"][t] > a["first"][t + 1] - a["first"][t] + 1)
    below = a["rptr"][t] + a["first"][t + 1] - a["first"][t]
    rows[below], rows[below + 1] = rows[below + 1], rows[below]
    rc, msg = _import_with(arrays, rows=(rows, None))
    assert rc == 5 and "increasing rows below" in msg
    rows = a["rows"].copy()
    rows[a["rptr"][t]] += 1  # a supernode's own column replaced
    assert _import_with(arrays, rows=(rows, None))[0] == 5
    rows = a["rows"].copy()
    rows[a["rptr"][t + 1] - 1] = n  # a row past the matrix
    assert _import_with(arrays, rows=(rows, None))[0] == 5

    first = a["first"].copy()
    first[-1] = n + 1
    assert _import_with(arrays, first=(first, None))[0] == 5

    crow, ccol = a["crow"].copy(), a["ccol"].copy()
    e = int(np.flatnonzero(crow != ccol)[0])
    crow[e], ccol[e] = ccol[e], crow[e]  # an entry above the diagonal
    assert _import_with(arrays, crow=(crow, None), ccol=(ccol, None)) == \
        (5, "an entry's coordinates outside the lower triangle")

    upper_ptr = np.zeros(n + 1, np.int64)  # spans no entries
    assert _import_with(arrays, upper_ptr=(upper_ptr, None)) == (5, "upper_ptr does not span the entries")

    bad = _lib.SymbolicArrays()
    C.pointer(bad)[0] = arrays
    bad.rows_len = -1
    st = _lib.Status()
    h = C.c_void_p()
    assert lib.fc_symbolic_import(C.byref(bad), C.byref(h), C.byref(st)) == 8  # FC_INVALID_ARGUMENT


def test_upper_columns_are_the_oracles():
    """UpperColumns::from_symmetric (cholesky.rs:112-145) in the Python mirror and in the oracle:
    the same columns, rows and values, on matrices with empty rows and unsymmetric storage order."""
    rng = np.random.default_rng(4)
    for n in [0, 1, 7, 40]:
        dense = np.zeros((n, n))
        mask = rng.random((n, n)) < 0.2
        dense[mask] = rng.standard_normal(mask.sum())
        dense = dense + dense.T
        if n > 3:
            dense[2, :] = dense[:, 2] = 0.0  # an empty row
        csr = Csr.from_dense(dense)
        up = UpperColumns.from_symmetric(csr)
        ptr, idx, val = oracle.upper_from_symmetric(csr.n, csr.ptr, csr.idx, csr.val)
        assert np.array_equal(up.ptr, ptr) and np.array_equal(up.idx, idx) and np.array_equal(up.val, val)


def test_status_codes_raise_the_reference_errors():
    """FactorError (cholesky.rs:346-361) from the ABI's codes: the variant, its column or sizes."""
    import fieldcraft_b200.cholesky as M
    cases = [(1, M.NotPositiveDefinite), (2, M.Singular), (3, M.TooLarge), (4, M.OutOfMemory), (5, M.Internal),
             (6, M.Cancelled), (7, M.Timeout), (8, ValueError), (9, M.DeviceError)]
    for code, kind in cases:
        st = _lib.Status()
        st.code, st.column, st.entries, st.limit, st.message = code, 17, 100, 10, b"why"
        with pytest.raises(kind) as e:
            M.raise_for(st)
        if code in (1, 2):
            assert e.value.column == 17
        if code == 3:
            assert (e.value.entries, e.value.limit) == (100, 10)
    st = _lib.Status()
    M.raise_for(st)  # FC_OK

"""ORACLE (test infrastructure): ctypes access to ``liboracle.so``, the CPU restatement of the
reference's supernodal Cholesky and LDL^T (chol_oracle.cpp). Used only by the tests, by the smoke
check and by the benchmark's CPU-baseline leg, as the checker and the timed CPU reference."""
from __future__ import annotations

import ctypes as C
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "liboracle.so"
i32, i64, u64, P = C.c_int32, C.c_int64, C.c_uint64, C.c_void_p

_SIG = {
    "or_set_threads": (None, [C.c_int]),
    "or_get_threads": (C.c_int, []),
    "or_upper_from_symmetric": (i64, [i64, P, P, P, P, P, P]),
    "or_analyse": (C.c_int, [i64, P, P, u64, C.POINTER(P), P]),
    "or_sym_free": (None, [P]),
    "or_sym_info": (i64, [P, C.c_int]),
    "or_sym_export": (C.c_int, [P, C.c_int, P]),
    "or_pattern": (C.c_int, [i64, P, P, P, P, P, P, P, P]),
    "or_tree_counts": (C.c_int, [i64, P, P, C.c_int, P, P]),
    "or_postorder": (C.c_int, [i64, P, P]),
    "or_factor_new": (C.c_int, [P, P, P, C.POINTER(P), P]),
    "or_factor_free": (None, [P]),
    "or_factor_values": (i64, [P, P]),
    "or_solve": (C.c_int, [P, P, i64]),
    "or_spmv": (None, [i64, P, P, P, P, P]),
    "or_products": (i64, [i64, P, i64, i64, i64, i64, i64, i64, C.c_int, P]),
    "or_subtract": (C.c_int, [P, i64, i64, P, i64, i64, P]),
    "or_ldlt_new": (C.c_int, [P, P, P, C.POINTER(P), P]),
    "or_ldlt_free": (None, [P]),
    "or_ldlt_values": (i64, [P, P]),
    "or_ldlt_pivots": (None, [P, P, P]),
    "or_ldlt_info": (i64, [P, C.c_int]),
    "or_ldlt_solve": (C.c_int, [P, P, i64]),
    "or_fem_box": (C.c_int, [i64, i64, i64, C.c_double, C.c_double, C.c_double, P, C.c_double, P, C.c_int,
                             C.POINTER(P)]),
    "or_fem_info": (i64, [P, C.c_int]),
    "or_fem_export": (None, [P, P, P, P, P, P]),
    "or_fem_free": (None, [P]),
}
_lib = None

NS_INFO = {"n": 0, "ns": 1, "entries": 2, "rows": 3, "lower": 4, "updates": 5, "tasks": 6, "top": 7, "blocks": 8,
           "nnz": 9}
EXPORT = {"perm": (0, "n"), "first": (1, "ns+1"), "rptr": (2, "ns+1"), "rows": (3, "rows"), "sparent": (4, "ns"),
          "lptr": (5, "n+1"), "lidx": (6, "lower"), "slot": (7, "nnz"), "crow": (8, "nnz"), "ccol": (9, "nnz"),
          "uptr": (10, "ns+1"), "uk": (11, "updates"), "up1": (12, "updates"), "up2": (13, "updates"),
          "task_lo": (14, "tasks"), "task_hi": (15, "tasks"), "top": (16, "top")}


def build():
    subprocess.run(["make", "-s", "-C", str(HERE)], check=True)


def _stale() -> bool:
    if not LIB.exists():
        return True
    t = LIB.stat().st_mtime
    return any(src.stat().st_mtime > t for src in HERE.glob("*.cpp") if src.exists())


def load():
    global _lib
    if _lib is None:
        if _stale():
            build()
        lib = C.CDLL(str(LIB))
        for k, (r, a) in _SIG.items():
            f = getattr(lib, k)
            f.restype, f.argtypes = r, a
        _lib = lib
    return _lib


def _p(a):
    return None if a is None else a.ctypes.data


def set_threads(t: int):
    load().or_set_threads(int(t))


def fem_box(nx, ny, nz, lx, ly, lz, young, nu, clamped_nodes, threads=0):
    """The oracle's own K_ff of an nx x ny x nz hex8 box (fem_oracle.cpp): `young` per element
    (label order) or one value, `clamped_nodes` a boolean mask over the nodes. Returns (n, ptr,
    idx, val, order, eq): K_ff by rows, the node elimination order and each mesh DOF's equation."""
    import os
    lib = load()
    ne = nx * ny * nz
    young = np.ascontiguousarray(np.broadcast_to(np.asarray(young, np.float64), (ne,)), np.float64)
    clamped = np.ascontiguousarray(clamped_nodes, np.uint8)
    h = P()
    rc = lib.or_fem_box(nx, ny, nz, lx, ly, lz, young.ctypes.data, float(nu), clamped.ctypes.data,
                        int(threads or os.cpu_count() or 1), C.byref(h))
    if rc != 0:
        raise OracleError(rc)
    try:
        n, nnz, nodes = (int(lib.or_fem_info(h, w)) for w in range(3))
        ptr, idx, val = np.empty(n + 1, np.int64), np.empty(nnz, np.int32), np.empty(nnz)
        order, eq = np.empty(nodes, np.int64), np.empty(3 * nodes, np.int64)
        lib.or_fem_export(h, ptr.ctypes.data, idx.ctypes.data, val.ctypes.data, order.ctypes.data, eq.ctypes.data)
    finally:
        lib.or_fem_free(h)
    return n, ptr, idx, val, order, eq


class OracleError(Exception):
    def __init__(self, code, column=-1, info=None):
        super().__init__(f"oracle code {code} column {column} info {info}")
        self.code, self.column, self.info = code, column, info


class Sym:
    def __init__(self, n, ptr, idx, max_entries=2**64 - 1):
        lib = load()
        self.ptr = np.ascontiguousarray(ptr, np.int64)
        self.idx = np.ascontiguousarray(idx, np.int32)
        info = np.zeros(2, np.int64)
        h = P()
        rc = lib.or_analyse(int(n), _p(self.ptr), _p(self.idx), int(min(max_entries, 2**64 - 1)), C.byref(h), _p(info))
        if rc != 0:
            raise OracleError(rc, info=tuple(info))
        self.h = h

    def info(self, what):
        return int(load().or_sym_info(self.h, NS_INFO[what]))

    def array(self, name):
        code, size = EXPORT[name]
        if size == "ns+1":
            count = self.info("ns") + 1
        elif size == "n+1":
            count = self.info("n") + 1
        else:
            count = self.info(size)
        out = np.zeros(max(count, 0), np.int64)
        if count > 0:
            load().or_sym_export(self.h, code, _p(out))
        return out

    def __del__(self):
        if getattr(self, "h", None):
            load().or_sym_free(self.h)
            self.h = None


class Fac:
    def __init__(self, sym: Sym, upper_val, cancel=None):
        self.sym = sym
        v = np.ascontiguousarray(upper_val, np.float64)
        col = np.zeros(1, np.int64)
        h = P()
        rc = load().or_factor_new(sym.h, _p(v), C.byref(cancel) if cancel is not None else None, C.byref(h), _p(col))
        if rc != 0:
            raise OracleError(rc, int(col[0]))
        self.h = h

    def values(self):
        count = load().or_factor_values(self.h, None)
        out = np.empty(count, np.float64)
        load().or_factor_values(self.h, _p(out))
        return out

    def solve(self, b):
        """b: [n] or Fortran [n, k]; solved in place and returned."""
        b = np.asfortranarray(b, dtype=np.float64)
        k = 1 if b.ndim == 1 else b.shape[1]
        load().or_solve(self.h, _p(b), int(k))
        return b

    def __del__(self):
        if getattr(self, "h", None):
            load().or_factor_free(self.h)
            self.h = None


class Ldlt:
    """The symmetric indefinite factor P A P^T = L D L^T on an analysis (ldlt.rs LdltFactor):
    bounded Bunch-Kaufman pivots inside supernodes."""

    def __init__(self, sym: Sym, upper_val, cancel=None):
        self.sym = sym
        v = np.ascontiguousarray(upper_val, np.float64)
        col = np.zeros(1, np.int64)
        h = P()
        rc = load().or_ldlt_new(sym.h, _p(v), C.byref(cancel) if cancel is not None else None, C.byref(h), _p(col))
        if rc != 0:
            raise OracleError(rc, int(col[0]))
        self.h = h

    def values(self):
        count = load().or_ldlt_values(self.h, None)
        out = np.empty(count, np.float64)
        load().or_ldlt_values(self.h, _p(out))
        return out

    def pivots(self):
        """(pivots, order): per postorder column its pivot kind (0 one, 1 first, 2 second of a
        2 x 2) and the supernode-local column at that pivot position."""
        n = self.sym.info("n")
        piv, order = np.zeros(n, np.int64), np.zeros(n, np.int64)
        load().or_ldlt_pivots(self.h, _p(piv), _p(order))
        return piv, order

    def two_by_two(self) -> int:
        return int(load().or_ldlt_info(self.h, 0))

    def inertia(self):
        """(positive, negative) eigenvalue counts."""
        return int(load().or_ldlt_info(self.h, 1)), int(load().or_ldlt_info(self.h, 2))

    def solve(self, b):
        """b: [n] or Fortran [n, k]; solved in place and returned."""
        b = np.asfortranarray(b, dtype=np.float64)
        k = 1 if b.ndim == 1 else b.shape[1]
        load().or_ldlt_solve(self.h, _p(b), int(k))
        return b

    def __del__(self):
        if getattr(self, "h", None):
            load().or_ldlt_free(self.h)
            self.h = None


def solve_refined(n, ptr, idx, val, factor, b, steps: int, cholesky: bool = False):
    """Symmetric::solve_refined (ldlt.rs:524-560): solve, then x += A^-1 (b - A x) while the
    residual's largest magnitude shrinks, at most `steps` times; a Cholesky solution is returned
    as solved. `factor` has .solve; (ptr, idx, val) is the matrix by rows, both triangles."""
    rhs = np.array(b, np.float64)
    x = factor.solve(rhs.copy())
    if cholesky:
        return x
    r = rhs - spmv(n, ptr, idx, val, x)
    size = float(np.max(np.abs(r))) if n else 0.0
    for _ in range(steps):
        if not size > 0.0:
            break
        trial = x + factor.solve(r.copy())
        nxt = rhs - spmv(n, ptr, idx, val, trial)
        nsize = float(np.max(np.abs(nxt)))
        if not nsize < size:
            break
        x, r, size = trial, nxt, nsize
    return x


def upper_from_symmetric(n, ptr, idx, val):
    lib = load()
    ptr = np.ascontiguousarray(ptr, np.int64)
    idx = np.ascontiguousarray(idx, np.int32)
    val = np.ascontiguousarray(val, np.float64)
    total = lib.or_upper_from_symmetric(int(n), _p(ptr), _p(idx), _p(val), None, None, None)
    op = np.zeros(n + 1, np.int64)
    oi = np.zeros(total, np.int32)
    ov = np.zeros(total, np.float64)
    lib.or_upper_from_symmetric(int(n), _p(ptr), _p(idx), _p(val), _p(op), _p(oi), _p(ov))
    return op, oi, ov


def spmv(n, ptr, idx, val, x):
    ptr = np.ascontiguousarray(ptr, np.int64)
    idx = np.ascontiguousarray(idx, np.int32)
    val = np.ascontiguousarray(val, np.float64)
    x = np.ascontiguousarray(x, np.float64)
    y = np.empty(n, np.float64)
    load().or_spmv(int(n), _p(ptr), _p(idx), _p(val), _p(x), _p(y))
    return y


def tree_counts(n, ptr, idx, by_columns=False):
    ptr = np.ascontiguousarray(ptr, np.int64)
    idx = np.ascontiguousarray(idx, np.int32)
    parent = np.zeros(n, np.int64)
    counts = np.zeros(n, np.int64)
    blocks = load().or_tree_counts(int(n), _p(ptr), _p(idx), 1 if by_columns else 0, _p(parent), _p(counts))
    return parent, counts, bool(blocks)


def postorder(parent):
    parent = np.ascontiguousarray(parent, np.int64)
    out = np.zeros(parent.size, np.int64)
    load().or_postorder(int(parent.size), _p(parent), _p(out))
    return out


def pattern(n, ptr, idx, inverse):
    ptr = np.ascontiguousarray(ptr, np.int64)
    idx = np.ascontiguousarray(idx, np.int32)
    inverse = np.ascontiguousarray(inverse, np.int64)
    nnz = int(ptr[-1])
    lptr = np.zeros(n + 1, np.int64)
    lidx = np.zeros(nnz, np.int32)
    slot = np.zeros(nnz, np.int64)
    crow = np.zeros(nnz, np.int32)
    ccol = np.zeros(nnz, np.int32)
    load().or_pattern(int(n), _p(ptr), _p(idx), _p(inverse), _p(lptr), _p(lidx), _p(slot), _p(crow), _p(ccol))
    return lptr, lidx, slot, crow, ccol


def products(m, data, k0, kw, p, mu, wu, tiled):
    data = np.ascontiguousarray(data, np.float64)
    count = load().or_products(int(m), _p(data), int(data.size), k0, kw, p, mu, wu, 1 if tiled else 0, None)
    if count < 0:
        return None
    out = np.empty(count, np.float64)
    load().or_products(int(m), _p(data), int(data.size), k0, kw, p, mu, wu, 1 if tiled else 0, _p(out))
    return out


def subtract(own, m, tiles_flat, mu, wu, rel):
    own = np.ascontiguousarray(own, np.float64)
    tiles_flat = np.ascontiguousarray(tiles_flat, np.float64)
    rel = np.ascontiguousarray(rel, np.int64)
    rc = load().or_subtract(_p(own), int(own.size), int(m), _p(tiles_flat), int(mu), int(wu), _p(rel))
    return rc, own

"""The reference's Cholesky API for this path, on a B200.

Mirrors ``crates/solver/src/cholesky.rs`` of FieldCraft 0.8.1: ``UpperColumns`` (:102-145),
``Factor::new`` (:1545), ``Factor::entries`` (:1557), ``Factor::solve`` (:1562),
``Factor::solve_many`` (:1568) and ``FactorError`` (:346-361), with the same argument meanings and
the same errors. The symbolic analysis runs on the host (bit for bit the reference's); the numeric
phase and the solves run on the GPU through ``libfieldcraft_b200.so``; there is no CPU path.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _lib
from ._lib import Status

FC_OK, FC_NOT_POSITIVE_DEFINITE, FC_SINGULAR, FC_TOO_LARGE, FC_OUT_OF_MEMORY = 0, 1, 2, 3, 4
FC_INTERNAL, FC_CANCELLED, FC_TIMEOUT, FC_INVALID_ARGUMENT, FC_CUDA_ERROR = 5, 6, 7, 8, 9
FP64, FP32_IR, LDLT = 0, 1, 2


class FactorError(Exception):
    """Why a factorization stopped (cholesky.rs:346-361)."""


class NotPositiveDefinite(FactorError):
    def __init__(self, column: int):
        super().__init__(f"NotPositiveDefinite {{ column: {column} }}")
        self.column = column

    def __eq__(self, other):
        return isinstance(other, NotPositiveDefinite) and other.column == self.column


class Singular(FactorError):
    def __init__(self, column: int):
        super().__init__(f"Singular {{ column: {column} }}")
        self.column = column


class TooLarge(FactorError):
    def __init__(self, entries: int, limit: int):
        super().__init__(f"TooLarge {{ entries: {entries}, limit: {limit} }}")
        self.entries, self.limit = entries, limit


class OutOfMemory(FactorError):
    def __init__(self, entries: int):
        super().__init__(f"OutOfMemory {{ entries: {entries} }}")
        self.entries = entries


class Internal(FactorError):
    def __init__(self, what: str):
        super().__init__(f"Internal({what!r})")
        self.what = what


class Cancelled(FactorError):
    def __init__(self):
        super().__init__("Cancelled")


class DeviceError(RuntimeError):
    """The CUDA runtime refused a call (no device, a failed launch)."""


class Timeout(RuntimeError):
    """A bounded device wait gave up."""


def raise_for(st: Status):
    code = st.code
    msg = st.message.decode(errors="replace")
    if code == FC_OK:
        return
    if code == FC_NOT_POSITIVE_DEFINITE:
        raise NotPositiveDefinite(int(st.column))
    if code == FC_SINGULAR:
        raise Singular(int(st.column))
    if code == FC_TOO_LARGE:
        raise TooLarge(int(st.entries), int(st.limit))
    if code == FC_OUT_OF_MEMORY:
        raise OutOfMemory(int(st.entries))
    if code == FC_INTERNAL:
        raise Internal(msg)
    if code == FC_CANCELLED:
        raise Cancelled()
    if code == FC_TIMEOUT:
        raise Timeout(msg)
    if code == FC_INVALID_ARGUMENT:
        raise ValueError(msg or "invalid argument")
    raise DeviceError(msg or f"code {code}")


@dataclass
class Csr:
    """A square sparse matrix by rows, both triangles, sorted columns (sparse.rs:26-31)."""
    n: int
    ptr: np.ndarray  # int64 [n+1]
    idx: np.ndarray  # int32 [nnz]
    val: np.ndarray  # float64 [nnz]

    @staticmethod
    def from_dense(a) -> "Csr":
        a = np.asarray(a, dtype=np.float64)
        n = a.shape[0]
        ptr, idx, val = [0], [], []
        for row in a:
            nz = np.nonzero(row)[0]
            idx.extend(nz.tolist())
            val.extend(row[nz].tolist())
            ptr.append(len(idx))
        return Csr(n, np.array(ptr, np.int64), np.array(idx, np.int32), np.array(val, np.float64))


@dataclass
class UpperColumns:
    """The upper triangle by columns: column k holds A(i, k) for i <= k, rows sorted (cholesky.rs:102-107)."""
    n: int
    ptr: np.ndarray  # int64 [n+1]
    idx: np.ndarray  # int32
    val: np.ndarray  # float64

    @staticmethod
    def from_symmetric(a: Csr) -> "UpperColumns":
        """Row k's entries with column <= k are column k of the upper triangle (cholesky.rs:112-145)."""
        n = a.n
        rows = np.repeat(np.arange(n, dtype=np.int64), np.diff(a.ptr))
        keep = a.idx.astype(np.int64) <= rows
        counts = np.bincount(rows[keep], minlength=n) if n else np.zeros(0, np.int64)
        ptr = np.zeros(n + 1, np.int64)
        np.cumsum(counts, out=ptr[1:])
        return UpperColumns(n, ptr, np.ascontiguousarray(a.idx[keep], np.int32),
                            np.ascontiguousarray(a.val[keep], np.float64))


class Symbolic:
    """The structure of the factor (Symbolic::new, cholesky.rs:1212-1378), on the host."""

    def __init__(self, a: UpperColumns, max_entries: int):
        lib = _lib.load()
        self._ptr = np.ascontiguousarray(a.ptr, np.int64)
        self._idx = np.ascontiguousarray(a.idx, np.int32)
        st = Status()
        h = C.c_void_p()
        lib.fc_symbolic_analyse(int(a.n), _lib.ptr(self._ptr), _lib.ptr(self._idx),
                                min(int(max_entries), 2**64 - 1), C.byref(h), C.byref(st))
        raise_for(st)
        self.handle = h
        self.n = a.n

    @staticmethod
    def batch(parts: list[UpperColumns], max_entries: int) -> tuple["Symbolic", np.ndarray]:
        """The analysis of independent systems as one block-diagonal matrix (fc_chol_batch_analyse):
        (the Symbolic, each system's first unknown with the total last)."""
        lib = _lib.load()
        count = len(parts)
        ns = np.array([p.n for p in parts], np.int64)
        ptrs = [np.ascontiguousarray(p.ptr, np.int64) for p in parts]
        idxs = [np.ascontiguousarray(p.idx, np.int32) for p in parts]
        P = (C.c_void_p * max(count, 1))(*[C.c_void_p(a.ctypes.data) for a in ptrs])
        I = (C.c_void_p * max(count, 1))(*[C.c_void_p(a.ctypes.data) for a in idxs])  # noqa: E741
        offsets = np.zeros(count + 1, np.int64)
        st = Status()
        h = C.c_void_p()
        lib.fc_chol_batch_analyse(count, _lib.ptr(ns), P, I, min(int(max_entries), 2**64 - 1), C.byref(h),
                                  _lib.ptr(offsets), C.byref(st))
        raise_for(st)
        sym = Symbolic.__new__(Symbolic)
        sym.handle = h
        sym.n = int(offsets[-1]) if count else 0
        sym._keep = (ptrs, idxs)
        return sym, offsets

    def arrays(self) -> dict:
        """Copies of the analysis' arrays (fc_symbolic_arrays)."""
        lib = _lib.load()
        out = _lib.SymbolicArrays()
        lib.fc_symbolic_get(self.handle, C.byref(out))

        def take(p, count, dtype):
            if count == 0:
                return np.zeros(0, dtype)
            return np.ctypeslib.as_array(p, shape=(count,)).astype(dtype, copy=True)

        ns, n, nnz = out.ns, out.n, out.nnz
        return {
            "n": n, "ns": ns, "entries": out.entries,
            "perm": take(out.perm, n, np.int64), "first": take(out.first, ns + 1, np.int64),
            "rptr": take(out.rptr, ns + 1, np.int64), "rows": take(out.rows, out.rows_len, np.int64),
            "lptr": take(out.lptr, n + 1, np.int64), "lidx": take(out.lidx, out.lower_len, np.int64),
            "slot": take(out.slot, nnz, np.int64), "crow": take(out.crow, nnz, np.int64),
            "ccol": take(out.ccol, nnz, np.int64), "uptr": take(out.uptr, ns + 1, np.int64),
            "uk": take(out.uk, out.updates_len, np.int64), "up1": take(out.up1, out.updates_len, np.int64),
            "up2": take(out.up2, out.updates_len, np.int64),
            "task_lo": take(out.task_lo, out.tasks_len, np.int64),
            "task_hi": take(out.task_hi, out.tasks_len, np.int64), "top": take(out.top, out.top_len, np.int64),
        }

    def __del__(self):
        h = getattr(self, "handle", None)
        if h:
            try:
                _lib.load().fc_symbolic_free(h)
            except TypeError:  # interpreter shutdown: the module's globals are gone
                pass
            self.handle = None


class Factor:
    """A Cholesky factor on the GPU: L by supernodes for the matrix in postorder (cholesky.rs:1534)."""

    def __init__(self, symbolic: Symbolic, precision: int = FP64, device: int = 0):
        lib = _lib.load()
        st = Status()
        h = C.c_void_p()
        lib.fc_chol_create(symbolic.handle, int(precision), int(device), C.byref(h), C.byref(st))
        raise_for(st)
        self.handle = h
        self.n = symbolic.n
        self.symbolic = symbolic

    @staticmethod
    def new(a: UpperColumns, max_entries: int, precision: int = FP64, device: int = 0,
            cancel: C.c_int32 | None = None) -> "Factor":
        """Factor::new (cholesky.rs:1545): the analysis (refused with TooLarge above max_entries),
        then the numeric phase on the GPU. `cancel`, a ctypes int32 set non-zero from another
        thread, stops the factorization between levels of the supernodal tree (Cancelled)."""
        sym = Symbolic(a, max_entries)
        f = Factor(sym, precision, device)
        f.factor(a.val, cancel)
        return f

    def factor(self, val: np.ndarray, cancel: C.c_int32 | None = None):
        """Symbolic::numeric + factor with new values on the analysed pattern."""
        v = np.ascontiguousarray(val, np.float64)
        st = Status()
        _lib.load().fc_chol_factor(self.handle, _lib.ptr(v), int(v.size),
                                   C.byref(cancel) if cancel is not None else None, C.byref(st))
        raise_for(st)

    def entries(self) -> int:
        return int(_lib.load().fc_chol_entries(self.handle))

    def solve(self, b: np.ndarray):
        """Solve A x = b in place (cholesky.rs:1562); b of the factor's length."""
        if b.ndim != 1 or b.shape[0] != self.n or b.dtype != np.float64 or not b.flags.c_contiguous:
            raise ValueError("right-hand side length")
        self._solve(b, 1, self.n)

    def solve_many(self, bs):
        """Solve for each of `bs` in place (cholesky.rs:1568): a list of 1-D arrays, or a 2-D
        Fortran-ordered array whose columns are the right-hand sides."""
        if isinstance(bs, np.ndarray) and bs.ndim == 2:
            if bs.shape[0] != self.n or not bs.flags.f_contiguous or bs.dtype != np.float64:
                raise ValueError("right-hand side length")
            self._solve(bs, bs.shape[1], self.n)
            return
        if any(b.shape != (self.n,) for b in bs):
            raise ValueError("right-hand side length")
        if not bs:
            return
        block = np.asfortranarray(np.stack(bs, axis=1))
        self._solve(block, block.shape[1], self.n)
        for j, b in enumerate(bs):
            b[:] = block[:, j]

    def _solve(self, b, nrhs, ld):
        st = Status()
        _lib.load().fc_chol_solve(self.handle, _lib.ptr(b), int(nrhs), int(ld), C.byref(st))
        raise_for(st)

    def solve_device(self, b_tensor, nrhs: int, ld: int):
        """Solve in place on device memory (a CUDA tensor, column-major n x nrhs, leading dimension ld)."""
        st = Status()
        _lib.load().fc_chol_solve_device(self.handle, C.c_void_p(b_tensor.data_ptr()), int(nrhs), int(ld),
                                         C.byref(st))
        raise_for(st)

    def refine_solve_device(self, csr_device, b, x, nrhs: int, ld: int, tol: float = 1e-10, max_iter: int = 20):
        """Iterative refinement in FP64 around this factor (the mixed-precision mode's FP32 factor or
        the FP64 one): solves A x = b to ||b - A x|| <= tol ||b|| per right-hand side. csr_device =
        (ptr, idx, val) CUDA tensors of A by rows; b, x CUDA tensors, column-major n x nrhs with
        leading dimension ld. Returns (relative residuals, iterations); raises Timeout if max_iter
        solves were not enough."""
        ptr, idx, val = csr_device
        rel = np.zeros(nrhs)
        it = C.c_int32(0)
        st = Status()
        _lib.load().fc_chol_refine_solve_device(self.handle, C.c_void_p(ptr.data_ptr()), C.c_void_p(idx.data_ptr()),
                                                C.c_void_p(val.data_ptr()), C.c_void_p(b.data_ptr()),
                                                C.c_void_p(x.data_ptr()), int(nrhs), int(ld), float(tol),
                                                int(max_iter), _lib.ptr(rel), C.byref(it), C.byref(st))
        if st.code == FC_TIMEOUT:
            raise Timeout(f"{st.message.decode()} after {it.value} solves, residuals {rel}")
        raise_for(st)
        return rel, it.value

    def values(self) -> np.ndarray:
        """The factor in the reference's layout: per supernode its lower trapezoid by columns."""
        out = np.empty(self.entries(), np.float64)
        st = Status()
        _lib.load().fc_chol_values(self.handle, _lib.ptr(out), C.byref(st))
        raise_for(st)
        return out

    def stat(self, what: int) -> int:
        return int(_lib.load().fc_chol_stat(self.handle, what))

    # fc_chol_option: the solve's schedule (0 level by level, 1 persistent), the persistent solve's
    # wait limit in nanoseconds, and (tests) a planted dependency that no task meets
    SOLVE_SCHEDULE, WAIT_LIMIT_NS, PLANT_UNMET_WAIT, TRACE, REFINEMENT, FP32_UPDATES, SOLVE_CLUSTER, SOLVE_NARROW, \
        SOLVE_DEEP, CHILDREN_FIRST, SOLVE_PDL = 1, 2, 3, 4, 5, 6, 7, 8, 9, 10, 11

    def option(self, option: int, value: int):
        if _lib.load().fc_chol_option(self.handle, int(option), int(value)) != 0:
            raise ValueError(f"option {option} = {value}")

    def set_stream(self, stream_ptr: int | None):
        _lib.load().fc_chol_set_stream(self.handle, C.c_void_p(stream_ptr) if stream_ptr else None)

    def close(self):
        h = getattr(self, "handle", None)
        if h:
            _lib.load().fc_chol_destroy(h)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except TypeError:  # interpreter shutdown: the module's globals are gone
            pass


@dataclass(frozen=True)
class Inertia:
    """The counts of positive and negative eigenvalues (ldlt.rs:83-89)."""
    positive: int
    negative: int


class LdltFactor(Factor):
    """The symmetric indefinite factor P A P^T = L D L^T on the GPU (LdltFactor, ldlt.rs:365-447):
    bounded Bunch-Kaufman pivots inside the supernodes of the same analysis. Factors, values,
    inertia, solve and solve_many (level by level; the refined solve is the Cholesky factor's)."""

    def __init__(self, symbolic: Symbolic, device: int = 0):
        super().__init__(symbolic, LDLT, device)

    @staticmethod
    def new(a: UpperColumns, max_entries: int, device: int = 0, cancel: C.c_int32 | None = None) -> "LdltFactor":
        """LdltFactor::new (ldlt.rs:374-376): the analysis, then the pivoted numeric phase
        (Singular for a column with no acceptable pivot in its supernode)."""
        f = LdltFactor(Symbolic(a, max_entries), device)
        f.factor(a.val, cancel)
        return f

    def _counts(self):
        pos, neg, two = C.c_int64(0), C.c_int64(0), C.c_int64(0)
        st = Status()
        _lib.load().fc_chol_inertia(self.handle, C.byref(pos), C.byref(neg), C.byref(two), C.byref(st))
        raise_for(st)
        return pos.value, neg.value, two.value

    def inertia(self) -> Inertia:
        """Sylvester's law on D (ldlt.rs:415-447)."""
        pos, neg, _ = self._counts()
        return Inertia(pos, neg)

    def pivots(self):
        """(pivots, order): per column in postorder its pivot kind (0 one, 1 first, 2 second of a
        2 x 2) and the supernode-local column at that pivot position, as the oracle reports them."""
        piv = np.zeros(self.n, np.int8)
        order = np.zeros(self.n, np.int32)
        st = Status()
        _lib.load().fc_chol_ldlt_pivots(self.handle, _lib.ptr(piv), _lib.ptr(order), C.byref(st))
        raise_for(st)
        return piv.astype(np.int64), order.astype(np.int64)

    def two_by_two(self) -> int:
        return self._counts()[2]


class Kind:
    """Which factorization a symmetric solve uses (ldlt.rs:452-463)."""
    DEFINITE, INDEFINITE, AUTO = 0, 1, 2


class Symmetric:
    """A factored symmetric matrix, Cholesky or LDL^T (ldlt.rs:465-561): Kind.AUTO tries Cholesky
    and takes LDL^T when the matrix is not positive definite, one analysis serving both."""

    def __init__(self, factor: Factor):
        self.factor = factor

    @staticmethod
    def new(a: UpperColumns, max_entries: int, kind: int = Kind.DEFINITE, device: int = 0) -> "Symmetric":
        if kind == Kind.DEFINITE:
            return Symmetric(Factor.new(a, max_entries, FP64, device))
        if kind == Kind.INDEFINITE:
            return Symmetric(LdltFactor.new(a, max_entries, device))
        sym = Symbolic(a, max_entries)
        f = Factor(sym, FP64, device)
        try:
            f.factor(a.val)
            return Symmetric(f)
        except NotPositiveDefinite:
            f.close()
        g = LdltFactor(sym, device)
        g.factor(a.val)
        return Symmetric(g)

    @property
    def n(self) -> int:
        return self.factor.n

    def is_cholesky(self) -> bool:
        return not isinstance(self.factor, LdltFactor)

    def entries(self) -> int:
        return self.factor.entries()

    def inertia(self) -> Inertia:
        """A Cholesky factor's matrix is positive definite (ldlt.rs:500-506)."""
        if self.is_cholesky():
            return Inertia(self.n, 0)
        return self.factor.inertia()

    def solve(self, b: np.ndarray):
        self.factor.solve(b)

    def solve_many(self, bs):
        self.factor.solve_many(bs)

    def solve_refined(self, a: Csr, b: np.ndarray, steps: int):
        """Solve, then refine with the residual against `a` (both triangles) while its largest
        magnitude shrinks, at most `steps` times (ldlt.rs:524-560); Cholesky solutions are
        returned as solved. The products are the reference's Csr::mul, on the host."""
        rhs = b.copy()
        self.solve(b)
        if self.is_cholesky():
            return

        def residual(x):
            rows = np.repeat(np.arange(a.n), np.diff(a.ptr))
            ax = np.zeros(a.n)
            np.add.at(ax, rows, a.val * x[a.idx])
            return rhs - ax

        r = residual(b)
        size = float(np.max(np.abs(r))) if a.n else 0.0
        for _ in range(steps):
            if not size > 0.0:
                break
            dx = r.copy()
            self.solve(dx)
            trial = b + dx
            nxt = residual(trial)
            nsize = float(np.max(np.abs(nxt)))
            if not nsize < size:
                break
            b[:] = trial
            r, size = nxt, nsize

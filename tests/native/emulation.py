"""TEST INFRASTRUCTURE: builds and loads the CPU emulation of the device LDL^T panel
(ldlt_emulation.cpp beside this file), which runs the kernel's own source on host threads."""
from __future__ import annotations

import ctypes as C
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
SRC = HERE / "ldlt_emulation.cpp"
HEADER = HERE.parent.parent / "fieldcraft_b200" / "csrc" / "cuda" / "ldlt_panel.cuh"
LIB = HERE / "libldlt_emulation.so"
_lib = None


def build():
    if LIB.exists() and LIB.stat().st_mtime >= max(SRC.stat().st_mtime, HEADER.stat().st_mtime):
        return
    subprocess.run(["g++", "-O2", "-std=c++17", "-fPIC", "-shared", "-pthread", "-ffp-contract=off", "-fno-fast-math",
                    "-Wall", "-Wextra", f"-I{HEADER.parent.parent}", "-o", str(LIB), str(SRC)], check=True)


def load():
    global _lib
    if _lib is None:
        build()
        _lib = C.CDLL(str(LIB))
        _lib.emu_ldlt_front.restype = C.c_int
        _lib.emu_ldlt_front.argtypes = [C.c_int64, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int,
                                        C.c_int, C.c_void_p]
        _lib.emu_ldlt_after.restype = C.c_int
        _lib.emu_ldlt_after.argtypes = [C.c_int64, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                        C.c_int]
        _lib.emu_apply_d_inverse.restype = None
        _lib.emu_apply_d_inverse.argtypes = [C.c_int64, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
        _lib.emu_unit_lower_inverse.restype = C.c_int
        _lib.emu_unit_lower_inverse.argtypes = [C.c_void_p, C.c_int64, C.c_int, C.c_void_p, C.c_int64, C.c_int]
        _lib.emu_permute_rows_below.restype = C.c_int
        _lib.emu_permute_rows_below.argtypes = [C.c_int64, C.c_int, C.c_void_p, C.c_void_p, C.c_int]
        _lib.emu_update_tiles.restype = C.c_int64
        _lib.emu_update_tiles.argtypes = [C.c_int64, C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                          C.c_void_p, C.c_int64]
    return _lib


def factor_front(front: np.ndarray, w: int, scale: np.ndarray, threads: int, jitter: int = 0):
    """Factors an m x w front (rows >= columns meaningful) with the panel source on `threads`
    host threads. Returns (result, F, pivots, order, 2 x 2 count): result -1, or the own column
    found singular; -2 / -3 when the threads disagreed."""
    m = front.shape[0]
    F = np.asfortranarray(front[:, :w], dtype=np.float64).copy(order="F")
    scale = np.ascontiguousarray(scale, np.float64)
    order = np.zeros(w, np.int32)
    pivots = np.zeros(w, np.int8)
    twos = C.c_int(0)
    rc = load().emu_ldlt_front(m, w, F.ctypes.data, scale.ctypes.data, order.ctypes.data, pivots.ctypes.data,
                               threads, jitter, C.byref(twos))
    return rc, F, pivots, order, twos.value


def packed(F: np.ndarray, w: int) -> np.ndarray:
    """The front's lower trapezoid by columns (the reference's layout)."""
    return np.concatenate([F[c:, c] for c in range(w)]) if w else np.zeros(0)


def update_tiles(m: int, w: int, c1: int):
    """The update tiles after a panel that ended at c1: a list of (i0, j0, M, N, lower)."""
    lib = load()
    count = lib.emu_update_tiles(m, w, c1, None, None, None, None, None, 0)
    assert count >= 0, "update_tiles disagrees with update_tile"
    i0, j0 = np.zeros(count, np.int64), np.zeros(count, np.int32)
    M, N, low = np.zeros(count, np.int32), np.zeros(count, np.int32), np.zeros(count, np.int8)
    lib.emu_update_tiles(m, w, c1, i0.ctypes.data, j0.ctypes.data, M.ctypes.data, N.ctypes.data, low.ctypes.data,
                         count)
    return list(zip(i0.tolist(), j0.tolist(), M.tolist(), N.tolist(), low.astype(bool).tolist()))


def after_factor(F: np.ndarray, w: int, pivots: np.ndarray, threads: int):
    """W21 = L21 D and D split out of a factored front (F changed in place to unit lower).
    Returns (W21 [(m - w) x w], d, e)."""
    m = F.shape[0]
    w21 = np.zeros((max(m - w, 1), w), order="F")
    d, e = np.zeros(w), np.zeros(w)
    piv = np.ascontiguousarray(pivots, np.int8)
    rc = load().emu_ldlt_after(m, w, F.ctypes.data, piv.ctypes.data, w21.ctypes.data, d.ctypes.data, e.ctypes.data,
                               threads)
    assert rc == 0
    return w21[:m - w], d, e


def apply_d_inverse(d, e, pivots, y):
    """y [n, R] (C order) <- D^-1 y."""
    y = np.ascontiguousarray(y, np.float64)
    load().emu_apply_d_inverse(y.shape[0], y.shape[1], np.ascontiguousarray(d).ctypes.data,
                               np.ascontiguousarray(e).ctypes.data, np.ascontiguousarray(pivots, np.int8).ctypes.data,
                               y.ctypes.data)
    return y


def unit_lower_inverse(Lb: np.ndarray, threads: int) -> np.ndarray:
    """X = Lb^-1 for a unit lower block (its diagonal not read), zero above the diagonal."""
    nb = Lb.shape[0]
    L = np.asfortranarray(Lb, np.float64)
    X = np.zeros((nb, nb), order="F")
    assert load().emu_unit_lower_inverse(L.ctypes.data, nb, nb, X.ctypes.data, nb, threads) == 0
    return X


def permute_rows_below(F: np.ndarray, w: int, frm: np.ndarray, threads: int) -> np.ndarray:
    G = np.asfortranarray(F, np.float64).copy(order="F")
    frm = np.ascontiguousarray(frm, np.int32)
    assert load().emu_permute_rows_below(G.shape[0], w, G.ctypes.data, frm.ctypes.data, threads) == 0
    return G

"""ctypes binding of ``libfieldcraft_b200.so`` (the C ABI of include/fieldcraft_chol.h and
include/fieldcraft_fem.h). The library is built in the source tree; a missing library is an error,
never a silent fallback."""
from __future__ import annotations

import ctypes as C
from pathlib import Path

_PKG = Path(__file__).resolve().parent
LIB_PATH = _PKG / "libfieldcraft_b200.so"

i32, i64, u64, f64 = C.c_int32, C.c_int64, C.c_uint64, C.c_double
P = C.c_void_p
pi32, pi64, pf64 = C.POINTER(i32), C.POINTER(i64), C.POINTER(f64)


class Status(C.Structure):
    _fields_ = [("code", i32), ("reserved", i32), ("column", i64), ("entries", i64), ("limit", i64),
                ("message", C.c_char * 224)]


class SymbolicArrays(C.Structure):
    _fields_ = [(k, i64) for k in ("n", "ns", "entries", "nnz", "rows_len", "lower_len", "updates_len",
                                   "tasks_len", "top_len")] + [
        ("perm", pi64), ("first", pi64), ("rptr", pi64), ("rows", pi32), ("upper_ptr", pi64), ("upper_idx", pi32),
        ("lptr", pi64), ("lidx", pi32), ("slot", pi64), ("crow", pi32), ("ccol", pi32), ("uptr", pi64),
        ("uk", pi64), ("up1", pi64), ("up2", pi64), ("task_lo", pi64), ("task_hi", pi64), ("top", pi64)]


# name -> (restype, argtypes); every symbol include/*.h declares.
SIGNATURES = {
    # fieldcraft_chol.h
    "fc_symbolic_analyse": (i32, [i64, P, P, u64, C.POINTER(P), C.POINTER(Status)]),
    "fc_symbolic_free": (None, [P]),
    "fc_symbolic_get": (i32, [P, C.POINTER(SymbolicArrays)]),
    "fc_symbolic_import": (i32, [C.POINTER(SymbolicArrays), C.POINTER(P), C.POINTER(Status)]),
    "fc_chol_create": (i32, [P, i32, i32, C.POINTER(P), C.POINTER(Status)]),
    "fc_chol_destroy": (None, [P]),
    "fc_chol_set_stream": (i32, [P, P]),
    "fc_chol_factor": (i32, [P, P, i64, P, C.POINTER(Status)]),
    "fc_chol_factor_device": (i32, [P, P, i64, C.POINTER(Status)]),
    "fc_chol_factor_device_async": (i32, [P, P, i64]),
    "fc_chol_check": (i32, [P, C.POINTER(Status)]),
    "fc_chol_ldlt_pivots": (i32, [P, P, P, C.POINTER(Status)]),
    "fc_chol_batch_analyse": (i32, [i32, P, P, P, u64, C.POINTER(P), P, C.POINTER(Status)]),
    "fc_chol_batch_locate": (i32, [i32, P, i64, C.POINTER(i32), C.POINTER(i64)]),
    "fc_chol_entries": (i64, [P]),
    "fc_chol_solve": (i32, [P, P, i32, i64, C.POINTER(Status)]),
    "fc_chol_solve_device": (i32, [P, P, i32, i64, C.POINTER(Status)]),
    "fc_chol_solve_device_async": (i32, [P, P, i32, i64]),
    "fc_chol_solve_device_noalloc": (i32, [P, P, i32, i64, C.POINTER(Status)]),
    "fc_chol_values": (i32, [P, P, C.POINTER(Status)]),
    "fc_chol_inertia": (i32, [P, P, P, P, C.POINTER(Status)]),
    "fc_chol_stat": (i64, [P, i32]),
    "fc_chol_refine_solve_device": (i32, [P, P, P, P, P, P, i32, i64, f64, i32, P, P, C.POINTER(Status)]),
    "fc_chol_option": (i32, [P, i32, i64]),
    "fc_chol_trace_read": (i64, [P, P, i64]),
    "fc_chol_profile": (i32, [P, i32]),
    "fc_chol_profile_read": (i32, [P, P, P, i32]),
    "fc_chol_profile_launches": (i64, [P, P, P, P, P, i64]),
    "fc_csr_spmv_device": (i32, [i64, P, P, P, P, P, i32, i64, P]),
    "fc_version": (C.c_char_p, []),
    # fieldcraft_fem.h
    "fc_fem_box": (i32, [i32, i32, i32, f64, f64, f64, P, f64, P, i32, C.POINTER(P)]),
    "fc_fem_free": (None, [P]),
    "fc_fem_n": (i64, [P]),
    "fc_fem_nnz": (i64, [P]),
    "fc_fem_nodes": (i64, [P]),
    "fc_fem_csr": (i32, [P, P, P, P]),
    "fc_fem_order": (i32, [P, P]),
    "fc_fem_equations": (i32, [P, P]),
    "fc_nested_dissection": (i32, [i64, P, P, P, P]),
    "fc_graph_dissection": (i32, [i64, P, P, P]),
    "fc_fill_reducing_order": (i32, [i64, P, P, P, P]),
    "fc_fill": (i64, [i64, P, P, P]),
    "fc_hex8_stiffness": (i32, [P, f64, f64, P]),
    "fc_fem_device_create": (i32, [i32, i32, i32, f64, f64, f64, i64, P, P, P, i32, C.POINTER(P)]),
    "fc_fem_assemble_device": (i32, [P, P, f64, P, P]),
    "fc_fem_reactions_device": (i32, [P, P, P, P, P, P]),
    "fc_fem_stresses_device": (i32, [P, P, f64, P, P, P, P, P]),
    "fc_fem_device_free": (None, [P]),
    # fieldcraft_unet.h
    "fc_unet_create": (i32, [i32, i32, i32, i64, P, P, f64, u64, i32, C.POINTER(P), C.POINTER(Status)]),
    "fc_unet_destroy": (None, [P]),
    "fc_unet_set_stream": (i32, [P, P]),
    "fc_unet_param_count": (i64, [P]),
    "fc_unet_get_params": (i32, [P, P]),
    "fc_unet_set_params": (i32, [P, P]),
    "fc_unet_get_grads": (i32, [P, P]),
    "fc_unet_forward_grid": (i32, [P, P, P]),
    "fc_unet_backward_grid": (i32, [P, P]),
    "fc_unet_apply": (i32, [P, P, P]),
    "fc_unet_train_step": (i32, [P, P, P, P, P, P, C.c_float, i32, P]),
    "fc_unet_create_levels": (i32, [i32, i32, i32, i64, P, P, f64, i32, u64, i32, C.POINTER(P), C.POINTER(Status)]),
    "fc_unet_set_operator": (i32, [P, P, P, P]),
    "fc_unet_stat": (i64, [P, i32]),
    "fc_unet_enable": (i32, [P, i32]),
    "fc_unet_set_odd": (i32, [P, i32]),
    "fc_unet_train_batch": (i32, [P, P, P, i32, i64, P, P, P, C.c_float, i32, P]),
    "fc_fcg_solve": (i32, [P, P, i64, P, P, P, P, P, f64, i32, i32, C.POINTER(i32), C.POINTER(f64), C.POINTER(i32),
                           C.POINTER(Status)]),
}

_lib = None


def load() -> C.CDLL:
    """The library, loaded once; raises if it has not been built."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise RuntimeError(
                f"{LIB_PATH} is missing: build it with `python -m fieldcraft_b200.build` "
                "(the CUDA path has no fallback)")
        lib = C.CDLL(str(LIB_PATH))
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _lib = lib
    return _lib


def ptr(a) -> int | None:
    """Address of a numpy array's data, or of a torch tensor's."""
    if a is None:
        return None
    if hasattr(a, "data_ptr"):
        return a.data_ptr()
    return a.ctypes.data

"""Chooses a handle's execution variants by timing them on the system itself: the kernels' tile
shapes for the mixed-precision factor's update products (tcgen05 128 x 128 or mma.sync 64 x 64)
and for the solve's products with few right-hand sides (64 x 8 / 64 x 16 or 64 x 64, and the
short launches' copy ring of 8 or 3 stages), the solve's schedule (level by level, or one
persistent dependency-driven launch per direction), how the level-by-level solve splits the K of
its short products (8-CTA clusters or chunks) and,
for a factor used as a preconditioner, conjugate gradients or plain refinement. Each
candidate is run (factorisation + solve to the tolerance, device-timed with CUDA events) and the
fastest is kept in the handle; results can be cached in a JSON file keyed by the system's shape.
No reference counterpart (the reference has one CPU code path)."""
from __future__ import annotations

import ctypes as C
import itertools
import json
from pathlib import Path

from . import _lib
from .cholesky import FP32_IR, Factor


def candidates(precision: int, nrhs: int = 64) -> list[dict]:
    # the solve: level by level with its short products' K split over 8-CTA clusters or in chunks
    # of separate CTAs, or the persistent dependency-driven launch (where the split does not apply);
    # with at most 16 right-hand sides also the products' tile shape (64 x 8 / 64 x 16 or 64 x 64)
    # and, for the narrow tiles, the copy ring of the short launches (8 stages or 3)
    base = {Factor.SOLVE_NARROW: 1, Factor.SOLVE_DEEP: 1}
    solves = [{Factor.SOLVE_SCHEDULE: 0, Factor.SOLVE_CLUSTER: 0, **base},
              {Factor.SOLVE_SCHEDULE: 0, Factor.SOLVE_CLUSTER: 1, **base},
              {Factor.SOLVE_SCHEDULE: 1, Factor.SOLVE_CLUSTER: 0, **base}]
    if nrhs <= 16:
        solves += [{Factor.SOLVE_SCHEDULE: 0, Factor.SOLVE_CLUSTER: 0, Factor.SOLVE_NARROW: 1, Factor.SOLVE_DEEP: 0},
                   {Factor.SOLVE_SCHEDULE: 0, Factor.SOLVE_CLUSTER: 0, Factor.SOLVE_NARROW: 0, Factor.SOLVE_DEEP: 0}]
    if precision == FP32_IR:
        return [{Factor.FP32_UPDATES: u, **sv, Factor.REFINEMENT: r}
                for u, sv, r in itertools.product([0, 1], solves, [0, 1])]
    return [dict(sv) for sv in solves]


def signature(factor: Factor, precision: int, nrhs: int) -> str:
    return f"n{factor.n}-e{factor.entries()}-s{factor.stat(4)}-p{precision}-r{nrhs}"


def autotune(factor: Factor, precision: int, d_val, nnz: int, csr_device, d_b, nrhs: int, tol: float, torch,
             repeats: int = 2, cache: str | Path | None = None, stream=None) -> dict:
    """Times every candidate on this system and applies the fastest. d_val: the matrix's upper
    values on the device; csr_device = (ptr, idx, val) of its rows; d_b the right-hand sides
    (column-major n x nrhs). Returns {"options": {name: value}, "ms": {candidate: ms}}."""
    lib = _lib.load()
    key = signature(factor, precision, nrhs)
    if cache is not None and Path(cache).exists():
        known = json.loads(Path(cache).read_text())
        if key in known:
            for k, v in known[key]["options"].items():
                factor.option(int(k), int(v))
            return known[key]
    stream = stream or torch.cuda.current_stream()
    x = torch.zeros_like(d_b)
    timings = {}
    best, best_ms = None, float("inf")
    for cand in candidates(precision, nrhs):
        for k, v in cand.items():
            factor.option(k, v)
        runs = []
        for it in range(1 + repeats):
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            with torch.cuda.stream(stream):
                if lib.fc_chol_factor_device_async(factor.handle, C.c_void_p(d_val.data_ptr()), nnz) != 0:
                    raise RuntimeError("factorisation launch")
            factor.refine_solve_device(csr_device, d_b, x, nrhs, factor.n, tol=tol, max_iter=40)
            e1.record(stream)
            e1.synchronize()
            if it > 0:
                runs.append(e0.elapsed_time(e1))
        ms = sum(runs) / len(runs)
        timings[json.dumps({str(k): v for k, v in cand.items()})] = ms
        if ms < best_ms:
            best, best_ms = cand, ms
    for k, v in best.items():
        factor.option(k, v)
    result = {"options": {str(k): v for k, v in best.items()}, "ms": timings}
    if cache is not None:
        path = Path(cache)
        known = json.loads(path.read_text()) if path.exists() else {}
        known[key] = result
        path.write_text(json.dumps(known, indent=1))
    return result

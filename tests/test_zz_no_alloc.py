"""The allocation-free solve, fc_chol_solve_device_noalloc, against the ordinary device solve,
fc_chol_solve_device, through the C ABI.

Some callers cannot call cudaMalloc: an application whose own allocator owns the device's memory
under a fixed budget, where one more allocation could fail or fragment its pool. For them the
library solves from one fixed scratch array it reserves on each device. These checks: the same
answer as the ordinary solve, within the parity tests' solve tolerance, on two calls in a row
(the scratch keeps the previous call's contents), on two different factors one after the other,
and a clear refusal of a solve that does not fit the scratch. The file is collected last so a run
that stops at the first failure has run every other test first; it needs nothing from them."""
import ctypes as C

import numpy as np
import pytest

from fieldcraft_b200 import FP32_IR, FP64, Factor, Symbolic, _lib, problems
from fieldcraft_b200._lib import Status

pytestmark = pytest.mark.gpu

SOLVE_TOL = 1e-10  # relative, as the other parity tests
FC_INVALID_ARGUMENT = 8


def column_major(torch, rhs):
    """An n x k right-hand-side block as a contiguous column-major device buffer."""
    return torch.from_numpy(np.ascontiguousarray(rhs.T)).cuda()


def ordinary(lib, f, b, nrhs, n):
    out = b.clone()
    st = Status()
    assert lib.fc_chol_solve_device(f.handle, C.c_void_p(out.data_ptr()), nrhs, n, C.byref(st)) == 0, st.message
    return out


def no_alloc(lib, f, b, nrhs, n):
    out = b.clone()
    st = Status()
    rc = lib.fc_chol_solve_device_noalloc(f.handle, C.c_void_p(out.data_ptr()), nrhs, n, C.byref(st))
    assert rc == 0, st.message.decode()
    return out


def test_no_alloc_solve_matches_the_ordinary_solve(cuda):
    torch = cuda
    lib = _lib.load()
    block = problems.lognormal_block(8, nrhs=4)
    beam = problems.cantilever()
    fb = Factor.new(block.upper(), 2**62)
    fc = Factor.new(beam.upper(), 2**62)
    b1 = column_major(torch, block.rhs)
    b2 = column_major(torch, beam.rhs)
    ref1 = ordinary(lib, fb, b1, 4, block.n)
    ref2 = ordinary(lib, fc, b2, 1, beam.n)
    for _ in range(2):  # two calls in a row on the same factor
        x = no_alloc(lib, fb, b1, 4, block.n)
        assert ((x - ref1).norm() / ref1.norm()).item() <= SOLVE_TOL
    # another factor with another shape next, then the first again: the scratch's leftovers from
    # the previous call do not leak into the answer
    x = no_alloc(lib, fc, b2, 1, beam.n)
    assert ((x - ref2).norm() / ref2.norm()).item() <= SOLVE_TOL
    x = no_alloc(lib, fb, b1, 4, block.n)
    assert ((x - ref1).norm() / ref1.norm()).item() <= SOLVE_TOL
    fb.close()
    fc.close()


@pytest.mark.parametrize("precision", [FP64, FP32_IR], ids=["fp64", "fp32_ir"])
def test_no_alloc_solve_with_split_products(cuda, precision):
    """The 16^3 block: its top separator (867 columns) makes the solve split long products in
    chunks that the last CTA adds (partials and counters in the scratch), and its thin
    supernodes with more than 128 rows below sum their backward steps in chunks the same way.
    With the FP64 factor and with the mixed-precision one (a 4-byte L); two calls in a row."""
    torch = cuda
    lib = _lib.load()
    p = problems.lognormal_block(16, nrhs=5)
    up = p.upper()
    f = Factor(Symbolic(up, 2**62), precision=precision)
    f.factor(up.val)
    b = column_major(torch, p.rhs)
    ref = ordinary(lib, f, b, 5, p.n)
    for _ in range(2):
        x = no_alloc(lib, f, b, 5, p.n)
        assert ((x - ref).norm() / ref.norm()).item() <= SOLVE_TOL
    assert f.stat(8) > 0  # the launches of the last solve are counted
    f.close()


def test_no_alloc_solve_refuses_more_than_its_scratch(cuda):
    torch = cuda
    lib = _lib.load()
    beam = problems.cantilever()
    f = Factor.new(beam.upper(), 2**62)
    nrhs = 800  # two n x 800 vectors alone take 38.4 MB, more than the 32 MiB scratch
    b = torch.zeros((nrhs, beam.n), dtype=torch.float64, device="cuda")
    st = Status()
    rc = lib.fc_chol_solve_device_noalloc(f.handle, C.c_void_p(b.data_ptr()), nrhs, beam.n, C.byref(st))
    assert rc == FC_INVALID_ARGUMENT and st.code == FC_INVALID_ARGUMENT
    assert b"scratch" in st.message and b"limit" in st.message
    f.close()

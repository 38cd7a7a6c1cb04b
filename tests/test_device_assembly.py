"""K_ff assembled entry by entry (fieldcraft_b200/csrc/host/assembly.hpp, the device assembly's
code): each entry the sum over the elements holding both its nodes, in element label order, of
their stiffness entries (host/hex8.hpp, shared with the builder). On the host it must give the
builder's K (crates/solver/src/analysis.rs:199-234 restated in csrc/host/fem.cpp) bit for bit."""
import ctypes as C

import numpy as np
import pytest

from fieldcraft_b200 import _lib, problems


def host_assemble(nx, ny, nz, lx, ly, lz, p, young, poisson=0.3):
    lib = _lib.load()
    fn = lib.fc_test_fem_assemble_host
    fn.restype = C.c_int
    young = np.ascontiguousarray(np.broadcast_to(np.asarray(young, np.float64), (nx * ny * nz,)))
    val = np.empty(p.csr.val.size)
    keep = [np.ascontiguousarray(a) for a in (p.csr.ptr, p.csr.idx, p.eq)]
    rc = fn(nx, ny, nz, C.c_double(lx), C.c_double(ly), C.c_double(lz), C.c_int64(p.n),
            *(C.c_void_p(a.ctypes.data) for a in keep), C.c_void_p(young.ctypes.data), C.c_double(poisson),
            C.c_void_p(val.ctypes.data))
    assert rc == 0
    return val


@pytest.mark.parametrize("case", ["cantilever", "lognormal", "plate"])
def test_entry_by_entry_assembly_is_the_builders(case):
    if case == "cantilever":
        p = problems.cantilever()
        dims, lengths, young = (40, 4, 4), (100.0, 10.0, 10.0), 210e3
    elif case == "lognormal":
        p = problems.lognormal_block(10, nrhs=1, seed=3)
        dims, lengths, young = (10, 10, 10), (10.0, 10.0, 10.0), p.young
    else:
        p = problems.plate(12, 10, 3, nrhs=1)
        dims, lengths, young = (12, 10, 3), (12.0, 10.0, 3.0), p.young
    assert p.lengths == lengths
    got = host_assemble(*dims, *lengths, p, young)
    assert np.array_equal(got.view(np.uint64), p.csr.val.view(np.uint64))


@pytest.mark.gpu
@pytest.mark.skip(reason="the device assembly has not run on a GPU yet")
def test_device_assembly_is_the_builders(cuda):
    """fc_fem_assemble_device: K_ff on the GPU from element moduli in device memory, the
    builder's values bit for bit."""
    torch = cuda
    p = problems.lognormal_block(12, nrhs=1, seed=4)
    d = problems.DeviceAssembly(p)
    young = torch.from_numpy(p.young).cuda()
    val = torch.empty(p.csr.val.size, dtype=torch.float64, device="cuda")
    d.assemble(young, val)
    assert np.array_equal(val.cpu().numpy().view(np.uint64), p.csr.val.view(np.uint64))
    young[5] = -1.0
    with pytest.raises(ValueError):
        d.assemble(young, val)
    d.close()


def host_reactions(nx, ny, nz, lx, ly, lz, p, young, q, f_full, poisson=0.3):
    lib = _lib.load()
    fn = lib.fc_test_fem_reactions_host
    fn.restype = C.c_int
    young = np.ascontiguousarray(np.broadcast_to(np.asarray(young, np.float64), (nx * ny * nz,)))
    r = np.empty(p.eq.size)
    keep = [np.ascontiguousarray(a, np.float64) if a.dtype.kind == "f" else np.ascontiguousarray(a)
            for a in (p.eq, young, q, f_full)]
    rc = fn(nx, ny, nz, C.c_double(lx), C.c_double(ly), C.c_double(lz), C.c_void_p(keep[0].ctypes.data),
            C.c_void_p(keep[1].ctypes.data), C.c_double(poisson), C.c_void_p(keep[2].ctypes.data),
            C.c_void_p(keep[3].ctypes.data), C.c_void_p(r.ctypes.data))
    assert rc == 0
    return r


def test_reactions_balance_the_loads():
    """The reactions at the clamped face (constraints.rs:1001-1015, a plain clamp) for the
    oracle's solution of the cantilever (1 kN total, -z): they balance the applied load in every
    direction, and the free DOFs carry none."""
    from oracle import oracle
    p = problems.cantilever()
    up = p.upper()
    s = oracle.Sym(up.n, up.ptr, up.idx)
    q = oracle.Fac(s, up.val).solve(p.rhs[:, 0].copy())
    r = host_reactions(40, 4, 4, 100.0, 10.0, 10.0, p, 210e3, q, np.zeros(p.eq.size))
    held = p.eq < 0
    assert np.all(r[~held] == 0.0) and np.any(r[held] != 0.0)
    dofs = np.flatnonzero(held)
    total = np.array([r[dofs[dofs % 3 == a]].sum() for a in range(3)])
    applied = np.array([0.0, 0.0, -1000.0])
    assert np.max(np.abs(total + applied)) <= 1e-8 * 1000.0, total


@pytest.mark.gpu
@pytest.mark.skip(reason="the device reactions have not run on a GPU yet")
def test_device_reactions_are_the_hosts(cuda):
    """fc_fem_reactions_device: the motion of every DOF and the reactions at the held ones, as the
    host code gives them for the same solution, bit for bit."""
    from oracle import oracle
    torch = cuda
    p = problems.cantilever()
    up = p.upper()
    q = oracle.Fac(oracle.Sym(up.n, up.ptr, up.idx), up.val).solve(p.rhs[:, 0].copy())
    d = problems.DeviceAssembly(p)
    young = torch.full((40 * 4 * 4,), 210e3, dtype=torch.float64, device="cuda")
    val = torch.empty(p.csr.val.size, dtype=torch.float64, device="cuda")
    d.assemble(young, val)
    r = torch.empty(p.eq.size, dtype=torch.float64, device="cuda")
    u = torch.empty_like(r)
    d.reactions(torch.from_numpy(q).cuda(), r=r, u=u)
    want = host_reactions(40, 4, 4, 100.0, 10.0, 10.0, p, 210e3, q, np.zeros(p.eq.size))
    assert np.array_equal(r.cpu().numpy().view(np.uint64), want.view(np.uint64))
    expected_u = np.where(p.eq >= 0, q[np.maximum(p.eq, 0)], 0.0)
    assert np.array_equal(u.cpu().numpy(), expected_u)
    d.close()

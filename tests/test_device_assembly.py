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


def host_stresses(nx, ny, nz, lx, ly, lz, young, u, poisson=0.3):
    lib = _lib.load()
    fn = lib.fc_test_fem_stresses_host
    fn.restype = C.c_int
    elements, nodes = nx * ny * nz, (nx + 1) * (ny + 1) * (nz + 1)
    young = np.ascontiguousarray(np.broadcast_to(np.asarray(young, np.float64), (elements,)))
    u = np.ascontiguousarray(u, np.float64)
    points, nodal, vm = np.empty(elements * 48), np.empty(nodes * 6), np.empty(nodes)
    rc = fn(nx, ny, nz, C.c_double(lx), C.c_double(ly), C.c_double(lz), C.c_void_p(young.ctypes.data),
            C.c_double(poisson), C.c_void_p(u.ctypes.data), C.c_void_p(points.ctypes.data),
            C.c_void_p(nodal.ctypes.data), C.c_void_p(vm.ctypes.data))
    assert rc == 0
    return points.reshape(elements, 8, 6), nodal.reshape(nodes, 6), vm


def test_a_linear_field_gives_its_constant_stress():
    """The patch test (crates/fem/src/tests.rs:153, extrapolation of linear fields): a linear
    displacement u = G x on a box of unequal elements gives sigma = D eps(G) at every Gauss point,
    at every corner after extrapolation and at every node after the mean, and its von Mises stress."""
    nx, ny, nz, lx, ly, lz, E, nu = 3, 2, 4, 3.0, 1.5, 2.0, 70e3, 0.33
    G = np.array([[1e-3, 2e-4, -3e-4], [5e-4, -2e-3, 1e-4], [-1e-4, 3e-4, 4e-4]])
    i, j, k = problems.node_grid(nx, ny, nz)
    xyz = np.stack([lx * i / nx, ly * j / ny, lz * k / nz], axis=1)
    u = (xyz @ G.T).reshape(-1)
    points, nodal, vm = host_stresses(nx, ny, nz, lx, ly, lz, E, u, nu)
    eps = np.array([G[0, 0], G[1, 1], G[2, 2], G[0, 1] + G[1, 0], G[0, 2] + G[2, 0], G[1, 2] + G[2, 1]])
    lam, mu = E * nu / ((1 + nu) * (1 - 2 * nu)), E / (2 * (1 + nu))
    D = np.zeros((6, 6))
    D[:3, :3] = lam
    D[np.arange(3), np.arange(3)] = lam + 2 * mu
    D[np.arange(3, 6), np.arange(3, 6)] = mu
    sigma = D @ eps
    scale = np.max(np.abs(sigma))
    assert np.max(np.abs(points - sigma)) <= 1e-10 * scale
    assert np.max(np.abs(nodal - sigma)) <= 1e-10 * scale
    s = sigma
    want_vm = np.sqrt(0.5 * ((s[0] - s[1]) ** 2 + (s[1] - s[2]) ** 2 + (s[2] - s[0]) ** 2) + 3 * (s[3:] ** 2).sum())
    assert np.max(np.abs(vm - want_vm)) <= 1e-10 * want_vm


@pytest.mark.gpu
def test_device_stresses_are_the_hosts(cuda):
    """fc_fem_stresses_device: Gauss-point stresses, nodal means and von Mises as the host code gives
    them for the same motion, bit for bit."""
    torch = cuda
    nx, ny, nz = 5, 3, 2
    p = problems.box(nx, ny, nz, 5.0, 3.0, 2.0, 210e3, 0.3, problems.node_grid(nx, ny, nz)[0] == 0)
    rng = np.random.default_rng(3)
    u = rng.standard_normal(p.eq.size) * 1e-3
    d = problems.DeviceAssembly(p)
    young = torch.full((nx * ny * nz,), 210e3, dtype=torch.float64, device="cuda")
    points = torch.empty(nx * ny * nz * 48, dtype=torch.float64, device="cuda")
    nodal = torch.empty(p.eq.size * 2, dtype=torch.float64, device="cuda")
    vm = torch.empty(p.eq.size // 3, dtype=torch.float64, device="cuda")
    d.stresses(young, torch.from_numpy(u).cuda(), points, nodal, vm)
    hp, hn, hv = host_stresses(nx, ny, nz, 5.0, 3.0, 2.0, 210e3, u)
    for got, want in [(points, hp), (nodal, hn), (vm, hv)]:
        assert np.array_equal(got.cpu().numpy().view(np.uint64), want.reshape(-1).view(np.uint64))
    d.close()

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

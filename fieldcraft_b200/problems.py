"""The stiffness systems K u = f the path is measured on: structured boxes of hex8 elements with
full 2x2x2 integration, held on one face (or the sides), in the reference's fill-reducing order
and equation numbering, assembled by the native builder (include/fieldcraft_fem.h).

Seeded synthetic inputs: the reference publishes no matrices for these workloads, so each is
generated here with the shapes, sizes and value distributions the workload names.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field

import numpy as np

from . import _lib
from .cholesky import Csr, UpperColumns


@dataclass
class Problem:
    name: str
    dims: tuple
    csr: Csr
    order: np.ndarray       # node elimination order
    eq: np.ndarray          # equation of each mesh DOF (3 per node), -1 when held
    nodes_xyz: np.ndarray   # [nodes, 3]
    rhs: np.ndarray = field(default=None)  # [n, nrhs], Fortran order
    young: np.ndarray = field(default=None)  # element moduli (when the workload keeps them)
    lengths: tuple = field(default=None)     # the box's lx, ly, lz

    @property
    def n(self) -> int:
        return self.csr.n

    def upper(self) -> UpperColumns:
        return UpperColumns.from_symmetric(self.csr)


def box(nx, ny, nz, lx, ly, lz, young, poisson, clamped_nodes, name="box", threads=0) -> Problem:
    """K_ff of an nx x ny x nz box of hex8 elements; `young` per element (e = i + nx (j + ny k))
    or one value; `clamped_nodes` a boolean mask over the nodes v = i + (nx+1) (j + (ny+1) k)."""
    lib = _lib.load()
    ne = nx * ny * nz
    young = np.ascontiguousarray(np.broadcast_to(np.asarray(young, np.float64), (ne,)), np.float64)
    clamped = np.ascontiguousarray(clamped_nodes, np.uint8)
    h = C.c_void_p()
    rc = lib.fc_fem_box(nx, ny, nz, lx, ly, lz, _lib.ptr(young), float(poisson), _lib.ptr(clamped), int(threads),
                        C.byref(h))
    if rc != 0:
        raise ValueError(f"fc_fem_box failed ({rc})")
    try:
        n, nnz, nodes = lib.fc_fem_n(h), lib.fc_fem_nnz(h), lib.fc_fem_nodes(h)
        ptr = np.empty(n + 1, np.int64)
        idx = np.empty(nnz, np.int32)
        val = np.empty(nnz, np.float64)
        order = np.empty(nodes, np.int64)
        eq = np.empty(3 * nodes, np.int64)
        lib.fc_fem_csr(h, _lib.ptr(ptr), _lib.ptr(idx), _lib.ptr(val))
        lib.fc_fem_order(h, _lib.ptr(order))
        lib.fc_fem_equations(h, _lib.ptr(eq))
    finally:
        lib.fc_fem_free(h)
    i, j, k = np.meshgrid(np.arange(nx + 1), np.arange(ny + 1), np.arange(nz + 1), indexing="ij")
    xyz = np.stack([lx * i / nx, ly * j / ny, lz * k / nz], axis=-1).transpose(2, 1, 0, 3).reshape(-1, 3)
    return Problem(name, (nx, ny, nz), Csr(int(n), ptr, idx, val), order, eq, xyz,
                   lengths=(float(lx), float(ly), float(lz)))


class DeviceAssembly:
    """K_ff of a box problem assembled on the GPU (fc_fem_device_*): the builder's values bit for
    bit, from element moduli in device memory."""

    def __init__(self, p: Problem, device: int = 0):
        lib = _lib.load()
        nx, ny, nz = p.dims
        lx, ly, lz = p.lengths
        self._keep = [np.ascontiguousarray(a) for a in (p.csr.ptr, p.csr.idx, p.eq)]
        h = C.c_void_p()
        rc = lib.fc_fem_device_create(nx, ny, nz, lx, ly, lz, p.n, *(_lib.ptr(a) for a in self._keep), device,
                                      C.byref(h))
        if rc != 0:
            raise ValueError(f"fc_fem_device_create failed ({rc})")
        self.handle = h

    def assemble(self, young, val, poisson: float = 0.3, stream_ptr: int | None = None):
        """val (a CUDA tensor of nnz doubles) <- K_ff's values for the moduli `young` (a CUDA tensor)."""
        rc = _lib.load().fc_fem_assemble_device(self.handle, C.c_void_p(young.data_ptr()), float(poisson),
                                                C.c_void_p(val.data_ptr()), C.c_void_p(stream_ptr or 0))
        if rc != 0:
            raise ValueError(f"fc_fem_assemble_device failed ({rc})")

    def reactions(self, q, r=None, u=None, f=None, stream_ptr: int | None = None):
        """After assemble(): from the free solution q (a CUDA tensor of n doubles), the motion of every
        DOF into u and the reactions at the held DOFs into r (CUDA tensors of 3 nodes doubles, either
        may be None), with the loads f over every DOF (None: none)."""
        p = lambda t: C.c_void_p(t.data_ptr()) if t is not None else None  # noqa: E731
        rc = _lib.load().fc_fem_reactions_device(self.handle, p(q), p(f), p(r), p(u), C.c_void_p(stream_ptr or 0))
        if rc != 0:
            raise ValueError(f"fc_fem_reactions_device failed ({rc})")

    def stresses(self, young, u, points=None, nodal=None, von_mises=None, poisson: float = 0.3,
                 stream_ptr: int | None = None):
        """Stress recovery from the motion of every DOF u (a CUDA tensor of 3 nodes doubles): the
        Gauss-point stresses (elements x 48), the nodal means (nodes x 6), the von Mises stress
        (nodes); CUDA tensors or None."""
        p = lambda t: C.c_void_p(t.data_ptr()) if t is not None else None  # noqa: E731
        rc = _lib.load().fc_fem_stresses_device(self.handle, p(young), float(poisson), p(u), p(points), p(nodal),
                                                p(von_mises), C.c_void_p(stream_ptr or 0))
        if rc != 0:
            raise ValueError(f"fc_fem_stresses_device failed ({rc})")

    def close(self):
        if getattr(self, "handle", None):
            _lib.load().fc_fem_device_free(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except TypeError:
            pass


def node_grid(nx, ny, nz):
    """(i, j, k) of every node in node order."""
    k, j, i = np.meshgrid(np.arange(nz + 1), np.arange(ny + 1), np.arange(nx + 1), indexing="ij")
    return i.ravel(), j.ravel(), k.ravel()


def nodal_load(p: Problem, nodes: np.ndarray, vectors: np.ndarray) -> np.ndarray:
    """A right-hand side with `vectors[q]` (3 components) at node nodes[q]; held DOFs dropped."""
    f = np.zeros(p.n)
    for a in range(3):
        e = p.eq[3 * nodes + a]
        ok = e >= 0
        np.add.at(f, e[ok], vectors[ok, a])
    return f


def cantilever() -> Problem:
    """Plain FP64 linear-elastic hex8 cantilever: 100 x 10 x 10 mm, 40 x 4 x 4 elements,
    E = 210 GPa (210000 MPa), nu = 0.3, x = 0 face clamped, 1 kN total -z on the x = 100 face
    split evenly over its nodes: 3000 free DOFs, one right-hand side."""
    nx, ny, nz = 40, 4, 4
    i, j, k = node_grid(nx, ny, nz)
    p = box(nx, ny, nz, 100.0, 10.0, 10.0, 210000.0, 0.3, i == 0, name="cantilever-40x4x4")
    end = np.nonzero(i == nx)[0]
    vec = np.zeros((end.size, 3))
    vec[:, 2] = -1000.0 / end.size
    p.rhs = np.asfortranarray(nodal_load(p, end, vec)[:, None])
    return p


def lognormal_block(n_el: int = 48, nrhs: int = 64, seed: int = 2024, sigma: float = 0.5) -> Problem:
    """Plain FP64 on GPU at scale: a block of n_el^3 unit hex8 elements, per-element E lognormal
    (median 210 GPa, sigma 0.5, iid, seeded), nu = 0.3, z = 0 face clamped; `nrhs` right-hand
    sides, each a seeded Gaussian nodal force on every top-face node."""
    rng = np.random.default_rng(seed)
    young = 210000.0 * np.exp(sigma * rng.standard_normal(n_el ** 3))
    i, j, k = node_grid(n_el, n_el, n_el)
    p = box(n_el, n_el, n_el, float(n_el), float(n_el), float(n_el), young, 0.3, k == 0,
            name=f"lognormal-block-{n_el}^3")
    p.young = young
    top = np.nonzero(k == n_el)[0]
    rhs = np.empty((p.n, nrhs), order="F")
    for r in range(nrhs):
        rhs[:, r] = nodal_load(p, top, rng.standard_normal((top.size, 3)))
    p.rhs = rhs
    return p


def gaussian_field(shape, corr: float, seed: int) -> np.ndarray:
    """A unit-variance Gaussian random field on a grid: white noise smoothed by a separable
    Gaussian kernel of standard deviation `corr` cells, then standardised."""
    rng = np.random.default_rng(seed)
    g = rng.standard_normal(shape)
    radius = int(np.ceil(3 * corr))
    x = np.arange(-radius, radius + 1)
    ker = np.exp(-0.5 * (x / corr) ** 2)
    ker /= ker.sum()
    for ax in range(g.ndim):
        g = np.apply_along_axis(lambda v: np.convolve(np.pad(v, radius, mode="wrap"), ker, mode="valid"), ax, g)
    return (g - g.mean()) / g.std()


def field_block(n_el: int = 64, nrhs: int = 16, corr: float = 6.0, contrast: float = 1e3, seed: int = 7) -> Problem:
    """Mixed precision on an ill-conditioned system: n_el^3 unit hex8 elements, E from a seeded
    lognormal Gaussian random field (correlation `corr` elements) scaled so that E at +-3 sigma
    spans `contrast`, nu = 0.3, z = 0 face clamped, `nrhs` Gaussian top-face loads."""
    g = gaussian_field((n_el, n_el, n_el), corr, seed)  # axes (k, j, i)
    s = np.log(contrast) / 6.0
    young = 210000.0 * np.exp(s * g).reshape(-1)
    i, j, k = node_grid(n_el, n_el, n_el)
    p = box(n_el, n_el, n_el, float(n_el), float(n_el), float(n_el), young, 0.3, k == 0,
            name=f"field-block-{n_el}^3")
    p.young = young
    rng = np.random.default_rng(seed + 1)
    top = np.nonzero(k == n_el)[0]
    rhs = np.empty((p.n, nrhs), order="F")
    for r in range(nrhs):
        rhs[:, r] = nodal_load(p, top, rng.standard_normal((top.size, 3)))
    p.rhs = rhs
    return p


def uneven_boxes(count: int = 256, lo: int = 4, hi: int = 24, nrhs: int = 8, seed: int = 11):
    """Batched uneven solves: `count` independent boxes with element counts drawn from [lo, hi]
    per axis, E uniform in [70, 210] GPa, nu uniform in [0.25, 0.35], z = 0 face clamped, `nrhs`
    random top-face loads each. Yields the problems one by one."""
    rng = np.random.default_rng(seed)
    for b in range(count):
        nx, ny, nz = (int(v) for v in rng.integers(lo, hi + 1, size=3))
        young = float(rng.uniform(70000.0, 210000.0))
        nu = float(rng.uniform(0.25, 0.35))
        i, j, k = node_grid(nx, ny, nz)
        p = box(nx, ny, nz, float(nx), float(ny), float(nz), young, nu, k == 0, name=f"box-{b}-{nx}x{ny}x{nz}")
        top = np.nonzero(k == nz)[0]
        rhs = np.empty((p.n, nrhs), order="F")
        for r in range(nrhs):
            rhs[:, r] = nodal_load(p, top, rng.standard_normal((top.size, 3)))
        p.rhs = rhs
        yield p


def plate(nx: int = 128, ny: int = 128, nz: int = 8, corr: float = 8.0, contrast: float = 100.0, seed: int = 5,
          nrhs: int = 1) -> Problem:
    """The learned-preconditioner workload: an nx x ny x nz plate of unit hex8 elements, E from a
    seeded lognormal Gaussian random field (correlation `corr` elements, E at +-3 sigma spanning
    `contrast`), nu = 0.3, the four side faces clamped, `nrhs` random top-face pressures (a
    smooth random field of vertical nodal forces). p.young holds the element moduli."""
    g = gaussian_field((nz, ny, nx), corr, seed)
    young = 210000.0 * np.exp(np.log(contrast) / 6.0 * g).reshape(-1)
    i, j, k = node_grid(nx, ny, nz)
    clamped = (i == 0) | (i == nx) | (j == 0) | (j == ny)
    p = box(nx, ny, nz, float(nx), float(ny), float(nz), young, 0.3, clamped, name=f"plate-{nx}x{ny}x{nz}")
    p.young = young
    p.rhs = top_pressures(p, nrhs, seed + 1)
    return p


def top_pressures(p: Problem, count: int, seed: int) -> np.ndarray:
    """`count` random top-face pressure loads: vertical nodal forces from a smooth random field
    (correlation 8 nodes) over the top nodes, each column scaled to unit norm."""
    nx, ny, nz = p.dims
    i, j, k = node_grid(nx, ny, nz)
    top = np.nonzero(k == nz)[0]
    rng = np.random.default_rng(seed)
    out = np.empty((p.n, count), order="F")
    for c in range(count):
        field = gaussian_field((ny + 1, nx + 1), 8.0, int(rng.integers(1 << 31))).reshape(-1)
        vec = np.zeros((top.size, 3))
        vec[:, 2] = -(1.0 + 0.5 * field)
        f = nodal_load(p, top, vec)
        out[:, c] = f / np.linalg.norm(f)
    return out


def node_feature(p: Problem) -> np.ndarray:
    """Per node: the mean log Young's modulus of the elements around it, standardised (the
    learned preconditioner's fixed input channel)."""
    nx, ny, nz = p.dims
    le = np.log(np.broadcast_to(np.asarray(p.young, np.float64), (nx * ny * nz,))).reshape(nz, ny, nx)
    acc = np.zeros((nz + 1, ny + 1, nx + 1))
    cnt = np.zeros_like(acc)
    for dz in (0, 1):
        for dy in (0, 1):
            for dx in (0, 1):
                acc[dz:dz + nz, dy:dy + ny, dx:dx + nx] += le
                cnt[dz:dz + nz, dy:dy + ny, dx:dx + nx] += 1
    f = acc / cnt
    sd = f.std()
    return ((f - f.mean()) / (sd if sd > 0 else 1.0)).reshape(-1).astype(np.float32)

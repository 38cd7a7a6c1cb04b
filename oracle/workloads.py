"""ORACLE (test infrastructure): the benchmark workloads built by the oracle alone, for the timed
CPU reference and the checks. K_ff comes from the oracle's own hex8 builder (fem_oracle.cpp,
restating the reference's node graph, fill-reducing order, element stiffness and assembly); the
seeded material fields and loads follow the workload definitions (per-element lognormal E, a
lognormal Gaussian random field, Gaussian top-face nodal forces). Nothing here imports the
product, so the CPU reference runs without the product's library."""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from . import oracle


@dataclass
class Workload:
    name: str
    dims: tuple
    n: int
    ptr: np.ndarray    # K_ff by rows (both triangles, columns sorted)
    idx: np.ndarray
    val: np.ndarray
    order: np.ndarray  # node elimination order
    eq: np.ndarray     # equation of each mesh DOF, -1 when held
    rhs: np.ndarray = None  # [n, nrhs], Fortran order
    young: np.ndarray = None

    def upper(self):
        """The upper triangle by columns (cholesky.rs:112-145): (ptr, idx, val)."""
        return oracle.upper_from_symmetric(self.n, self.ptr, self.idx, self.val)


def node_grid(nx, ny, nz):
    k, j, i = np.meshgrid(np.arange(nz + 1), np.arange(ny + 1), np.arange(nx + 1), indexing="ij")
    return i.ravel(), j.ravel(), k.ravel()


def box(nx, ny, nz, lx, ly, lz, young, nu, clamped, name="box") -> Workload:
    n, ptr, idx, val, order, eq = oracle.fem_box(nx, ny, nz, lx, ly, lz, young, nu, clamped)
    return Workload(name, (nx, ny, nz), n, ptr, idx, val, order, eq)


def nodal_load(w: Workload, nodes, vectors) -> np.ndarray:
    f = np.zeros(w.n)
    for a in range(3):
        e = w.eq[3 * nodes + a]
        ok = e >= 0
        np.add.at(f, e[ok], vectors[ok, a])
    return f


def cantilever() -> Workload:
    """40 x 4 x 4 hex8 on 100 x 10 x 10 mm, E 210 GPa, nu 0.3, x = 0 clamped, 1 kN -z over the
    x = 100 face's nodes (3000 free DOFs, one right-hand side)."""
    i, j, k = node_grid(40, 4, 4)
    w = box(40, 4, 4, 100.0, 10.0, 10.0, 210000.0, 0.3, i == 0, "cantilever-40x4x4")
    end = np.nonzero(i == 40)[0]
    vec = np.zeros((end.size, 3))
    vec[:, 2] = -1000.0 / end.size
    w.rhs = np.asfortranarray(nodal_load(w, end, vec)[:, None])
    return w


def lognormal_block(n_el: int = 48, nrhs: int = 64, seed: int = 2024, sigma: float = 0.5) -> Workload:
    """n_el^3 unit hex8 elements, E = 210 GPa exp(sigma xi_e) (xi iid N(0,1), seeded), nu 0.3,
    z = 0 clamped, `nrhs` seeded Gaussian nodal forces on the top-face nodes."""
    rng = np.random.default_rng(seed)
    young = 210000.0 * np.exp(sigma * rng.standard_normal(n_el ** 3))
    i, j, k = node_grid(n_el, n_el, n_el)
    w = box(n_el, n_el, n_el, float(n_el), float(n_el), float(n_el), young, 0.3, k == 0, f"lognormal-block-{n_el}^3")
    w.young = young
    top = np.nonzero(k == n_el)[0]
    rhs = np.empty((w.n, nrhs), order="F")
    for r in range(nrhs):
        rhs[:, r] = nodal_load(w, top, rng.standard_normal((top.size, 3)))
    w.rhs = rhs
    return w


def gaussian_field(shape, corr: float, seed: int) -> np.ndarray:
    """Unit-variance Gaussian random field: seeded white noise smoothed by a separable Gaussian
    kernel of standard deviation `corr` cells (periodic), then standardised."""
    rng = np.random.default_rng(seed)
    g = rng.standard_normal(shape)
    radius = int(np.ceil(3 * corr))
    x = np.arange(-radius, radius + 1)
    ker = np.exp(-0.5 * (x / corr) ** 2)
    ker /= ker.sum()
    for ax in range(g.ndim):
        g = np.apply_along_axis(lambda v: np.convolve(np.pad(v, radius, mode="wrap"), ker, mode="valid"), ax, g)
    return (g - g.mean()) / g.std()


def field_block(n_el: int = 64, nrhs: int = 16, corr: float = 6.0, contrast: float = 1e3, seed: int = 7) -> Workload:
    """n_el^3 unit hex8, E from a lognormal Gaussian random field (correlation `corr` elements,
    E at +-3 sigma spanning `contrast`), nu 0.3, z = 0 clamped, Gaussian top-face loads."""
    g = gaussian_field((n_el, n_el, n_el), corr, seed)
    young = 210000.0 * np.exp(np.log(contrast) / 6.0 * g).reshape(-1)
    i, j, k = node_grid(n_el, n_el, n_el)
    w = box(n_el, n_el, n_el, float(n_el), float(n_el), float(n_el), young, 0.3, k == 0, f"field-block-{n_el}^3")
    w.young = young
    rng = np.random.default_rng(seed + 1)
    top = np.nonzero(k == n_el)[0]
    rhs = np.empty((w.n, nrhs), order="F")
    for r in range(nrhs):
        rhs[:, r] = nodal_load(w, top, rng.standard_normal((top.size, 3)))
    w.rhs = rhs
    return w


def uneven_boxes(count: int = 256, lo: int = 4, hi: int = 24, nrhs: int = 8, seed: int = 11):
    """`count` boxes with nx, ny, nz ~ U{lo..hi}, E ~ U[70, 210] GPa, nu ~ U[0.25, 0.35], z = 0
    clamped, `nrhs` Gaussian top-face loads each (seeded); yields them one by one."""
    rng = np.random.default_rng(seed)
    for b in range(count):
        nx, ny, nz = (int(v) for v in rng.integers(lo, hi + 1, size=3))
        young = float(rng.uniform(70000.0, 210000.0))
        nu = float(rng.uniform(0.25, 0.35))
        i, j, k = node_grid(nx, ny, nz)
        w = box(nx, ny, nz, float(nx), float(ny), float(nz), young, nu, k == 0, f"box-{b}-{nx}x{ny}x{nz}")
        top = np.nonzero(k == nz)[0]
        rhs = np.empty((w.n, nrhs), order="F")
        for r in range(nrhs):
            rhs[:, r] = nodal_load(w, top, rng.standard_normal((top.size, 3)))
        w.rhs = rhs
        yield w


def stacked(parts) -> Workload:
    """diag(A_0, A_1, ...) of independent systems as one workload (rows and loads end to end)."""
    ptr, idx, val, rhs = [np.zeros(1, np.int64)], [], [], []
    c0 = z0 = 0
    for w in parts:
        ptr.append(w.ptr[1:] + z0)
        idx.append(w.idx.astype(np.int64) + c0)
        val.append(w.val)
        rhs.append(w.rhs)
        c0 += w.n
        z0 += int(w.ptr[-1])
    out = Workload("stacked", (), c0, np.concatenate(ptr), np.concatenate(idx).astype(np.int32), np.concatenate(val),
                   np.zeros(0, np.int64), np.zeros(0, np.int64))
    out.rhs = np.asfortranarray(np.concatenate(rhs, axis=0))
    return out


def plate(nx: int = 128, ny: int = 128, nz: int = 8, corr: float = 8.0, contrast: float = 100.0, seed: int = 5,
          nrhs: int = 1) -> Workload:
    """nx x ny x nz unit hex8 plate, E from a lognormal Gaussian random field (correlation `corr`,
    contrast `contrast`), nu 0.3, the four side faces clamped, random top-face pressures."""
    g = gaussian_field((nz, ny, nx), corr, seed)
    young = 210000.0 * np.exp(np.log(contrast) / 6.0 * g).reshape(-1)
    i, j, k = node_grid(nx, ny, nz)
    clamped = (i == 0) | (i == nx) | (j == 0) | (j == ny)
    w = box(nx, ny, nz, float(nx), float(ny), float(nz), young, 0.3, clamped, f"plate-{nx}x{ny}x{nz}")
    w.young = young
    w.rhs = top_pressures(w, nrhs, seed + 1)
    return w


def top_pressures(w: Workload, count: int, seed: int) -> np.ndarray:
    """`count` random top-face pressures: vertical nodal forces 1 + 0.5 g from a smooth random
    field g (correlation 8 nodes) over the top nodes, each column scaled to unit norm."""
    nx, ny, nz = w.dims
    i, j, k = node_grid(nx, ny, nz)
    top = np.nonzero(k == nz)[0]
    rng = np.random.default_rng(seed)
    out = np.empty((w.n, count), order="F")
    for c in range(count):
        field = gaussian_field((ny + 1, nx + 1), 8.0, int(rng.integers(1 << 31))).reshape(-1)
        vec = np.zeros((top.size, 3))
        vec[:, 2] = -(1.0 + 0.5 * field)
        f = nodal_load(w, top, vec)
        out[:, c] = f / np.linalg.norm(f)
    return out

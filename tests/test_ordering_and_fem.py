"""The input side of the path (include/fieldcraft_fem.h) against the reference's own tests:
the orderings (crates/solver/src/ordering.rs:284-400) and the hex8 model."""
import numpy as np
import pytest

from fieldcraft_b200 import _lib, problems
from oracle import oracle


def adjacency_csr(adj):
    ptr = np.zeros(len(adj) + 1, np.int64)
    ptr[1:] = np.cumsum([len(r) for r in adj])
    idx = np.array([c for r in adj for c in r], np.int32)
    return ptr, idx


def nd(xyz, adj):
    lib = _lib.load()
    ptr, idx = adjacency_csr(adj)
    xyz = np.ascontiguousarray(xyz, np.float64)
    out = np.zeros(len(adj), np.int64)
    assert lib.fc_nested_dissection(len(adj), _lib.ptr(xyz), _lib.ptr(ptr), _lib.ptr(idx), _lib.ptr(out)) == 0
    return out


def gd(adj):
    lib = _lib.load()
    ptr, idx = adjacency_csr(adj)
    out = np.zeros(len(adj), np.int64)
    assert lib.fc_graph_dissection(len(adj), _lib.ptr(ptr), _lib.ptr(idx), _lib.ptr(out)) == 0
    return out


def fro(xyz, adj):
    lib = _lib.load()
    ptr, idx = adjacency_csr(adj)
    xyz = np.ascontiguousarray(xyz, np.float64)
    out = np.zeros(len(adj), np.int64)
    assert lib.fc_fill_reducing_order(len(adj), _lib.ptr(xyz), _lib.ptr(ptr), _lib.ptr(idx), _lib.ptr(out)) == 0
    return out


def fill(adj, order):
    ptr, idx = adjacency_csr(adj)
    order = np.ascontiguousarray(order, np.int64)
    return int(_lib.load().fc_fill(len(adj), _lib.ptr(ptr), _lib.ptr(idx), _lib.ptr(order)))


def hex_grid(dims, wrap, at):
    """ordering.rs:316-348: the node graph of a structured hex8 grid (27-point stencil)."""
    ni = dims[0] if wrap else dims[0] + 1
    nj, nk = dims[1] + 1, dims[2] + 1
    ident = lambda i, j, k: (i % ni) + ni * (j + nj * k)
    xyz = np.zeros((ni * nj * nk, 3))
    adj = [[] for _ in range(ni * nj * nk)]
    for k in range(nk):
        for j in range(nj):
            for i in range(ni):
                xyz[ident(i, j, k)] = at(i, j, k)
                for t in range(27):
                    di, dj, dk = t % 3, (t // 3) % 3, t // 9
                    a, b, c = i + ni + di - 1, j + dj, k + dk
                    if wrap:
                        a = a % ni
                    elif a < ni or a >= 2 * ni:
                        continue
                    else:
                        a = a - ni
                    if 1 <= b <= nj and 1 <= c <= nk:
                        adj[ident(i, j, k)].append(ident(a, b - 1, c - 1))
    adj = [sorted(set(r)) for r in adj]
    return xyz, adj


def cylinder_wall():
    def at(i, j, k):
        t = i / 160.0 * 2 * np.pi
        r = 50.0 + j * 0.5
        return [r * np.cos(t), r * np.sin(t), k * 2.0]
    return hex_grid([160, 2, 40], True, at)


def test_a_permutation_with_separators_last():
    # ordering.rs:287-311
    m = 12
    ident = lambda i, j: i * m + j
    xyz = np.array([[v // m, v % m, 0.0] for v in range(m * m)], np.float64)
    adj = [[] for _ in range(m * m)]
    for i in range(m):
        for j in range(m):
            for di, dj in [(0, 1), (1, 0), (0, -1), (-1, 0), (0, 0)]:
                a, b = i + di, j + dj
                if 0 <= a < m and 0 <= b < m:
                    adj[ident(i, j)].append(ident(a, b))
    adj = [sorted(r) for r in adj]
    order = nd(xyz, adj)
    assert sorted(order.tolist()) == list(range(m * m))
    last = order[m * m - m:]
    assert np.all(last // m == last[0] // m) or np.all(last % m == last[0] % m), last
    assert np.array_equal(order, nd(xyz, adj))


def test_graph_dissection_is_a_deterministic_permutation():
    # ordering.rs:360-373
    _, adj = cylinder_wall()
    order = gd(adj)
    assert sorted(order.tolist()) == list(range(len(adj)))
    assert np.array_equal(order, gd(adj))
    _, two = hex_grid([6, 6, 6], False, lambda i, j, k: [i, j, k])
    m = len(two)
    two = two + [[v + m for v in r] for r in two] + [[]]
    assert sorted(gd(two).tolist()) == list(range(2 * m + 1))
    assert gd([]).size == 0


def test_the_graph_cuts_a_thin_curved_wall_with_less_fill():
    # ordering.rs:375-382
    xyz, adj = cylinder_wall()
    planes = fill(adj, nd(xyz, adj))
    graph = fill(adj, gd(adj))
    assert graph < planes, (graph, planes)
    assert fill(adj, fro(xyz, adj)) == graph


def test_a_block_keeps_the_better_ordering():
    # ordering.rs:384-390
    xyz, adj = hex_grid([16, 16, 16], False, lambda i, j, k: [i, j, k])
    planes = fill(adj, nd(xyz, adj))
    assert fill(adj, fro(xyz, adj)) <= planes


def test_fill_is_the_oracles_factor_entries():
    # fill (ordering.rs:257-281) is the entry count of the node graph's factor (cholesky.rs:215-218)
    xyz, adj = hex_grid([5, 4, 3], False, lambda i, j, k: [i, j, k])
    order = fro(xyz, adj)
    pos = np.empty(len(adj), np.int64)
    pos[order] = np.arange(len(adj))
    cols = [sorted({int(pos[w]) for w in adj[v] if pos[w] <= k} | {k}) for k, v in enumerate(order)]
    ptr = np.zeros(len(adj) + 1, np.int64)
    ptr[1:] = np.cumsum([len(c) for c in cols])
    idx = np.array([r for c in cols for r in c], np.int32)
    s = oracle.Sym(len(adj), ptr, idx)
    assert fill(adj, order) == s.info("entries")


def hex8_unit_stiffness(young=1000.0, nu=0.3, scale=(1.0, 1.0, 1.0)):
    corners = np.array([[0, 0, 0], [1, 0, 0], [1, 1, 0], [0, 1, 0], [0, 0, 1], [1, 0, 1], [1, 1, 1], [0, 1, 1]],
                       np.float64) * np.array(scale)
    out = np.zeros(576)
    assert _lib.load().fc_hex8_stiffness(_lib.ptr(np.ascontiguousarray(corners.ravel())), young, nu, _lib.ptr(out)) == 0
    return out.reshape(24, 24), corners


def test_hex8_stiffness_is_symmetric_with_rigid_body_modes():
    k, x = hex8_unit_stiffness(scale=(2.0, 1.0, 0.5))
    assert np.array_equal(k, k.T)  # mirrored, exactly symmetric (element.rs:745-774)
    w = np.linalg.eigvalsh(k)
    assert np.sum(np.abs(w) < 1e-9 * w.max()) == 6 and w.min() > -1e-9 * w.max()
    # translations and rotations produce no force
    for mode in range(6):
        u = np.zeros((8, 3))
        if mode < 3:
            u[:, mode] = 1.0
        else:
            axis = np.zeros(3)
            axis[mode - 3] = 1.0
            u = np.cross(axis, x)
        assert np.max(np.abs(k @ u.ravel())) < 1e-10 * np.abs(k).max()


def test_cantilever_workload_shape():
    p = problems.cantilever()
    assert p.n == 3000 and p.rhs.shape == (3000, 1)
    assert abs(p.rhs.sum() + 1000.0) < 1e-9
    k = problems.box(3, 2, 2, 3.0, 2.0, 2.0, 100.0, 0.25, problems.node_grid(3, 2, 2)[0] == 0).csr
    dense = np.zeros((k.n, k.n))
    for r in range(k.n):
        dense[r, k.idx[k.ptr[r]:k.ptr[r + 1]]] = k.val[k.ptr[r]:k.ptr[r + 1]]
    assert np.array_equal(dense, dense.T) and np.linalg.eigvalsh(dense).min() > 0
    assert all(np.all(np.diff(k.idx[k.ptr[r]:k.ptr[r + 1]]) > 0) for r in range(k.n))


@pytest.mark.slow
def test_hex8_cantilever_converges_to_timoshenko():
    # tests/verification.rs:185-245: hex8 (full integration) locks in bending and converges under
    # refinement, error below 4 % at 40 x 8 x 8 against Timoshenko's deflection.
    l, b, h, young, p = 10.0, 1.0, 1.0, 1000.0, 1.0
    exact = p * l ** 3 / (3 * young * b * h ** 3 / 12) + p * l / (5.0 / 6.0 * young / 2.0 * b * h)
    errs = []
    for n in ([5, 1, 1], [10, 2, 2], [20, 4, 4], [40, 8, 8]):
        nx, ny, nz = n
        i, j, k = problems.node_grid(nx, ny, nz)
        pr = problems.box(nx, ny, nz, l, b, h, young, 0.0, i == 0)
        # a uniform shear traction on the end face: each face element's bilinear corners share
        # its force equally (consistent loads of a constant traction on a rectangle)
        f = np.zeros(pr.n)
        area = (b / ny) * (h / nz)
        for jj in range(ny):
            for kk in range(nz):
                for dj in (0, 1):
                    for dk in (0, 1):
                        v = nx + (nx + 1) * ((jj + dj) + (ny + 1) * (kk + dk))
                        f[pr.eq[3 * v + 2]] -= p / (b * h) * area / 4
        ptr, idx, val = oracle.upper_from_symmetric(pr.n, pr.csr.ptr, pr.csr.idx, pr.csr.val)
        s = oracle.Sym(pr.n, ptr, idx)
        u = oracle.Fac(s, val).solve(f.copy())
        end = np.nonzero(i == nx)[0]
        d = -np.mean(u[pr.eq[3 * end + 2]])
        errs.append(abs(d - exact) / exact)
    assert all(b < a for a, b in zip(errs, errs[1:])), errs
    rate = np.log2(errs[-2] / errs[-1])
    assert rate > 1.5 and errs[-1] < 0.04, errs

"""Parity of the B200 numeric phase with the oracle, through the C ABI (via the Python mirror of
the reference's API). Every case runs the CUDA kernels; FP64 throughout.

Tolerances: the GPU computes each entry of L with a different operation order than the reference
(blocked right-looking fronts, fused multiply-adds on the FP64 tensor pipe), so parity is to
rounding: factor entries within 1e-11 of the largest entry, solutions within 1e-10 relative to the
oracle's (the path's stated accuracy bar), and the reference's own residual bounds where it states them."""
import ctypes as C

import numpy as np
import pytest

import helpers as H
from fieldcraft_b200 import (FP32_IR, FP64, Cancelled, Factor, NotPositiveDefinite, Symbolic, TooLarge, UpperColumns,
                              _lib, problems)
from fieldcraft_b200._lib import Status
from fieldcraft_b200.cholesky import Csr
from oracle import oracle

pytestmark = pytest.mark.gpu

FACTOR_TOL = 1e-11
SOLVE_TOL = 1e-10


def oracle_factor(csr: Csr):
    up = UpperColumns.from_symmetric(csr)
    s = oracle.Sym(up.n, up.ptr, up.idx)
    return s, oracle.Fac(s, up.val)


def cases():
    yield "grid7x5", lambda: Csr.from_dense(H.grid_7x5())
    yield "panels", H.panels_matrix
    yield "blocks40", lambda: Csr.from_dense(H.blocks40())
    yield "solid5", lambda: H.solid_stiffness(5)
    yield "solid5-roller", lambda: H.solid_stiffness(5, roller=True)
    yield "band", lambda: H.band_matrix()[1]
    yield "cantilever", lambda: problems.cantilever().csr
    yield "lognormal-12", lambda: problems.lognormal_block(12, nrhs=1).csr


@pytest.mark.parametrize("name,make", list(cases()), ids=[c[0] for c in cases()])
def test_factor_and_solve_match_the_oracle(cuda, name, make):
    csr = make()
    up = UpperColumns.from_symmetric(csr)
    f = Factor.new(up, 2**62)
    _, ref = oracle_factor(csr)
    lv, rv = f.values(), ref.values()
    assert f.entries() == rv.size
    assert np.max(np.abs(lv - rv)) <= FACTOR_TOL * np.max(np.abs(rv)), name
    x = H.sin_solution(csr.n)
    b = oracle.spmv(csr.n, csr.ptr, csr.idx, csr.val, x)
    got = b.copy()
    f.solve(got)
    exp = ref.solve(b.copy())
    assert np.linalg.norm(got - exp) <= SOLVE_TOL * np.linalg.norm(exp), name
    r = oracle.spmv(csr.n, csr.ptr, csr.idx, csr.val, got) - b
    assert np.linalg.norm(r) <= 1e-10 * np.linalg.norm(b), name


def test_reference_residual_bounds(cuda):
    # cholesky.rs:1707 (1e-13) and :1761 (1e-12) on the GPU factor
    for csr, tol in ((Csr.from_dense(H.grid_7x5()), 1e-13), (H.panels_matrix(), 1e-12)):
        f = Factor.new(UpperColumns.from_symmetric(csr), 2**62)
        x = H.sin_solution(csr.n)
        b = oracle.spmv(csr.n, csr.ptr, csr.idx, csr.val, x)
        f.solve(b)
        assert np.max(np.abs(b - x)) < tol


def test_errors_match_the_reference(cuda):
    csr = Csr.from_dense(H.grid_7x5())
    up = UpperColumns.from_symmetric(csr)
    with pytest.raises(TooLarge):
        Factor.new(up, 10)
    sing = UpperColumns.from_symmetric(Csr.from_dense(H.grid_7x5(shift=False)))
    with pytest.raises(NotPositiveDefinite) as e:
        Factor.new(sing, 2**62)
    assert e.value.column == 34
    flag = C.c_int32(1)
    with pytest.raises(Cancelled):
        Factor.new(up, 2**62, cancel=flag)
    empty = UpperColumns(0, np.zeros(1, np.int64), np.zeros(0, np.int32), np.zeros(0))
    f = Factor.new(empty, 10)
    assert f.entries() == 0
    f.solve(np.zeros(0))
    one = UpperColumns.from_symmetric(Csr.from_dense([[4.0]]))
    f = Factor.new(one, 10)
    b = np.array([2.0])
    f.solve(b)
    assert b.tolist() == [0.5]
    with pytest.raises(ValueError):
        f.solve(np.zeros(2))


def test_solve_many_is_each_solve_bit_for_bit(cuda):
    csr = H.panels_matrix()
    f = Factor.new(UpperColumns.from_symmetric(csr), 2**62)
    rhs = [np.sin((np.arange(csr.n) * 7 + s * 13) * 0.11) for s in range(5)]
    alone = []
    for b in rhs:
        x = b.copy()
        f.solve(x)
        alone.append(x)
    together = [b.copy() for b in rhs]
    f.solve_many(together)
    for a, t in zip(alone, together):
        assert np.array_equal(a.view(np.uint64), t.view(np.uint64))


@pytest.mark.parametrize("n_el", [16, 24])
def test_split_solve_does_not_depend_on_how_many_are_solved(cuda, n_el):
    """The 16^3 block's top separator (867 columns) makes the solve split its long GEMMs in chunks
    whose last CTA adds the partials; the 24^3 block's backward products over the rows below its
    second-level separators take more chunks than one CTA adds (groups of chunks, then the groups'
    sums): a right-hand side's solution is still bit for bit the same solved alone, among 5, and
    among 70 (two blocks of 64 right-hand sides)."""
    csr = problems.lognormal_block(n_el, nrhs=1).csr
    f = Factor.new(UpperColumns.from_symmetric(csr), 2**62)
    rng = np.random.default_rng(5)
    rhs = rng.standard_normal((70, csr.n))
    alone = {}
    for j in (0, 3, 69):
        x = rhs[j].copy()
        f.solve(x)
        alone[j] = x
    five = [rhs[j].copy() for j in range(5)]
    f.solve_many(five)
    many = [rhs[j].copy() for j in range(70)]
    f.solve_many(many)
    same = lambda a, b: np.array_equal(a.view(np.uint64), b.view(np.uint64))
    assert same(alone[0], five[0]) and same(alone[3], five[3])
    assert same(alone[0], many[0]) and same(alone[3], many[3]) and same(alone[69], many[69])
    r = oracle.spmv(csr.n, csr.ptr, csr.idx, csr.val, alone[69]) - rhs[69]
    assert np.linalg.norm(r) <= 1e-10 * np.linalg.norm(rhs[69])


@pytest.mark.parametrize("precision", [FP64, FP32_IR], ids=["fp64", "fp32_ir"])
def test_narrow_solve_tiles_give_the_same_bits(cuda, precision):
    """With up to 16 right-hand sides the solve's products run in 64 x 8 / 64 x 16 tiles; with the
    option off in the 64 x 64 tiles. On the 16^3 block (split products, thin chunks), for the FP64
    factor and the FP32 one (a 4-byte L widened in the products), 1, 7 and 16 right-hand sides
    give the same bits both ways, and the same bits as among 70; 70 give the same bits with the
    short launches' deeper copy ring on and off."""
    torch = cuda
    lib = _lib.load()
    p = problems.lognormal_block(16, nrhs=1)
    up = p.upper()
    f = Factor(Symbolic(up, 2**62), precision=precision)
    f.factor(up.val)
    rng = np.random.default_rng(9)
    rhs = torch.from_numpy(rng.standard_normal((70, p.n))).cuda()  # row j: right-hand side j

    def solve(k):
        x = rhs[:k].clone()
        st = Status()
        assert lib.fc_chol_solve_device(f.handle, C.c_void_p(x.data_ptr()), k, p.n, C.byref(st)) == 0, st.message
        return x

    many = solve(70)
    f.option(Factor.SOLVE_DEEP, 0)
    shallow = solve(70)
    f.option(Factor.SOLVE_DEEP, 1)
    assert torch.equal(many, shallow)  # the deeper copy ring of short launches changes no bit
    for k in (1, 7, 16):
        f.option(Factor.SOLVE_NARROW, 1)
        narrow = solve(k)
        f.option(Factor.SOLVE_NARROW, 0)
        wide = solve(k)
        assert torch.equal(narrow, wide) and torch.equal(narrow, many[:k]), k
    f.option(Factor.SOLVE_NARROW, 1)
    f.close()


@pytest.mark.parametrize("precision", [FP64, FP32_IR], ids=["fp64", "fp32_ir"])
def test_programmatic_dependent_launches_give_the_same_bits(cuda, precision):
    """The level-by-level solve's kernels start while their predecessors finish (programmatic
    dependent launches, an option) and wait for them before touching the solve's vectors: on the
    16^3 block, 1, 16 and 70 right-hand sides give the same bits as with ordinary launches, in the
    captured graph (thin launches beside the wide ones on a second stream) and launched directly
    with every launch timed (one stream)."""
    torch = cuda
    lib = _lib.load()
    p = problems.lognormal_block(16, nrhs=1)
    up = p.upper()
    f = Factor(Symbolic(up, 2**62), precision=precision)
    f.factor(up.val)
    rng = np.random.default_rng(11)
    rhs = torch.from_numpy(rng.standard_normal((70, p.n))).cuda()

    def solve(k):
        x = rhs[:k].clone()
        st = Status()
        assert lib.fc_chol_solve_device(f.handle, C.c_void_p(x.data_ptr()), k, p.n, C.byref(st)) == 0, st.message
        return x

    for k in (1, 16, 70):
        f.option(Factor.SOLVE_PDL, 1)
        pdl = solve(k)
        again = solve(k)
        lib.fc_chol_profile(f.handle, 1)
        direct = solve(k)
        lib.fc_chol_profile(f.handle, 0)
        f.option(Factor.SOLVE_PDL, 0)
        plain = solve(k)
        assert torch.equal(pdl, plain) and torch.equal(pdl, again) and torch.equal(pdl, direct), k
    f.close()


@pytest.mark.parametrize("precision", [FP64, FP32_IR], ids=["fp64", "fp32_ir"])
def test_children_first_update_matrices(cuda, precision):
    """The wide supernodes' update matrices take their children's contributions first (beside the
    panels) and the update product subtracts from them (the default), or the product stores and
    the children are added after it: on the 16^3 block both factors agree to rounding (1e-12 of
    the largest entry in FP64, 1e-5 in FP32), the FP64 one matches the oracle, and the factorisation
    stays bit for bit repeatable."""
    p = problems.lognormal_block(16, nrhs=1)
    up = p.upper()
    f = Factor(Symbolic(up, 2**62), precision=precision)
    vals = {}
    for on in (1, 0, 1):
        f.option(Factor.CHILDREN_FIRST, on)
        f.factor(up.val)
        vals.setdefault(on, []).append(f.values())
    assert np.array_equal(vals[1][0], vals[1][1])
    big = np.max(np.abs(vals[0][0]))
    assert np.max(np.abs(vals[1][0] - vals[0][0])) <= (1e-12 if precision == FP64 else 1e-5) * big
    if precision == FP64:
        _, ref = oracle_factor(p.csr)
        rv = ref.values()
        assert np.max(np.abs(vals[1][0] - rv)) <= FACTOR_TOL * np.max(np.abs(rv))
    f.close()


def test_cluster_split_solve(cuda):
    """The 16^3 block's short solve products run with K split over 8-CTA clusters (the default) or
    in chunks of separate CTAs: both match the oracle; the cluster form is bit for bit the same on
    every run and for a right-hand side alone or among 70."""
    p = problems.lognormal_block(16, nrhs=1)
    csr = p.csr
    f = Factor.new(UpperColumns.from_symmetric(csr), 2**62)
    _, ref = oracle_factor(csr)
    rng = np.random.default_rng(8)
    rhs = np.asfortranarray(rng.standard_normal((csr.n, 70)))
    exp = ref.solve(rhs.copy())
    runs = {}
    for cluster in (1, 0, 1):
        f.option(Factor.SOLVE_CLUSTER, cluster)
        x = rhs.copy(order="F")
        f.solve_many(x)
        for j in range(x.shape[1]):
            assert np.linalg.norm(x[:, j] - exp[:, j]) <= SOLVE_TOL * np.linalg.norm(exp[:, j]), (cluster, j)
        runs.setdefault(cluster, []).append(x)
    assert np.array_equal(runs[1][0].view(np.uint64), runs[1][1].view(np.uint64))
    alone = np.ascontiguousarray(rhs[:, 5])
    f.solve(alone)
    assert np.array_equal(alone.view(np.uint64), runs[1][0][:, 5].copy().view(np.uint64))


def test_factorisation_is_deterministic(cuda):
    csr = problems.lognormal_block(10, nrhs=1).csr
    up = UpperColumns.from_symmetric(csr)
    a = Factor.new(up, 2**62).values()
    b = Factor.new(up, 2**62).values()
    assert np.array_equal(a.view(np.uint64), b.view(np.uint64))


def test_device_entry_points(cuda):
    torch = cuda
    p = problems.lognormal_block(8, nrhs=4)
    up = p.upper()
    sym = Symbolic(up, 2**62)
    f = Factor(sym)
    st = __import__("fieldcraft_b200._lib", fromlist=["Status"]).Status()
    from fieldcraft_b200 import _lib
    lib = _lib.load()
    dval = torch.from_numpy(up.val).cuda()
    assert lib.fc_chol_factor_device(f.handle, C.c_void_p(dval.data_ptr()), up.val.size, C.byref(st)) == 0
    b = torch.from_numpy(np.ascontiguousarray(p.rhs.T)).cuda()  # rows are right-hand sides: column-major n x 4
    x = b.clone()
    f.solve_device(x, 4, p.n)
    _, ref = oracle_factor(p.csr)
    exp = ref.solve(p.rhs.copy())
    got = x.cpu().numpy().T
    assert np.linalg.norm(got - exp) <= SOLVE_TOL * np.linalg.norm(exp)
    # y = K x on the device (Csr::mul)
    dptr = torch.from_numpy(p.csr.ptr).cuda()
    didx = torch.from_numpy(p.csr.idx).cuda()
    dv = torch.from_numpy(p.csr.val).cuda()
    y = torch.empty_like(x)
    assert lib.fc_csr_spmv_device(p.n, C.c_void_p(dptr.data_ptr()), C.c_void_p(didx.data_ptr()),
                                  C.c_void_p(dv.data_ptr()), C.c_void_p(x.data_ptr()), C.c_void_p(y.data_ptr()), 4,
                                  p.n, None) == 0
    torch.cuda.synchronize()
    yref = np.stack([oracle.spmv(p.n, p.csr.ptr, p.csr.idx, p.csr.val, got[:, j]) for j in range(4)], axis=1)
    assert np.max(np.abs(y.cpu().numpy().T - yref)) <= 1e-12 * np.max(np.abs(yref))


@pytest.mark.parametrize("n_el", [20])
def test_lognormal_block_residual(cuda, n_el):
    # the benchmark's workload at a size the oracle finishes in seconds: 20^3 elements, 8 RHS
    p = problems.lognormal_block(n_el, nrhs=8)
    f = Factor.new(p.upper(), 2**62)
    x = np.asfortranarray(p.rhs.copy())
    f.solve_many(x)
    _, ref = oracle_factor(p.csr)
    exp = ref.solve(p.rhs.copy())
    for j in range(x.shape[1]):
        assert np.linalg.norm(x[:, j] - exp[:, j]) <= SOLVE_TOL * np.linalg.norm(exp[:, j])
        r = oracle.spmv(p.n, p.csr.ptr, p.csr.idx, p.csr.val, x[:, j]) - p.rhs[:, j]
        assert np.linalg.norm(r) <= 1e-10 * np.linalg.norm(p.rhs[:, j])


def test_batch_of_uneven_systems(cuda):
    # independent boxes of uneven sizes factored and solved together in one handle; each
    # system's solution matches the oracle's, and a singular system is reported as its own
    from fieldcraft_b200.batch import BatchFactor
    boxes = list(problems.uneven_boxes(count=6, lo=2, hi=7, nrhs=3, seed=5))
    parts = [b.upper() for b in boxes]
    bf = BatchFactor(parts, 2**62)
    bf.factor([p.val for p in parts])
    xs = bf.solve([b.rhs for b in boxes])
    for b, x in zip(boxes, xs):
        _, ref = oracle_factor(b.csr)
        exp = ref.solve(b.rhs.copy())
        assert np.linalg.norm(x - exp) <= SOLVE_TOL * np.linalg.norm(exp)
    # a box held nowhere is singular: the batch names the system and its own column, the column
    # a factorisation of that box alone names
    i, j, k = problems.node_grid(3, 2, 2)
    free = problems.box(3, 2, 2, 3.0, 2.0, 2.0, 1000.0, 0.3, np.zeros(i.size, bool))
    alone = None
    try:
        Factor.new(free.upper(), 2**62)
    except NotPositiveDefinite as e:
        alone = e.column
    assert alone is not None
    parts2 = [parts[0], free.upper(), parts[1]]
    bf2 = BatchFactor(parts2, 2**62)
    with pytest.raises(NotPositiveDefinite) as e:
        bf2.factor([p.val for p in parts2])
    assert e.value.system == 1 and e.value.column == alone


def device_csr(torch, csr):
    return (torch.from_numpy(csr.ptr).cuda(), torch.from_numpy(csr.idx).cuda(), torch.from_numpy(csr.val).cuda())


@pytest.mark.parametrize("name,make,values_tol", [("lognormal-12", lambda: problems.lognormal_block(12, nrhs=4), 1e-4),
                                                  ("cantilever", problems.cantilever, None)],
                         ids=["lognormal-12", "cantilever"])
def test_mixed_precision_refines_to_the_fp64_answer(cuda, name, make, values_tol):
    # FP32 factor (3xTF32 updates, FP64 diagonal blocks) of S A S + FP64 refinement: every
    # right-hand side reaches ||b - A x|| <= 1e-10 ||b||, and x agrees with the FP64 direct solve
    # to what the system's conditioning allows (1e-6 relative). On the well-conditioned block the
    # FP32 factor itself is the FP64 one to FP32 precision; on the slender cantilever (condition
    # ~1e9) its trailing pivots are not, which is what the refinement is for.
    from fieldcraft_b200 import FP32_IR
    torch = cuda
    p = make()
    up = p.upper()
    sym = Symbolic(up, 2**62)
    f32 = Factor(sym, precision=FP32_IR)
    f32.factor(up.val)
    k = p.rhs.shape[1]
    b = torch.from_numpy(np.ascontiguousarray(p.rhs.T)).cuda()
    x = torch.zeros_like(b)
    rel, its = f32.refine_solve_device(device_csr(torch, p.csr), b, x, k, p.n, tol=1e-10, max_iter=30)
    assert np.all(rel <= 1e-10) and its <= 30, (rel, its)
    # plain refinement reaches the same answer, in at least as many solves as the CG form
    f32.option(Factor.REFINEMENT, 1)
    xp = torch.zeros_like(b)
    relp, itsp = f32.refine_solve_device(device_csr(torch, p.csr), b, xp, k, p.n, tol=1e-10, max_iter=60)
    f32.option(Factor.REFINEMENT, 0)
    assert np.all(relp <= 1e-10) and itsp >= its, (itsp, its)
    assert torch.linalg.vector_norm(xp - x).item() <= 1e-8 * torch.linalg.vector_norm(x).item()
    _, ref = oracle_factor(p.csr)
    exp = ref.solve(p.rhs.copy())
    got = x.cpu().numpy().T
    assert np.linalg.norm(got - exp) <= 1e-6 * np.linalg.norm(exp)
    if values_tol is not None:
        lv, rv = f32.values(), ref.values()
        assert np.max(np.abs(lv - rv)) <= values_tol * np.max(np.abs(rv))
    # the FP64 factor refines in one or two solves
    f64 = Factor(sym)
    f64.factor(up.val)
    x64 = torch.zeros_like(b)
    rel64, its64 = f64.refine_solve_device(device_csr(torch, p.csr), b, x64, k, p.n, tol=1e-10, max_iter=5)
    assert np.all(rel64 <= 1e-10) and its64 <= 2


@pytest.mark.parametrize("name,make", [("lognormal-12", lambda: problems.lognormal_block(12, nrhs=70)),
                                       ("cantilever", problems.cantilever)], ids=["lognormal-12", "cantilever"])
def test_solve_schedules_agree(cuda, name, make):
    # the persistent dependency-driven solve and the level-by-level launches both match the
    # oracle; the persistent one is bit-for-bit the same on every run (70 right-hand sides: two
    # blocks of columns)
    p = make()
    up = p.upper()
    f = Factor.new(up, 2**62)
    _, ref = oracle_factor(p.csr)
    exp = ref.solve(p.rhs.copy())
    runs = []
    for schedule in (1, 1, 0):
        f.option(Factor.SOLVE_SCHEDULE, schedule)
        x = np.asfortranarray(p.rhs.copy())
        f.solve_many(x)
        runs.append(x)
        for j in range(x.shape[1]):
            assert np.linalg.norm(x[:, j] - exp[:, j]) <= SOLVE_TOL * np.linalg.norm(exp[:, j]), (name, schedule, j)
    assert np.array_equal(runs[0].view(np.uint64), runs[1].view(np.uint64))


def test_solve_wait_limit_reports_timeout(cuda):
    # a dependency that nothing meets ends the persistent solve with Timeout after the wait limit
    # (the CTAs return; no fault), and the handle keeps working afterwards
    from fieldcraft_b200 import Timeout
    csr = H.panels_matrix()
    f = Factor.new(UpperColumns.from_symmetric(csr), 2**62)
    x = H.sin_solution(csr.n)
    b = oracle.spmv(csr.n, csr.ptr, csr.idx, csr.val, x)
    f.option(Factor.SOLVE_SCHEDULE, 1)
    f.option(Factor.WAIT_LIMIT_NS, 50_000_000)
    f.option(Factor.PLANT_UNMET_WAIT, 1)
    with pytest.raises(Timeout):
        f.solve(b.copy())
    got = b.copy()
    f.solve(got)
    assert np.max(np.abs(got - x)) < 1e-12


def test_autotuner_picks_a_working_variant(cuda, tmp_path):
    # every candidate (update kernel x solve schedule x refinement) solves the batch to the
    # tolerance; the autotuner keeps the fastest and a second call reads it from the cache
    from fieldcraft_b200 import FP32_IR
    from fieldcraft_b200.autotune import autotune, candidates
    from fieldcraft_b200.batch import block_diagonal
    torch = cuda
    boxes = list(problems.uneven_boxes(count=5, lo=3, hi=8, nrhs=2, seed=7))
    up = block_diagonal([b.upper() for b in boxes])
    rows = [b.csr for b in boxes]
    ptr = [np.zeros(1, np.int64)]
    idx, val, c0, z0 = [], [], 0, 0
    for c in rows:
        ptr.append(c.ptr[1:] + z0)
        idx.append(c.idx.astype(np.int64) + c0)
        val.append(c.val)
        c0 += c.n
        z0 += int(c.ptr[-1])
    csr = Csr(c0, np.concatenate(ptr), np.concatenate(idx).astype(np.int32), np.concatenate(val))
    rhs = np.concatenate([b.rhs for b in boxes], axis=0)
    f = Factor(Symbolic(up, 2**62), precision=FP32_IR)
    d_val = torch.from_numpy(up.val).cuda()
    d_b = torch.from_numpy(np.ascontiguousarray(rhs.T)).cuda()
    cache = tmp_path / "tune.json"
    res = autotune(f, FP32_IR, d_val, up.val.size, device_csr(torch, csr), d_b, 2, 1e-10, torch, repeats=1, cache=cache)
    assert len(res["ms"]) == len(candidates(FP32_IR, 2)) and cache.exists()
    again = autotune(f, FP32_IR, d_val, up.val.size, device_csr(torch, csr), d_b, 2, 1e-10, torch, cache=cache)
    assert again["options"] == res["options"]
    x = torch.zeros_like(d_b)
    rel, _ = f.refine_solve_device(device_csr(torch, csr), d_b, x, 2, c0, tol=1e-10, max_iter=30)
    assert np.all(rel <= 1e-10)

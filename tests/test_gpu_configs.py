"""Parity with the oracle on the benchmark workloads themselves, at sizes the oracle finishes in
seconds: the FP64 factor and solve of the 24^3 lognormal block, FP32+IR to rel-res 1e-12 on a
24^3 block whose E is the ill-conditioned random field of the 64^3 mixed-precision workload
(correlation 6 elements, contrast 1e3), and a batch of 32 uneven boxes of 4 to 12 elements a
side. Each right-hand side's error is taken against the oracle's FP64 solution, as
cholesky.rs:1686-1738 checks the reference's solve.

Tolerances: the FP64 device factor's entries within 1e-11 of the largest entry and its solutions
within 1e-10 relative to the oracle's (the path's accuracy bar). The FP32+IR answer has residual
<= 1e-12; its distance to the oracle's FP64 answer is then bounded by the condition of K times
that residual plus the oracle's own rounding, so it is checked against the FP64 device solution's
own distance to the oracle on the same system (at most 100 times it, and at most 1e-8)."""
import numpy as np
import pytest

from fieldcraft_b200 import FP32_IR, FP64, Factor, Symbolic, problems
from oracle import oracle

pytestmark = pytest.mark.gpu

FACTOR_TOL = 1e-11
SOLVE_TOL = 1e-10


def oracle_solution(p):
    up = p.upper()
    s = oracle.Sym(up.n, up.ptr, up.idx)
    f = oracle.Fac(s, up.val)
    return f, f.solve(p.rhs.copy())


def per_rhs_error(x, ref):
    return np.linalg.norm(x - ref, axis=0) / np.linalg.norm(ref, axis=0)


def device_csr(torch, csr):
    return tuple(torch.from_numpy(a).cuda() for a in (csr.ptr, csr.idx, csr.val))


def test_fp64_lognormal_block_24(cuda):
    """The headline workload's generator at 24^3 elements (45 000 DOFs, 16 RHS): every entry of L
    and every right-hand side's solution against the oracle."""
    p = problems.lognormal_block(24, nrhs=16)
    f = Factor.new(p.upper(), 2**62)
    ref_f, ref = oracle_solution(p)
    lv, rv = f.values(), ref_f.values()
    assert np.max(np.abs(lv - rv)) <= FACTOR_TOL * np.max(np.abs(rv))
    x = np.asfortranarray(p.rhs.copy())
    f.solve_many(x)
    err = per_rhs_error(x, ref)
    assert np.all(err <= SOLVE_TOL), err
    for j in range(x.shape[1]):
        r = oracle.spmv(p.n, p.csr.ptr, p.csr.idx, p.csr.val, x[:, j]) - p.rhs[:, j]
        assert np.linalg.norm(r) <= 1e-10 * np.linalg.norm(p.rhs[:, j])


def test_fp32_ir_random_field_to_1e12(cuda):
    """The mixed-precision workload's random field (correlation 6, contrast 1e3) on a 24^3 block,
    4 RHS: the FP32 factor plus FP64 refinement reaches rel-res 1e-12 on every right-hand side, and
    its answer is as close to the oracle's as the FP64 device solve's."""
    torch = cuda
    p = problems.field_block(24, nrhs=4)
    up = p.upper()
    sym = Symbolic(up, 2**62)
    _, ref = oracle_solution(p)
    b = torch.from_numpy(np.ascontiguousarray(p.rhs.T)).cuda()
    csr = device_csr(torch, p.csr)
    f64 = Factor(sym, precision=FP64)
    f64.factor(up.val)
    x64 = torch.zeros_like(b)
    rel64, _ = f64.refine_solve_device(csr, b, x64, 4, p.n, tol=1e-12, max_iter=10)
    err64 = per_rhs_error(x64.cpu().numpy().T, ref)
    assert np.all(rel64 <= 1e-12) and np.all(err64 <= SOLVE_TOL), (rel64, err64)
    f32 = Factor(sym, precision=FP32_IR)
    f32.factor(up.val)
    x32 = torch.zeros_like(b)
    rel32, its = f32.refine_solve_device(csr, b, x32, 4, p.n, tol=1e-12, max_iter=40)
    err32 = per_rhs_error(x32.cpu().numpy().T, ref)
    assert np.all(rel32 <= 1e-12), (rel32, its)
    assert np.all(err32 <= np.maximum(100 * err64, 1e-14)) and np.all(err32 <= 1e-8), (err32, err64)
    f32.close()
    f64.close()


@pytest.mark.parametrize("precision", [FP64, FP32_IR], ids=["fp64", "fp32_ir"])
def test_batch_of_32_uneven_boxes(cuda, precision):
    """The batched workload's generator with 32 boxes of 4 to 12 elements a side (8 RHS each),
    factored and solved as one block-diagonal system: every system's every right-hand side
    against the oracle's solution of that system alone."""
    from fieldcraft_b200.batch import BatchFactor
    torch = cuda
    boxes = list(problems.uneven_boxes(count=32, lo=4, hi=12, nrhs=8, seed=11))
    parts = [b.upper() for b in boxes]
    bf = BatchFactor(parts, 2**62, precision=precision)
    bf.factor([q.val for q in parts])
    if precision == FP64:
        xs = bf.solve([b.rhs for b in boxes])
    else:
        xs = bf.refine_solve([b.csr for b in boxes], [b.rhs for b in boxes], tol=1e-10, torch=torch)
    for b, x in zip(boxes, xs):
        _, ref = oracle_solution(b)
        err = per_rhs_error(x, ref)
        assert np.all(err <= (SOLVE_TOL if precision == FP64 else 1e-8)), (b.name, err)
        for j in range(x.shape[1]):
            r = oracle.spmv(b.n, b.csr.ptr, b.csr.idx, b.csr.val, x[:, j]) - b.rhs[:, j]
            assert np.linalg.norm(r) <= 1e-10 * np.linalg.norm(b.rhs[:, j]), b.name
    bf.close()

"""Shift-invert block Lanczos (fieldcraft_b200/lanczos.py) against the reference's own test
(crates/solver/src/eigen.rs:492-560, `lanczos_finds_repeated_and_zero_eigenvalues`): K and M
diagonal, six zero eigenvalues, 1 twice, then 1.5, 2, ...; the modes, their M-orthonormality, a
range, the cap as an error and tiny problems."""
import numpy as np
import pytest

from fieldcraft_b200.lanczos import NotConverged, Operator, Random, Wanted, lanczos


class Diagonal(Operator):
    def __init__(self, k, m, shift):
        self.k, self.m, self.shift = np.asarray(k, float), np.asarray(m, float), shift
        self.n = len(k)

    def mass(self, x):
        return self.m * x

    def solve_many(self, xs):
        return xs / (self.k - self.shift * self.m)[:, None]


def test_random_is_the_references_xorshift():
    """eigen.rs:155-173: state ^= >> 12, ^= << 25, ^= >> 27; v = state * 0x2545F4914F6CDD1D;
    (v >> 11) / 2^52 - 1, every value in [-1, 1) and the sequence seeded."""
    a, b = Random(7), Random(7)
    xs = [a.uniform() for _ in range(1000)]
    assert xs == [b.uniform() for _ in range(1000)]
    assert min(xs) >= -1.0 and max(xs) < 1.0 and abs(np.mean(xs)) < 0.1
    assert Random(0).state == 1


def test_lanczos_finds_repeated_and_zero_eigenvalues():
    n = 200
    lambdas = [0.0 if i < 6 else 1.0 if i < 8 else 1.0 + (i - 7) * 0.5 for i in range(n)]
    m = [1.0 + (i % 7) * 0.1 for i in range(n)]
    k = [l * mm for l, mm in zip(lambdas, m)]
    shift = -1e-3
    op = Diagonal(k, m, shift)
    pairs = lanczos(op, shift, Wanted(10), 6, n, 1e-9)
    assert len(pairs.values) == 10
    want = [0.0] * 6 + [1.0, 1.0, 1.5, 2.0]
    assert all(abs(g - w) < 1e-8 for g, w in zip(pairs.values, want)), pairs.values
    for i, a in enumerate(pairs.vectors):
        for j, b in enumerate(pairs.vectors):
            assert abs(float(a @ op.mass(b)) - (1.0 if i == j else 0.0)) < 1e-8
    ranged = lanczos(op, shift, Wanted(100, 1.2, 3.2), 6, n, 1e-9)
    assert len(ranged.values) == 4 and all(abs(g - w) < 1e-8 for g, w in zip(ranged.values, [1.5, 2.0, 2.5, 3.0]))
    with pytest.raises(NotConverged):
        lanczos(op, shift, Wanted(50), 6, 24, 1e-9)
    small = Diagonal([2.0, 1.0, 3.0], [1.0] * 3, 0.0)
    everything = lanczos(small, 0.0, Wanted(5), 6, 100, 1e-9)
    assert len(everything.values) == 3
    assert abs(everything.values[0] - 1.0) < 1e-12 and abs(everything.values[2] - 3.0) < 1e-12

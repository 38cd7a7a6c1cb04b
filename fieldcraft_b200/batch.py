"""Many independent systems factored and solved together on one GPU.

The systems' matrices are laid end to end as one block-diagonal matrix: its elimination forest is
the union of their trees, so the symbolic analysis finds the same supernodes for each (no
supernode spans two systems) and the device schedule takes every system's supernodes of one level
in the same launches. One factorisation and one solve (each a single captured CUDA graph after
the first call) then serve the whole batch, uneven sizes included.
"""
from __future__ import annotations

import numpy as np

from .cholesky import FP64, Factor, NotPositiveDefinite, Symbolic, UpperColumns


def block_diagonal(parts: list[UpperColumns]) -> UpperColumns:
    """The upper columns of diag(A_0, A_1, ...)."""
    n = sum(p.n for p in parts)
    ptr = [np.zeros(1, np.int64)]
    idx, val = [], []
    col0 = nnz0 = 0
    for p in parts:
        ptr.append(p.ptr[1:].astype(np.int64) + nnz0)
        idx.append(p.idx.astype(np.int64) + col0)
        val.append(p.val)
        col0 += p.n
        nnz0 += int(p.ptr[-1])
    return UpperColumns(n, np.concatenate(ptr), np.concatenate(idx).astype(np.int32),
                        np.concatenate(val).astype(np.float64))


def shard(costs, world: int) -> list[list[int]]:
    """Independent systems over `world` ranks with no collective on the data path: longest first,
    each to the least-loaded rank (ties to the lowest rank), so every rank gets a deterministic
    share of about the same estimated work. Returns each rank's system indices in increasing order."""
    load = [0.0] * world
    share: list[list[int]] = [[] for _ in range(world)]
    for i in sorted(range(len(costs)), key=lambda k: (-float(costs[k]), k)):
        r = min(range(world), key=lambda q: (load[q], q))
        share[r].append(i)
        load[r] += float(costs[i])
    return [sorted(x) for x in share]


def factor_cost(part: UpperColumns) -> float:
    """Estimated factor work of one system: the sum of squared column counts of its analysis."""
    a = Symbolic(part, 2**62).arrays()
    w = np.diff(a["first"])
    m = np.diff(a["rptr"])
    return float(sum(float(np.dot(mm - np.arange(ww, dtype=np.float64), mm - np.arange(ww, dtype=np.float64)))
                     for mm, ww in zip(m, w)))


class BatchFactor:
    """Factors of several SPD systems at once. `offsets[b]` is system b's first unknown in the
    stacked vectors; a failing pivot is reported as (system, column)."""

    def __init__(self, parts: list[UpperColumns], max_entries: int, precision: int = FP64, device: int = 0):
        self.sizes = np.array([p.n for p in parts], np.int64)
        self.offsets = np.concatenate([[0], np.cumsum(self.sizes)]).astype(np.int64)
        self.nnz = np.array([int(p.ptr[-1]) for p in parts], np.int64)
        whole = block_diagonal(parts)
        self.n = whole.n
        self.symbolic = Symbolic(whole, max_entries)
        self.factor_ = Factor(self.symbolic, precision, device)
        self._whole_pattern = whole

    def locate(self, column: int) -> tuple[int, int]:
        """The system and its own column of a column of the stacked matrix."""
        b = int(np.searchsorted(self.offsets, column, side="right") - 1)
        return b, int(column - self.offsets[b])

    def factor(self, values: list[np.ndarray]):
        """New values for every system (each in its UpperColumns order). A failing pivot raises
        NotPositiveDefinite with `.system` and `.column` set to the system's own column."""
        v = np.concatenate([np.asarray(x, np.float64) for x in values])
        try:
            self.factor_.factor(v)
        except NotPositiveDefinite as e:
            b, c = self.locate(e.column)
            err = NotPositiveDefinite(c)
            err.system = b
            raise err from None

    def solve(self, rhs: list[np.ndarray]) -> list[np.ndarray]:
        """Solves every system for its right-hand sides (each an n_b x k array, the same k for
        all), all at once; returns the solutions in the same shapes."""
        k = rhs[0].shape[1] if rhs[0].ndim == 2 else 1
        block = np.zeros((self.n, k), order="F")
        for b, r in enumerate(rhs):
            block[self.offsets[b]:self.offsets[b + 1], :] = r.reshape(self.sizes[b], k)
        self.factor_.solve_many(block)
        return [block[self.offsets[b]:self.offsets[b + 1], :].copy() for b in range(len(rhs))]

    def entries(self) -> int:
        return self.factor_.entries()

    def close(self):
        self.factor_.close()

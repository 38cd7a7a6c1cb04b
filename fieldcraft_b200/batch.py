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
        self._csr_dev = None
        self.sizes = np.array([p.n for p in parts], np.int64)
        self.nnz = np.array([int(p.ptr[-1]) for p in parts], np.int64)
        self.symbolic, self.offsets = Symbolic.batch(parts, max_entries)  # fc_chol_batch_analyse
        self.n = self.symbolic.n
        self.factor_ = Factor(self.symbolic, precision, device)

    def locate(self, column: int) -> tuple[int, int]:
        """The system and its own column of a column of the stacked matrix (fc_chol_batch_locate)."""
        import ctypes as C
        from . import _lib
        b, local = C.c_int32(0), C.c_int64(0)
        rc = _lib.load().fc_chol_batch_locate(len(self.sizes), _lib.ptr(self.offsets), int(column), C.byref(b),
                                              C.byref(local))
        if rc != 0:
            raise ValueError(f"column {column} is outside the batch")
        return int(b.value), int(local.value)

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

    def refine_solve(self, csrs, rhs: list[np.ndarray], tol: float = 1e-10, torch=None, max_iter: int = 40):
        """Iterative refinement in FP64 around the batch's factor (FP32 or FP64) until every system
        reaches ||b_s - A_s x_s|| <= tol ||b_s|| for each of its right-hand sides: each system's
        right-hand sides are scaled to unit norm and the stacked system is refined to
        tol / sqrt(systems), which bounds every system's own residual by tol. `csrs` are the
        systems' rows (Csr); returns the solutions in the shapes of `rhs`."""
        import torch as _torch_default
        torch = torch or _torch_default
        k = rhs[0].shape[1] if rhs[0].ndim == 2 else 1
        self.refine_solve_prepare(csrs, torch)
        block = np.zeros((k, self.n))
        scale = np.ones((len(rhs), k))
        for b, r in enumerate(rhs):
            r = r.reshape(self.sizes[b], k)
            nb = np.linalg.norm(r, axis=0)
            scale[b] = np.where(nb > 0, nb, 1.0)
            block[:, self.offsets[b]:self.offsets[b + 1]] = (r / scale[b]).T
        d_b = torch.from_numpy(block).cuda()
        d_x = torch.zeros_like(d_b)
        self.factor_.refine_solve_device(self._csr_dev, d_b, d_x, k, self.n, tol=tol / np.sqrt(len(rhs)),
                                         max_iter=max_iter)
        x = d_x.cpu().numpy()
        return [(x[:, self.offsets[b]:self.offsets[b + 1]].T * scale[b]).copy() for b in range(len(rhs))]

    def upload(self, values: list[np.ndarray], csrs, rhs: list[np.ndarray], torch=None):
        """Puts the systems' values, rows and right-hand sides (each scaled to unit norm per
        column, as refine_solve does) in device memory for run_device."""
        import torch as _torch_default
        torch = torch or _torch_default
        self.refine_solve_prepare(csrs, torch)
        k = rhs[0].shape[1] if rhs[0].ndim == 2 else 1
        block = np.zeros((k, self.n))
        self._scale = np.ones((len(rhs), k))
        for b, r in enumerate(rhs):
            r = r.reshape(self.sizes[b], k)
            nb = np.linalg.norm(r, axis=0)
            self._scale[b] = np.where(nb > 0, nb, 1.0)
            block[:, self.offsets[b]:self.offsets[b + 1]] = (r / self._scale[b]).T
        self._k = k
        self._d_val = torch.from_numpy(np.concatenate([np.asarray(v, np.float64) for v in values])).cuda()
        self._d_b = torch.from_numpy(block).cuda()
        self._d_x = torch.zeros_like(self._d_b)

    def run_device(self, tol: float = 1e-10, max_iter: int = 40):
        """From the uploaded inputs in device memory: the numeric factorisation and refinement of
        every system to tol (per system and right-hand side). Returns (residuals, solves)."""
        from . import _lib
        import ctypes as C
        rc = _lib.load().fc_chol_factor_device_async(self.factor_.handle, C.c_void_p(self._d_val.data_ptr()),
                                                     int(self._d_val.numel()))
        if rc != 0:
            from .cholesky import DeviceError, Status, raise_for
            st = Status()
            _lib.load().fc_chol_check(self.factor_.handle, C.byref(st))
            raise_for(st)
            raise DeviceError(f"factorisation refused ({rc})")
        self._d_x.zero_()
        return self.factor_.refine_solve_device(self._csr_dev, self._d_b, self._d_x, self._k, self.n,
                                                tol=tol / np.sqrt(len(self.sizes)), max_iter=max_iter)

    def download(self) -> list[np.ndarray]:
        """The systems' solutions of the last run_device (n_b x k each, unscaled)."""
        x = self._d_x.cpu().numpy()
        return [(x[:, self.offsets[b]:self.offsets[b + 1]].T * self._scale[b]).copy() for b in range(len(self.sizes))]

    def refine_solve_prepare(self, csrs, torch):
        if self._csr_dev is None:
            ptr, idx, val = [np.zeros(1, np.int64)], [], []
            z = 0
            for b, c in enumerate(csrs):
                ptr.append(c.ptr[1:].astype(np.int64) + z)
                idx.append(c.idx.astype(np.int64) + self.offsets[b])
                val.append(c.val)
                z += int(c.ptr[-1])
            self._csr_dev = (torch.from_numpy(np.concatenate(ptr)).cuda(),
                             torch.from_numpy(np.concatenate(idx).astype(np.int32)).cuda(),
                             torch.from_numpy(np.concatenate(val).astype(np.float64)).cuda())

    def entries(self) -> int:
        return self.factor_.entries()

    def close(self):
        self.factor_.close()


class ShardedBatch:
    """Independent systems split over the ranks of a process group (one process per GPU): `shard`
    gives each rank a share of about equal estimated factor work, each rank factors and solves its
    share as one block-diagonal batch on its own GPU (no collective on the data path), and
    `gather` brings every system's solution to every rank with one all-gather at the end.

    `systems` are objects with `upper()`, `csr` and `rhs` (n x k, the same k for all), the same
    list on every rank. `solver`, when given, replaces the device batch: a function of the
    rank's systems returning their solutions (used to test the host logic without a GPU)."""

    def __init__(self, systems, rank: int, world: int, precision: int = FP64, device: int = 0,
                 max_entries: int = 2**62, costs=None, solver=None):
        self.systems = systems
        self.rank, self.world = rank, world
        self.k = systems[0].rhs.shape[1] if systems else 0
        parts = [s.upper() for s in systems]
        costs = costs if costs is not None else [factor_cost(p) for p in parts]
        self.shares = shard(costs, world)
        self.share = self.shares[rank]
        self.solver = solver
        self.batch = None
        self._parts = [parts[i] for i in self.share]
        if solver is None and self.share:
            self.batch = BatchFactor(self._parts, max_entries, precision, device)

    def factor(self):
        if self.batch is not None:
            self.batch.factor([p.val for p in self._parts])

    def solve(self, tol: float | None = None, torch=None) -> list[np.ndarray]:
        """This rank's systems' solutions (n_i x k each): the direct solve, or refinement to `tol`
        relative residual per system and right-hand side."""
        mine = [self.systems[i] for i in self.share]
        if self.solver is not None:
            return self.solver(mine)
        if self.batch is None:
            return []
        if tol is None:
            return self.batch.solve([s.rhs for s in mine])
        return self.batch.refine_solve([s.csr for s in mine], [s.rhs for s in mine], tol=tol, torch=torch)

    def upload(self, torch=None):
        """This rank's systems' values, rows and right-hand sides into its GPU's memory."""
        if self.batch is not None:
            mine = [self.systems[i] for i in self.share]
            self.batch.upload([p.val for p in self._parts], [s.csr for s in mine], [s.rhs for s in mine], torch)

    def step(self, tol: float = 1e-10, max_iter: int = 40):
        """One factorisation and refined solve of this rank's share from device memory (no
        collective). Returns (residuals, solves), or None for an empty share."""
        if self.batch is None:
            return None
        return self.batch.run_device(tol, max_iter)

    def local_solutions(self) -> list[np.ndarray]:
        """This rank's systems' solutions of the last step, in share order."""
        if self.solver is not None or self.batch is None:
            return self.solve() if self.solver is not None else []
        return self.batch.download()

    def gather(self, local: list[np.ndarray], torch=None, device=None) -> list[np.ndarray]:
        """Every system's solution on every rank: the ranks' solutions, each flattened in share
        order and padded to the longest share, in one all_gather (over NCCL, on `device`, or gloo
        on the host)."""
        import torch as _torch
        import torch.distributed as dist
        torch = torch or _torch
        sizes = [int(s.rhs.shape[0]) * self.k for s in self.systems]
        lengths = [sum(sizes[i] for i in sh) for sh in self.shares]
        most = max(lengths) if lengths else 0
        flat = np.zeros(most)
        at = 0
        for x in local:
            flat[at:at + x.size] = np.asarray(x).ravel(order="F")
            at += x.size
        t = torch.from_numpy(flat)
        if device is not None:
            t = t.to(device)
        if self.world > 1:
            out = [torch.empty_like(t) for _ in range(self.world)]
            dist.all_gather(out, t)
        else:
            out = [t]
        result: list = [None] * len(self.systems)
        for r, sh in enumerate(self.shares):
            buf = out[r].cpu().numpy()
            at = 0
            for i in sh:
                n = int(self.systems[i].rhs.shape[0])
                result[i] = buf[at:at + n * self.k].reshape((n, self.k), order="F").copy()
                at += n * self.k
        return result

    def close(self):
        if self.batch is not None:
            self.batch.close()
            self.batch = None

"""The batch's multi-rank path on the CPU: two gloo ranks (127.0.0.1) run the library's
ShardedBatch over 12 independent boxes: the systems are sharded by estimated factor work with no
collective on the data path, each rank solves its own share (the oracle's solve is injected in
place of the GPU batch, so the host logic runs without a device), and one all-gather at the end
brings every system's solution to every rank: each system solved exactly once, every rank's
gathered solutions bit for bit the same, each to 1e-10."""
import os
import socket

import numpy as np
import torch.distributed as dist
import torch.multiprocessing as mp

from fieldcraft_b200 import problems
from fieldcraft_b200.batch import ShardedBatch, shard


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _oracle_solver(rank, seen):
    from oracle import oracle

    def solve(systems):
        out = []
        for b in systems:
            up = b.upper()
            f = oracle.Fac(oracle.Sym(up.n, up.ptr, up.idx), up.val)
            out.append(f.solve(np.asfortranarray(b.rhs.copy())))
            seen.append(b.name)
        return out
    return solve


def _rank(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=__import__("datetime").timedelta(seconds=60))
    boxes = list(problems.uneven_boxes(count=12, lo=2, hi=5, nrhs=2, seed=3))
    seen = []
    sb = ShardedBatch(boxes, rank, world, solver=_oracle_solver(rank, seen))
    sb.factor()
    local = sb.solve()
    xs = sb.gather(local)
    dist.destroy_process_group()
    from oracle import oracle
    res = [max(np.linalg.norm(oracle.spmv(b.n, b.csr.ptr, b.csr.idx, b.csr.val, x[:, j]) - b.rhs[:, j]) / np.linalg.norm(b.rhs[:, j]) for j in range(2))
           for b, x in zip(boxes, xs)]
    out.put((rank, sb.share, seen, np.concatenate([x.ravel() for x in xs]), max(res)))


def test_two_ranks_shard_the_batch():
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    got = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    got.sort(key=lambda g: g[0])
    shares = [g[1] for g in got]
    assert sorted(i for sh in shares for i in sh) == list(range(12)) and all(shares)
    assert len(got[0][2]) + len(got[1][2]) == 12  # each system solved once, by its own rank
    assert np.array_equal(got[0][3], got[1][3])  # every rank holds every solution
    assert max(g[4] for g in got) <= 1e-10


def test_shard_balances_and_is_deterministic():
    costs = [5, 1, 9, 3, 3, 7, 2, 8]
    a = shard(costs, 3)
    assert a == shard(costs, 3)
    assert sorted(i for s in a for i in s) == list(range(len(costs)))
    loads = [sum(costs[i] for i in s) for s in a]
    assert max(loads) - min(loads) <= max(costs)

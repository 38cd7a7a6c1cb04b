"""The batch's multi-rank path on the CPU: two gloo ranks (127.0.0.1) shard 12 independent boxes
by estimated factor work with no collective on the data path, each solves its own share (the
oracle stands in for the device here), and one all-gather at the end brings every system's
residual to every rank: each system solved exactly once, to 1e-10."""
import os
import socket

import numpy as np
import torch.distributed as dist
import torch.multiprocessing as mp

from fieldcraft_b200 import problems
from fieldcraft_b200.batch import factor_cost, shard


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=__import__("datetime").timedelta(seconds=60))
    from oracle import oracle
    boxes = list(problems.uneven_boxes(count=12, lo=2, hi=5, nrhs=2, seed=3))
    parts = [b.upper() for b in boxes]
    mine = shard([factor_cost(p) for p in parts], world)[rank]
    local = {}
    for i in mine:
        p, up = boxes[i], parts[i]
        f = oracle.Fac(oracle.Sym(up.n, up.ptr, up.idx), up.val)
        x = f.solve(np.asfortranarray(p.rhs.copy()))
        r = max(np.linalg.norm(oracle.spmv(p.n, p.csr.ptr, p.csr.idx, p.csr.val, x[:, j]) - p.rhs[:, j])
                / np.linalg.norm(p.rhs[:, j]) for j in range(x.shape[1]))
        local[i] = (rank, float(r))
    gathered = [None] * world
    dist.all_gather_object(gathered, local)
    dist.destroy_process_group()
    if rank == 0:
        merged = {}
        for d in gathered:
            for k, v in d.items():
                assert k not in merged
                merged[k] = v
        out.put(merged)


def test_two_ranks_shard_the_batch():
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    merged = q.get(timeout=120)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert sorted(merged) == list(range(12))
    assert {v[0] for v in merged.values()} == {0, 1}
    assert max(v[1] for v in merged.values()) <= 1e-10


def test_shard_balances_and_is_deterministic():
    costs = [5, 1, 9, 3, 3, 7, 2, 8]
    a = shard(costs, 3)
    assert a == shard(costs, 3)
    assert sorted(i for s in a for i in s) == list(range(len(costs)))
    loads = [sum(costs[i] for i in s) for s in a]
    assert max(loads) - min(loads) <= max(costs)

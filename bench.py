#!/usr/bin/env python
"""Benchmark of the B200 supernodal Cholesky: seconds to relative residual <= 1e-10 for the FP64
direct solve of K u = f on a 48^3 hex8 block (345 744 free DOFs, per-element lognormal E, 64
Gaussian top-face load cases), the workload the headline FP64-on-GPU metric is quoted on.

One step = the numeric factorisation of K (values already in HBM), the solve of the 64
right-hand sides, and the residual check ||f - K u|| / ||f|| of every one of them on the device.
`value` is the mean seconds per step (lower is better). `e2e` is the same step through the public
C ABI with host buffers (values and right-hand sides copied in, solutions copied out).

python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]
With N > 1 (torchrun), every rank solves its own replica (the path does not shard: replicas only)
and the slowest rank's time is reported.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "s to rel-res 1e-10: FP32+IR & NN-FCG vs FP64 GPU Cholesky; TFLOP/s, GB/s"
UNIT = "s"
N_EL, NRHS, SEED = 48, 64, 2024
# profile kinds (fc_chol_profile_read) and their names
KERNEL_KINDS = [(0, "assemble"), (1, "panel"), (3, "gemm"), (12, "gemm_tcgen05"), (15, "pack_tcgen05"),
                (10, "inverse_products"),
                (11, "inverse_blocks"),
                (19, "solve_gemm"), (20, "solve_assemble"),
                (22, "solve_fwd_inverse"), (23, "solve_bwd_inverse"), (29, "solve_thin_fwd"),
                (30, "solve_thin_bwd")]


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["b200", "reference"], default="b200")
    ap.add_argument("--n-el", type=int, default=N_EL)
    ap.add_argument("--nrhs", type=int, default=NRHS)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--ref-budget-s", type=float, default=300.0,
                    help="the reference arm's time budget for its full runs (at least one run is made)")
    ap.add_argument("--no-fp32", action="store_true", help="skip the mixed-precision measurement")
    ap.add_argument("--profile-only", action="store_true", help="a short run for ncu (no baselines, no e2e)")
    ap.add_argument("--no-nn", action="store_true", help="skip the learned-preconditioner measurement")
    ap.add_argument("--nn-pairs", type=int, default=256, help="training pairs of the headline's learned preconditioner")
    ap.add_argument("--nn-epochs", type=int, default=3, help="training epochs of the learned preconditioner")
    ap.add_argument("--nn-plate", type=int, default=64, metavar="N",
                    help="the headline line's learned preconditioner on an N x N x 8 plate (the config-5 "
                         "workload at N = 128) with on-policy training; 0: on the headline's own K")
    ap.add_argument("--profile-kernels", choices=["fp32-factor", "unet"], default=None,
                    help="a short run for a profiler: two FP32 factorisations of the --n-el block, or the "
                         "U-Net's forward and backward passes on a 64x64x8 plate, twice")
    ap.add_argument("--ldlt", type=int, default=0, metavar="N_EL",
                    help="instead: the symmetric indefinite LDL^T (factor, inertia and solve of 16 RHS) on the "
                         "N_EL^3 lognormal block shifted by 2%% of its mean diagonal, against the oracle's LDL^T")
    ap.add_argument("--assembly", type=int, default=0, metavar="N_EL",
                    help="instead: K_ff of the N_EL^3 lognormal block assembled on the device (element matrices "
                         "and the gather), checked bit for bit against the host builder")
    ap.add_argument("--config", type=int, choices=[1, 2, 3, 4, 5], default=2,
                    help="workload: 2 (default) the 48^3 block the metric is quoted on; 1 cantilever, 3 256 "
                         "uneven boxes batched, 4 64^3 random-field block to 1e-12, 5 128x128x8 plate (NN-FCG)")
    return ap.parse_args()


def factor_flops(problem):
    """Sum of squared column counts of L (the Davis convention the metric's TFLOP/s uses)."""
    from fieldcraft_b200 import Symbolic
    a = Symbolic(problem.upper(), 2**62).arrays()
    w = np.diff(a["first"])
    m = np.diff(a["rptr"])
    tot = 0.0
    for mm, ww in zip(m, w):
        c = mm - np.arange(ww, dtype=np.float64)
        tot += float(np.dot(c, c))
    return tot, int(a["entries"])


def oracle_factor_flops(sym) -> float:
    """Sum of squared column counts of L from the oracle's own analysis."""
    first, rptr = sym.array("first"), sym.array("rptr")
    tot = 0.0
    for mm, ww in zip(np.diff(rptr), np.diff(first)):
        c = mm - np.arange(ww, dtype=np.float64)
        tot += float(np.dot(c, c))
    return tot


def cpu_model() -> str:
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def oracle_full_run(w, threads: int, runs_budget_s: float, max_runs: int, min_runs: int = 1):
    """The oracle (the reference's CPU algorithm restated) on the whole workload `w` (an oracle
    workload: its own builder, no product code): the symbolic analysis once, then up to
    `max_runs` runs of the numeric factorisation and the solve of every right-hand side, timed
    apart, while the next run still fits `runs_budget_s` (at least `min_runs`). The factor uses
    `threads` threads (subtree tasks and row tiles, as cholesky.rs:1443-1529); the solve is
    sequential over groups of 6 right-hand sides, as solve_supernodes_many (cholesky.rs:876-897)
    is. Returns the timings and the last run's solution."""
    from oracle import oracle
    oracle.set_threads(threads)
    uptr, uidx, uval = w.upper()
    t0 = time.perf_counter()
    sym = oracle.Sym(w.n, uptr, uidx)
    t_sym = time.perf_counter() - t0
    fac_s, sol_s, x = [], [], None
    spent = 0.0
    while len(fac_s) < max_runs:
        if len(fac_s) >= min_runs and spent + (fac_s[-1] + sol_s[-1]) > runs_budget_s:
            break
        t0 = time.perf_counter()
        f = oracle.Fac(sym, uval)
        t1 = time.perf_counter()
        x = f.solve(w.rhs.copy())
        t2 = time.perf_counter()
        del f
        fac_s.append(t1 - t0)
        sol_s.append(t2 - t1)
        spent += t2 - t0
    return {"symbolic_s": t_sym, "factor_s": fac_s, "solve_s": sol_s, "flops": oracle_factor_flops(sym),
            "entries": sym.info("entries"), "x": x}


class Clocks:
    """nvidia-smi samples during the timed region."""

    def __init__(self, index: int):
        self.index = index
        self.file = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.proc = None

    def __enter__(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=self.file, stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        self.file.flush()
        self.file.seek(0)
        sm, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.file.read().splitlines():
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = max(mx, float(f[2]))
            except ValueError:
                continue
            for name, val in zip(names, f[5:9]):
                if val.lower() == "active":
                    reasons.add(name)
        os.unlink(self.file.name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx or None,
                "reasons": sorted(reasons), "samples": len(sm)}


def dgemm_peak(torch):
    """Measured FP64 peak: cuBLAS DGEMM 8192^3 (torch.matmul), best of 5, TFLOP/s."""
    n = 8192
    a = torch.randn(n, n, dtype=torch.float64, device="cuda")
    b = torch.randn(n, n, dtype=torch.float64, device="cuda")
    c = a @ b
    best = 1e30
    for _ in range(5):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        c = a @ b
        e1.record()
        e1.synchronize()
        best = min(best, e0.elapsed_time(e1))
    del a, b, c
    return 2.0 * n ** 3 / (best * 1e-3) / 1e12


def run_reference(args, rank, world):
    """The reference arm: the reference's CPU algorithm (the oracle restatement; the Rust reference
    cannot be built here) on the host cores, on the whole benchmark workload built by the oracle's
    own hex8 builder (no product code is loaded). Each step is one numeric factorisation plus the
    solve of every right-hand side of the full 48^3 system; as many steps as fit the time budget
    are run (at least one), and the line says how many. Under torchrun only rank 0 works."""
    if rank != 0:
        return
    from oracle import workloads
    threads = os.cpu_count() or 1
    t0 = time.perf_counter()
    w = workloads.lognormal_block(args.n_el, nrhs=args.nrhs, seed=SEED)
    t_build = time.perf_counter() - t0
    want = max(1, args.steps)
    # every run is timed: each allocates its factor afresh (as the reference's Symbolic::allocate
    # does), so a first run has no cold state the later ones skip; the untimed analysis and input
    # build come first
    r = oracle_full_run(w, threads, args.ref_budget_s, max_runs=want, min_runs=1)
    runs = [a + b for a, b in zip(r["factor_s"], r["solve_s"])]
    warm = 0
    timed = runs
    value = float(np.mean(timed))
    fx = r["x"]
    # the answer's residual, so the timed work is known to be the solve
    rel = max(float(np.linalg.norm(oracle_spmv(w, fx[:, j]) - w.rhs[:, j]) / np.linalg.norm(w.rhs[:, j]))
              for j in range(0, fx.shape[1], max(1, fx.shape[1] // 4)))
    sample = (f"the whole workload (n={w.n}, {r['flops']:.3e} factor flops): {len(runs)} run(s) of the oracle's "
              f"numeric factorisation on {threads} threads + the solve of {args.nrhs} RHS (sequential groups "
              f"of 6, as the reference), {len(timed)} timed of "
              f"{want} requested within a {args.ref_budget_s:.0f} s budget; symbolic analysis "
              f"{r['symbolic_s']:.2f} s and input build {t_build:.1f} s untimed; CPU {cpu_model()}")
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": len(timed), "steps_requested": args.steps, "warmup": warm, "ms_per_step": value * 1e3,
        "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded lognormal E, Gaussian loads), built by the oracle's own hex8 builder",
        "config": {"workload": f"FP64 direct solve, hex8 block {args.n_el}^3 lognormal E (sigma 0.5), z=0 clamped, "
                               f"{args.nrhs} Gaussian top-face RHS", "n": w.n, "nnz": int(w.idx.size),
                   "nrhs": args.nrhs, "factor_entries": r["entries"], "factor_flops": r["flops"]},
        "phases_s": {"symbolic": r["symbolic_s"], "factor": r["factor_s"], "solve": r["solve_s"],
                     "factor_best": min(r["factor_s"]), "solve_best": min(r["solve_s"])},
        "timed_region_s": float(np.sum(timed)), "relres_max_sampled": rel,
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port", "sample": sample,
                         "cpu_model": cpu_model()},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def same_system(w, csr, rhs) -> bool:
    """Whether the oracle-built workload is bit for bit the system the device solves."""
    same = lambda a, b: a.shape == b.shape and a.dtype == b.dtype and a.tobytes() == b.tobytes()
    return (w.n == csr.n and same(w.ptr.astype(np.int64), csr.ptr.astype(np.int64)) and same(w.idx, csr.idx)
            and same(w.val, csr.val) and same(np.asfortranarray(w.rhs), np.asfortranarray(rhs)))


def per_rhs_error(x, ref):
    """||x_j - ref_j|| / ||ref_j|| for each column j."""
    return np.linalg.norm(x - ref, axis=0) / np.linalg.norm(ref, axis=0)


def oracle_spmv(w, x):
    from oracle import oracle
    return oracle.spmv(w.n, w.ptr, w.idx, w.val, x)


def nn_plate_block(size: int, torch, lib) -> dict:
    """nn_fcg_block on the size x size x 8 plate (problems.plate: the config-5 workload at 128):
    1 000 Cholesky pairs for 8 epochs, then three on-policy rounds of 24 right-hand sides x 9
    snapshots for 4 epochs each, a 3-level network, two held-out right-hand sides. On the 128 x 128
    x 8 plate itself the same schedule left the loss near 0.6 and the network was dropped."""
    from fieldcraft_b200 import Factor, Symbolic, problems
    p = problems.plate(size, size, 8, nrhs=2)
    up = p.upper()
    f = Factor(Symbolic(up, 2**62))
    n = p.n
    d_val = torch.from_numpy(up.val).cuda()
    csr = tuple(torch.from_numpy(a).cuda() for a in (p.csr.ptr, p.csr.idx, p.csr.val))
    b = torch.from_numpy(np.ascontiguousarray(p.rhs[:, 0])).cuda()
    stream = torch.cuda.Stream()
    f.set_stream(stream.cuda_stream)
    tt = []
    for _ in range(3):
        x = b.clone()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        with torch.cuda.stream(stream):
            assert lib.fc_chol_factor_device_async(f.handle, C.c_void_p(d_val.data_ptr()), up.val.size) == 0
            assert lib.fc_chol_solve_device_async(f.handle, C.c_void_p(x.data_ptr()), 1, n) == 0
        e1.record(stream)
        e1.synchronize()
        tt.append(e0.elapsed_time(e1))
    f.set_stream(None)
    out = nn_fcg_block(p, f, csr, torch, pairs=1000, epochs=8, cols=[0, 1], cap=3000, chol_ms=float(np.min(tt[1:])),
                       batch=16, levels=3, lr=3e-4, rounds=3, round_rhs=24, round_epochs=4, round_lr=2e-4)
    out["problem"] = (f"plate {size}x{size}x8 (n = {n}), E a lognormal random field (contrast 100), side faces "
                      f"clamped, held-out random top-face pressures")
    f.close()
    return out


def nn_levels(p) -> int:
    """U-Net levels for a box problem's node grid: pooling until the longest side is about 8 nodes."""
    longest = max(p.dims) + 1
    levels = 1
    while longest > 8 and levels < 6:
        longest = (longest + 1) // 2
        levels += 1
    return levels


def nn_fcg_block(p, factor64, csr_dev, torch, pairs: int, epochs: int, cols, cap: int, chol_ms: float,
                 batch: int = 8, levels: int | None = None, lr: float = 1e-3, rounds: int = 0, round_rhs: int = 24,
                 round_epochs: int = 4, round_lr: float = 2e-4) -> dict:
    """The learned preconditioner on the same K: pairs (r, K^-1 r) from the Cholesky solve, minibatch
    Adam training on the GPU of a U-Net whose output is added to K's nodal block-Jacobi part (then
    `rounds` on-policy rounds: pairs from the residuals of the network's own Krylov solve, see
    train_on_policy), then flexible CG to rel-res 1e-10 from zero on held-out right-hand sides with
    the network ('nn_fcg'), with the block-Jacobi part alone ('bj') and with no preconditioner
    ('cg'), all capped at `cap` iterations with the Cholesky solve as fallback; each the median of
    three timed runs after an untimed one. chol_ms: the FP64 Cholesky's time for one right-hand side (factor + solve) on the
    same K."""
    from fieldcraft_b200.unet import UNet, fcg, output_scale, train, train_on_policy, training_pairs
    levels = levels or nn_levels(p)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    R, E = training_pairs(factor64, p, pairs, seed=SEED + 5, torch=torch)
    torch.cuda.synchronize()
    t1 = time.perf_counter()
    net = UNet(p, seed=0, kref=output_scale(R, E), levels=levels, operator=csr_dev)
    losses = train(net, R, E, epochs=epochs, lr=lr, torch=torch, csr_device=csr_dev, batch=batch, warmup=50)
    round_losses = []
    if rounds:
        R, E, round_losses = train_on_policy(net, factor64, p, csr_dev, R, E, rounds, round_rhs, round_epochs,
                                             round_lr, torch, batch=batch, seed=SEED)
    torch.cuda.synchronize()
    t2 = time.perf_counter()
    del R, E
    runs = []
    for j in cols:
        b = torch.from_numpy(np.ascontiguousarray(p.rhs[:, j])).cuda()
        exact = b.clone()
        factor64.solve_device(exact, 1, p.n)
        row = {}
        for name, use, on in (("nn_fcg", net, True), ("bj", net, False), ("cg", None, True)):
            if use is not None:
                use.enable(on)
            # one untimed run first (first-call set-up, clocks up after the host-side phases), then
            # three timed ones, their median reported (the solve synchronises with the host every
            # few iterations, so one stall of the host shows in a single run)
            times = []
            for timed in (False, True, True, True):
                x = torch.zeros_like(b)
                torch.cuda.synchronize()
                ta = time.perf_counter()
                it, rel, fb = fcg(csr_dev, b, x, net=use, fallback=factor64, tol=1e-10, max_iter=cap, keep=4)
                torch.cuda.synchronize()
                if timed:
                    times.append(time.perf_counter() - ta)
            dt = float(np.median(times))
            err = float((torch.linalg.vector_norm(x - exact) / torch.linalg.vector_norm(exact)).item())
            row[name] = {"iterations": it, "s": dt, "s_runs": times, "relres": rel, "fallback": fb,
                         "err_vs_cholesky": err}
            if name == "nn_fcg":
                row[name]["network_iterations"] = net.stat(1)
                row[name]["network_dropped"] = bool(net.stat(2))
        net.enable(True)
        runs.append(row)
    nn_s = [r["nn_fcg"]["s"] for r in runs]
    net.close()
    return {"value": float(np.mean(nn_s)), "unit": UNIT,
            "speedup_vs_fp64": (chol_ms / 1e3) / float(np.mean(nn_s)),
            "speedup_vs_cg": float(np.mean([r["cg"]["s"] for r in runs])) / float(np.mean(nn_s)),
            "fp64_cholesky_1rhs_s": chol_ms / 1e3, "pairs": pairs, "epochs": epochs, "batch": batch, "lr": lr,
            "levels": levels, "pairs_s": t1 - t0, "train_s": t2 - t1, "loss_by_epoch": losses, "cap": cap,
            "on_policy_rounds": rounds, "on_policy_pairs_per_round": round_rhs * 9 if rounds else 0,
            "on_policy_epochs": round_epochs if rounds else 0, "on_policy_loss_by_round": round_losses,
            "rhs": runs,
            "what": f"{levels}-level 32-channel BF16 3D-conv U-Net added to K's nodal block-Jacobi inverse, trained "
                    "(energy-norm loss, minibatch Adam) on pairs from the Cholesky solve; flexible CG (4 kept "
                    "directions) from zero to rel-res 1e-10 on held-out right-hand sides; 'bj' the same solver "
                    "with the block-Jacobi part alone, 'cg' with no preconditioner; a run that did not converge "
                    "within the cap falls back to the Cholesky solve (fallback true, time included)"}


def block_csr(parts):
    """The rows of diag(A_0, A_1, ...) from each system's rows."""
    from fieldcraft_b200.cholesky import Csr
    ptr, idx, val = [np.zeros(1, np.int64)], [], []
    col0 = nnz0 = 0
    for c in parts:
        ptr.append(c.ptr[1:].astype(np.int64) + nnz0)
        idx.append(c.idx.astype(np.int64) + col0)
        val.append(c.val)
        col0 += c.n
        nnz0 += int(c.ptr[-1])
    return Csr(col0, np.concatenate(ptr), np.concatenate(idx).astype(np.int32), np.concatenate(val))


def shifted(problem, theta: float):
    """The problem's K - theta * mean(diag K) * I (indefinite for theta above the lowest eigenvalue's
    share): the full CSR and the upper triangle by columns."""
    from fieldcraft_b200.cholesky import Csr, UpperColumns
    csr = problem.csr
    rows = np.repeat(np.arange(csr.n), np.diff(csr.ptr))
    on = csr.idx == rows
    sigma = theta * float(np.mean(csr.val[on]))
    val = csr.val.copy()
    val[on] -= sigma
    a = Csr(csr.n, csr.ptr, csr.idx, val)
    return a, UpperColumns.from_symmetric(a), sigma


def run_ldlt(args, torch, lib, local: int):
    """The symmetric indefinite factor (FC_PRECISION_LDLT) on a shifted lognormal block: per step
    the factorisation from values in HBM, the solve of 16 right-hand sides (the first after a
    factorisation folds the pivot orders into the solve's structure) and the residual, timed on
    the device; the inertia; the oracle's LDL^T on a bounded sample, scaled by factor flops. One
    JSON line."""
    from fieldcraft_b200 import LDLT, Factor, Symbolic, problems
    from fieldcraft_b200.cholesky import Status, raise_for
    from oracle import oracle
    R = 16
    p = problems.lognormal_block(args.ldlt, nrhs=R, seed=SEED)
    a, up, sigma = shifted(p, 0.02)
    n = a.n
    f = Factor(Symbolic(up, 2**62), precision=LDLT, device=local)
    stream = torch.cuda.Stream()
    f.set_stream(stream.cuda_stream)
    d_val = torch.from_numpy(up.val).cuda()
    csr_dev = tuple(torch.from_numpy(v).cuda() for v in (a.ptr, a.idx, a.val))
    d_f = torch.from_numpy(np.ascontiguousarray(p.rhs.T)).cuda()
    d_x, d_r = torch.empty_like(d_f), torch.empty_like(d_f)
    fnorm = torch.linalg.vector_norm(d_f, dim=1)

    def step():
        with torch.cuda.stream(stream):
            assert lib.fc_chol_factor_device_async(f.handle, C.c_void_p(d_val.data_ptr()), up.val.size) == 0
            d_x.copy_(d_f)
            assert lib.fc_chol_solve_device_async(f.handle, C.c_void_p(d_x.data_ptr()), R, n) == 0
            lib.fc_csr_spmv_device(n, *(C.c_void_p(v.data_ptr()) for v in csr_dev), C.c_void_p(d_x.data_ptr()),
                                   C.c_void_p(d_r.data_ptr()), R, n, C.c_void_p(stream.cuda_stream))
            d_r.sub_(d_f)
            return torch.linalg.vector_norm(d_r, dim=1) / fnorm

    for _ in range(args.warmup):
        step()
    st = Status()
    lib.fc_chol_check(f.handle, C.byref(st))
    raise_for(st)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        rel = step()
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / args.steps
    pos, neg, two = C.c_int64(0), C.c_int64(0), C.c_int64(0)
    lib.fc_chol_inertia(f.handle, C.byref(pos), C.byref(neg), C.byref(two), C.byref(st))
    raise_for(st)
    # the oracle's LDL^T on the whole shifted system, once, from the oracle's own builder
    from oracle import workloads
    ow = workloads.lognormal_block(args.ldlt, nrhs=R, seed=SEED)
    rows = np.repeat(np.arange(ow.n), np.diff(ow.ptr))
    oval = ow.val.copy()
    oval[ow.idx == rows] -= sigma
    same_input = bool(np.array_equal(oval.view(np.uint64), a.val.view(np.uint64)))
    uptr, uidx, uval = oracle.upper_from_symmetric(ow.n, ow.ptr, ow.idx, oval)
    threads = os.cpu_count() or 1
    oracle.set_threads(threads)
    sym = oracle.Sym(ow.n, uptr, uidx)
    t0 = time.perf_counter()
    of = oracle.Ldlt(sym, uval)
    t1 = time.perf_counter()
    xo = of.solve(ow.rhs.copy(order="F"))
    t2 = time.perf_counter()
    err = per_rhs_error(d_x.cpu().numpy().T, xo)
    line = {
        "metric": "s per LDL^T factorisation + 16 solves (symmetric indefinite, FP64)", "value": ms / 1e3,
        "unit": "s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
        "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded)",
        "config": {"workload": f"hex8 block {args.ldlt}^3 lognormal E, K - {sigma:.4g} I (2% of the mean diagonal), "
                               f"{R} RHS", "n": n, "inertia": [pos.value, neg.value], "two_by_two": two.value},
        "relres_max": float(rel.max().item()), "err_vs_oracle_max": float(np.max(err)),
        "cpu_baseline": {"value": t2 - t0, "unit": "s", "cores": threads, "kind": "port", "cpu_model": cpu_model(),
                         "sample": f"the whole shifted system once (the oracle's own builder, bit for bit this K: "
                                   f"{same_input}): LDL^T factorisation {t1 - t0:.2f} s on {threads} threads + "
                                   f"{R} solves {t2 - t1:.2f} s"},
    }
    print(json.dumps(line), flush=True)
    f.close()


def run_assembly(args, torch, lib, local: int):
    """K_ff of the N_EL^3 lognormal block on the device (fc_fem_assemble_device) from element moduli
    in HBM, per step timed on the device; the values checked against the host builder's bit for
    bit; the host builder's whole run (mesh, order, pattern, assembly) and the same entry-by-entry
    assembly on one host thread beside it. One JSON line."""
    from fieldcraft_b200 import problems
    n_el = args.assembly
    t0 = time.perf_counter()
    p = problems.lognormal_block(n_el, nrhs=1, seed=SEED)
    t_builder = time.perf_counter() - t0
    d = problems.DeviceAssembly(p, device=local)
    young = torch.from_numpy(p.young).cuda()
    val = torch.empty(p.csr.val.size, dtype=torch.float64, device="cuda")
    stream = torch.cuda.Stream()
    for _ in range(args.warmup):
        d.assemble(young, val, stream_ptr=stream.cuda_stream)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        d.assemble(young, val, stream_ptr=stream.cuda_stream)
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / args.steps
    same = bool(np.array_equal(val.cpu().numpy().view(np.uint64), p.csr.val.view(np.uint64)))
    fn = lib.fc_test_fem_assemble_host
    fn.restype = C.c_int
    keep = [np.ascontiguousarray(a) for a in (p.csr.ptr, p.csr.idx, p.eq, p.young)]
    out = np.empty(p.csr.val.size)
    t0 = time.perf_counter()
    fn(n_el, n_el, n_el, C.c_double(float(n_el)), C.c_double(float(n_el)), C.c_double(float(n_el)), C.c_int64(p.n),
       *(C.c_void_p(a.ctypes.data) for a in keep), C.c_double(0.3), C.c_void_p(out.ctypes.data))
    t_host = time.perf_counter() - t0
    elements = n_el ** 3
    line = {
        "metric": "s per assembly of K_ff on the device (element matrices + gather)", "value": ms / 1e3, "unit": "s",
        "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": False,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded)",
        "config": {"workload": f"hex8 block {n_el}^3 lognormal E, z=0 clamped", "elements": elements, "n": p.n,
                   "nnz": int(p.csr.val.size)},
        "bitwise_equal_to_host_builder": same,
        "cpu_baseline": {"value": t_host, "unit": "s", "cores": 1, "kind": "port",
                         "sample": "the same entry-by-entry assembly on one host thread; the host builder's whole "
                                   f"run (mesh, order, pattern, parallel assembly) took {t_builder:.2f} s"},
    }
    print(json.dumps(line), flush=True)
    d.close()


def run_config(args, cfg: int, torch, lib, local: int):
    """Configs other than the headline: FP64 direct solve vs FP32+IR to the config's tolerance on
    the same K (and, for the plate, the learned preconditioner), each timed on the device from
    values and right-hand sides in HBM to the verified residual. One JSON line."""
    from fieldcraft_b200 import FP32_IR, FP64, Factor, Symbolic, problems
    from fieldcraft_b200.batch import block_diagonal
    from oracle import workloads
    t_host = time.perf_counter()
    sizes = None
    owl = None  # the same workload built by the oracle alone (its CPU leg and the per-RHS errors)
    if cfg == 1:
        owl = workloads.cantilever()
        p = problems.cantilever()
        csr, up, rhs, tol = p.csr, p.upper(), p.rhs, 1e-10
        workload = "cantilever 40x4x4 hex8 (100x10x10 mm, E 210 GPa, nu 0.3), x=0 clamped, 1 kN tip load, 1 RHS"
    elif cfg == 4:
        p = problems.field_block(64, nrhs=16)
        owl = workloads.field_block(64, nrhs=16) if not args.no_cpu_baseline else None
        csr, up, rhs, tol = p.csr, p.upper(), p.rhs, 1e-12
        workload = "hex8 block 64^3, lognormal random-field E (corr 6, contrast 1e3), z=0 clamped, 16 RHS, to 1e-12"
    elif cfg == 5:
        p = problems.plate(128, 128, 8, nrhs=4)
        owl = workloads.plate(128, 128, 8, nrhs=4) if not args.no_cpu_baseline else None
        csr, up, rhs, tol = p.csr, p.upper(), p.rhs, 1e-10
        workload = "hex8 plate 128x128x8, lognormal random-field E (corr 8, contrast 100), sides clamped, top pressures"
    else:
        boxes = list(problems.uneven_boxes(count=256, lo=4, hi=24, nrhs=8, seed=11))
        if not args.no_cpu_baseline:
            owl = workloads.stacked(list(workloads.uneven_boxes(count=256, lo=4, hi=24, nrhs=8, seed=11)))
        up = block_diagonal([b.upper() for b in boxes])
        csr = block_csr([b.csr for b in boxes])
        rhs = np.concatenate([b.rhs for b in boxes], axis=0)
        sizes = np.array([b.n for b in boxes])
        p = None
        tol = 1e-10
        workload = "256 independent hex8 boxes, nx,ny,nz ~ U{4..24}, E ~ U[70,210] GPa, nu ~ U[0.25,0.35], " \
                   "z=0 clamped, 8 RHS each, one block-diagonal factorisation and solve"
    sym = Symbolic(up, 2**62)
    host_s = time.perf_counter() - t_host
    n, R = csr.n, rhs.shape[1]
    same_input = owl is not None and same_system(owl, csr, rhs)
    stream = torch.cuda.Stream()
    csr_dev = tuple(torch.from_numpy(a).cuda() for a in (csr.ptr, csr.idx, csr.val))
    d_val = torch.from_numpy(up.val).cuda()
    d_b = torch.from_numpy(np.ascontiguousarray(rhs.T)).cuda()
    res, keep64, tuned = {}, None, {}
    for prec in (FP64, FP32_IR):
        f = Factor(sym, precision=prec, device=local)
        f.set_stream(stream.cuda_stream)
        if cfg == 3:
            # the batch's variants picked on the batch itself by the autotuner
            from fieldcraft_b200.autotune import autotune
            tuned[prec] = autotune(f, prec, d_val, up.val.size, csr_dev, d_b, R, tol, torch, repeats=1,
                                   stream=stream)
        times, its, rels = [], 0, None
        x = torch.zeros_like(d_b)
        for it in range(args.warmup + args.steps):
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            with torch.cuda.stream(stream):
                assert lib.fc_chol_factor_device_async(f.handle, C.c_void_p(d_val.data_ptr()), up.val.size) == 0
            rel, its = f.refine_solve_device(csr_dev, d_b, x, R, n, tol=tol, max_iter=40)
            e1.record(stream)
            e1.synchronize()
            if it >= args.warmup:
                times.append(e0.elapsed_time(e1))
        res[prec] = {"ms": float(np.mean(times)), "solves": int(its), "relres_max": float(np.max(rel)), "x": x}
        if prec == FP64:
            keep64 = f
            flops = float(f.stat(5))
            entries = int(f.entries())
        else:
            f.close()
    x64, x32 = res[FP64]["x"], res[FP32_IR]["x"]
    line = {
        "metric": METRIC, "value": res[FP64]["ms"] / 1e3, "unit": UNIT, "n_gpus": 1, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": res[FP64]["ms"], "higher_is_better": False, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded)",
        "config": {"workload": workload, "config": cfg, "n": n, "nnz": int(csr.idx.size), "nrhs": R,
                   "factor_entries": entries, "factor_flops": flops, "host_prep_s": host_s, "parallelism": "1 GPU"},
        "relres_max": res[FP64]["relres_max"], "relres_target": tol, "solved": res[FP64]["relres_max"] <= tol,
        "factor_tflops_incl_solve": flops / (res[FP64]["ms"] * 1e-3) / 1e12,
        "fp32_ir": {"value": res[FP32_IR]["ms"] / 1e3, "unit": UNIT, "refinement_solves": res[FP32_IR]["solves"],
                    "relres_max": res[FP32_IR]["relres_max"], "speedup_vs_fp64": res[FP64]["ms"] / res[FP32_IR]["ms"]},
    }
    if tuned:
        names = {"1": "solve_schedule", "5": "refinement", "6": "fp32_updates", "7": "solve_cluster", "8": "solve_narrow",
                 "9": "solve_deep"}
        line["autotuned"] = {("fp64" if prec == FP64 else "fp32_ir"):
                             {"options": {names[k]: v for k, v in t["options"].items()},
                              "candidates_ms": t["ms"]} for prec, t in tuned.items()}
    if sizes is not None:
        # every system's own residual of the FP64 batch solution
        r = torch.empty_like(x64)
        lib.fc_csr_spmv_device(n, *(C.c_void_p(a.data_ptr()) for a in csr_dev), C.c_void_p(x64.data_ptr()),
                               C.c_void_p(r.data_ptr()), R, n, None)
        r = (d_b - r) ** 2
        bb = d_b ** 2
        off = np.concatenate([[0], np.cumsum(sizes)])
        seg = torch.tensor(np.repeat(np.arange(sizes.size), sizes), device="cuda")
        rs = torch.zeros((R, sizes.size), dtype=torch.float64, device="cuda").index_add_(1, seg, r)
        bs = torch.zeros_like(rs).index_add_(1, seg, bb)
        line["per_system_relres_max"] = float(torch.sqrt(rs / bs).max().item())
        line["systems"] = int(sizes.size)
    if cfg == 5 and not args.no_nn:
        # FP64 Cholesky for one right-hand side on the same K (factor + solve), the NN-FCG's comparator
        b1 = d_b[0:1].clone()
        tt = []
        for it in range(3):
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            with torch.cuda.stream(stream):
                lib.fc_chol_factor_device_async(keep64.handle, C.c_void_p(d_val.data_ptr()), up.val.size)
                lib.fc_chol_solve_device_async(keep64.handle, C.c_void_p(b1.data_ptr()), 1, n)
            e1.record(stream)
            e1.synchronize()
            tt.append(e0.elapsed_time(e1))
        line["nn_fcg"] = nn_fcg_block(p, keep64, csr_dev, torch, pairs=2000, epochs=args.nn_epochs,
                                      cols=range(min(R, 2)), cap=3000, chol_ms=float(np.min(tt[1:])))
    if not args.no_cpu_baseline and owl is not None:
        threads = os.cpu_count() or 1
        r = oracle_full_run(owl, threads, 0.0, max_runs=1)
        xo = r["x"]
        line["cpu_baseline"] = {"value": r["factor_s"][0] + r["solve_s"][0], "unit": UNIT, "cores": threads,
                                "kind": "port", "cpu_model": cpu_model(),
                                "sample": f"the whole workload once (built by the oracle's own builder, bit for bit "
                                          f"this K and f: {same_input}): numeric factorisation "
                                          f"{r['factor_s'][0]:.2f} s on {threads} threads + solve of {R} RHS "
                                          f"{r['solve_s'][0]:.2f} s (sequential groups of 6); analysis "
                                          f"{r['symbolic_s']:.2f} s untimed"}
        for key, xx in (("fp64", x64), ("fp32_ir", x32)):
            e = per_rhs_error(xx.cpu().numpy().T, xo)
            (line if key == "fp64" else line["fp32_ir"])["err_vs_oracle_per_rhs"] = [float(v) for v in e]
    keep64.close()
    print(json.dumps(line), flush=True)


def run_batch_sharded(args, torch, rank: int, world: int, local: int):
    """The 256 uneven boxes over `world` GPUs (one rank each): ShardedBatch gives each rank a share
    of about equal estimated factor work, each rank factors its share and refines it to 1e-10 per
    system from inputs in its own HBM (no collective on the data path), the step time is the
    slowest rank's (CUDA events, max over ranks), and one all-gather brings every solution to
    every rank at the end (timed apart). FP64 and FP32+IR. One JSON line from rank 0."""
    import torch.distributed as dist
    from fieldcraft_b200 import FP32_IR, FP64, problems
    from fieldcraft_b200.batch import ShardedBatch
    boxes = list(problems.uneven_boxes(count=256, lo=4, hi=24, nrhs=8, seed=11))
    out = {}
    for prec in (FP64, FP32_IR):
        sb = ShardedBatch(boxes, rank, world, precision=prec, device=local)
        sb.upload(torch)
        times, worst = [], 0.0
        for it in range(args.warmup + args.steps):
            dist.barrier()
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            r = sb.step(tol=1e-10)
            e1.record()
            e1.synchronize()
            if it >= args.warmup:
                times.append(e0.elapsed_time(e1))
                worst = max(worst, float(np.max(r[0])) if r is not None else 0.0)
        t = torch.tensor([float(np.mean(times)), worst], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        torch.cuda.synchronize()
        g0 = time.perf_counter()
        xs = sb.gather(sb.local_solutions(), torch=torch, device=f"cuda:{local}")
        gather_s = time.perf_counter() - g0
        # every system's own residual, on the host of rank 0 (the gathered solutions)
        res = 0.0
        if rank == 0:
            from oracle import oracle
            for b, x in zip(boxes, xs):
                for j in range(x.shape[1]):
                    rr = oracle.spmv(b.n, b.csr.ptr, b.csr.idx, b.csr.val, x[:, j]) - b.rhs[:, j]
                    res = max(res, float(np.linalg.norm(rr) / np.linalg.norm(b.rhs[:, j])))
        out[prec] = {"ms": float(t[0].item()), "relres_max": float(t[1].item()), "gather_s": gather_s,
                     "per_system_relres_max": res, "share_systems": len(sb.share)}
        sb.close()
    if rank == 0:
        ms = out[FP64]["ms"]
        line = {
            "metric": METRIC, "value": ms / 1e3, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": False, "scaling": "strong",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded)",
            "config": {"workload": "256 independent hex8 boxes, nx,ny,nz ~ U{4..24}, E ~ U[70,210] GPa, "
                                   "nu ~ U[0.25,0.35], z=0 clamped, 8 RHS each, sharded over the GPUs by estimated "
                                   "factor work", "config": 3, "systems": len(boxes), "parallelism": f"shard x{world}"},
            "relres_max": out[FP64]["relres_max"], "per_system_relres_max": out[FP64]["per_system_relres_max"],
            "gather_s": out[FP64]["gather_s"],
            "fp32_ir": {"value": out[FP32_IR]["ms"] / 1e3, "unit": UNIT,
                        "speedup_vs_fp64": ms / out[FP32_IR]["ms"], "relres_max": out[FP32_IR]["relres_max"],
                        "per_system_relres_max": out[FP32_IR]["per_system_relres_max"]},
        }
        print(json.dumps(line), flush=True)


def hbm_peak() -> tuple:
    """The measured HBM copy bandwidth (GB/s) and where it comes from."""
    mp = ROOT / "MEASURED_PEAKS.json"
    try:
        return float(json.loads(mp.read_text())["hbm_gbs"]), "MEASURED_PEAKS.json hbm_gbs (measured copy)"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback 6.65 TB/s (no measured peaks file)"


def recorded_traffic(kernel: str, flops_per_launch: float):
    """DRAM bytes per launch of `kernel`: the DRAM bytes per useful flop of an ncu capture of a
    small case recorded in profiles/traffic.json, times this run's useful flops per launch. Used
    only while the kernel's source is the one captured (the SHA-256 of its section of the source
    file, between the two markers recorded, beside the figure); otherwise None and why."""
    import hashlib
    rec_file = ROOT / "profiles" / "traffic.json"
    try:
        rec = json.loads(rec_file.read_text())[kernel]
    except (OSError, KeyError, ValueError):
        return None, "no ncu capture recorded for this kernel"
    src = ROOT / rec["source"]
    text = src.read_bytes() if src.exists() else b""
    if "region" in rec:  # only the kernel's own section of the file (from one marker to the next)
        a, b = (m.encode() for m in rec["region"])
        i = text.find(a)
        j = text.find(b, i + 1) if i >= 0 else -1
        text = text[i:j] if i >= 0 and j > i else b""
    sha = hashlib.sha256(text).hexdigest() if text else None
    if sha != rec["source_sha256"]:
        return None, f"the recorded ncu capture was of another build of {rec['source']}"
    return int(rec["bytes_per_useful_flop"] * flops_per_launch), f"{rec['case']}; {rec['how']}"


def stream_time(torch, stream, fn, reps: int = 5, warm: int = 2) -> float:
    """Median milliseconds of fn() on `stream` (CUDA events), after warm-up."""
    for _ in range(warm):
        fn()
    torch.cuda.synchronize()
    ts = []
    for _ in range(reps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        fn()
        e1.record(stream)
        e1.synchronize()
        ts.append(e0.elapsed_time(e1))
    return float(np.median(ts))


def solve_only(lib, f, d_x, d_f, R, n, stream):
    import torch
    with torch.cuda.stream(stream):
        d_x.copy_(d_f)
        assert lib.fc_chol_solve_device_async(f.handle, C.c_void_p(d_x.data_ptr()), R, n) == 0


def assembly_bytes(f) -> float:
    """The front assembly's algorithmic bytes per factorisation (FP64 entries): every value of A
    read once, every child's update-matrix entry (lower triangle) read once, every front entry
    (the L trapezoid and the update matrix's lower triangle) written once."""
    from fieldcraft_b200.cholesky import Symbolic  # noqa: F401
    a = f.symbolic.arrays()
    w = np.diff(a["first"]).astype(np.float64)
    m = np.diff(a["rptr"]).astype(np.float64)
    u = m - w
    lower_u = u * (u + 1) / 2
    trap = w * m - w * (w - 1) / 2
    has_parent = u > 0
    nnz_upper = float(a["nnz"]) if "nnz" in a else float(a["slot"].size)
    return 8.0 * (nnz_upper + lower_u[has_parent].sum() + trap.sum() + lower_u.sum())


def roofline_table(p, f, ms_k, cnt_k, gemm_flops, dgemm, solve_graph_ms, spmv_ms, R, hbm):
    """Achieved rate and fraction of peak for every kernel class of the step, from algorithmic
    work over CUDA-event times: the FP64 update GEMM (flops, against cuBLAS DGEMM measured in the
    run), the front assembly (bytes, HBM), the triangular solve of R right-hand sides (bytes and
    flops; timed alone, graph replay), the residual SpMV (bytes, HBM)."""
    hbm_gbs, hbm_src = hbm
    entries = float(f.entries())
    n, nnz = p.n, float(p.csr.idx.size)
    asm_b = assembly_bytes(f)
    asm_ms = float(ms_k[0])
    solve_b = 2 * entries * 8 + 2 * n * R * 8
    solve_fl = 4 * entries * R
    spmv_b = (nnz * 12 + (n + 1) * 8 + 2 * n * 8) * R
    out = {
        "gemm": {"bound": "tensor", "achieved": gemm_flops / (ms_k[3] * 1e-3) / 1e12, "peak": dgemm,
                 "unit": "TFLOP/s", "ms": float(ms_k[3]), "launches": int(cnt_k[3])},
        "assemble": {"bound": "hbm", "achieved": asm_b / (asm_ms * 1e-3) / 1e9, "peak": hbm_gbs, "unit": "GB/s",
                     "bytes": asm_b, "ms": asm_ms, "launches": int(cnt_k[0]),
                     "algorithmic": "8 B per value of A, per child update entry read, per front entry written"},
        "solve": {"bound": "tensor", "achieved": solve_fl / (solve_graph_ms * 1e-3) / 1e12, "peak": dgemm,
                  "unit": "TFLOP/s", "ms": solve_graph_ms, "gbs": solve_b / (solve_graph_ms * 1e-3) / 1e9,
                  "gbs_frac": solve_b / (solve_graph_ms * 1e-3) / 1e9 / hbm_gbs,
                  "algorithmic": f"4 |L| R flops; 2 |L| 8 + 2 n R 8 bytes (R = {R}); timed alone"},
        "spmv": {"bound": "hbm", "achieved": spmv_b / (spmv_ms * 1e-3) / 1e9, "peak": hbm_gbs, "unit": "GB/s",
                 "ms": spmv_ms, "algorithmic": "(12 nnz + 8 (n+1) + 16 n) bytes per right-hand side"},
        "panel": {"bound": "latency", "ms": float(ms_k[1]), "launches": int(cnt_k[1])},
        "hbm_peak_source": hbm_src,
    }
    for k in ("gemm", "assemble", "solve", "spmv"):
        out[k]["frac"] = out[k]["achieved"] / out[k]["peak"]
    return out


def profile_kernels(args, torch, lib):
    """Runs for a profiler (no timing): the FP32 factorisation of the --n-el block twice (the
    tcgen05 update GEMMs), or the U-Net's forward and backward passes twice."""
    from fieldcraft_b200 import FP32_IR, Factor, Symbolic, problems
    if args.profile_kernels == "fp32-factor":
        p = problems.lognormal_block(args.n_el, nrhs=1, seed=SEED)
        up = p.upper()
        f = Factor(Symbolic(up, 2**62), precision=FP32_IR)
        d_val = torch.from_numpy(up.val).cuda()
        for _ in range(2):
            assert lib.fc_chol_factor_device_async(f.handle, C.c_void_p(d_val.data_ptr()), up.val.size) == 0
        torch.cuda.synchronize()
        f.close()
        print(json.dumps({"profile_kernels": "fp32-factor", "n": p.n}), flush=True)
    else:
        from fieldcraft_b200.unet import UNet
        p = problems.plate(64, 64, 8, nrhs=1)
        net = UNet(p, seed=0, kref=100.0)
        x = torch.randn(net.voxels * 16, device="cuda", dtype=torch.float32)
        y = torch.empty_like(x)
        for _ in range(2):
            net.forward_grid(x, y)
            net.backward_grid(x)
        torch.cuda.synchronize()
        net.close()
        print(json.dumps({"profile_kernels": "unet", "voxels": net.voxels}), flush=True)


def main():
    args = parse()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank, world)
        return
    import torch
    import torch.distributed as dist
    from fieldcraft_b200 import Factor, Symbolic, _lib, problems
    from fieldcraft_b200.cholesky import Status, raise_for

    torch.cuda.set_device(local)
    if world > 1:
        dist.init_process_group("nccl", init_method="env://", timeout=__import__("datetime").timedelta(seconds=600))
    lib = _lib.load()
    if args.profile_kernels:
        profile_kernels(args, torch, lib)
        return
    if args.assembly:
        if rank == 0:
            run_assembly(args, torch, lib, local)
        if world > 1:
            dist.destroy_process_group()
        return
    if args.ldlt:
        if rank == 0:
            run_ldlt(args, torch, lib, local)
        if world > 1:
            dist.destroy_process_group()
        return
    if args.config == 3 and world > 1:
        run_batch_sharded(args, torch, rank, world, local)
        dist.destroy_process_group()
        return
    if args.config != 2:
        if rank == 0:
            run_config(args, args.config, torch, lib, local)
        if world > 1:
            dist.destroy_process_group()
        return
    p = problems.lognormal_block(args.n_el, nrhs=args.nrhs, seed=SEED + rank)
    up = p.upper()
    full_flops, entries = factor_flops(p)
    sym = Symbolic(up, 2**62)
    f = Factor(sym, device=local)
    stream = torch.cuda.Stream()
    f.set_stream(stream.cuda_stream)
    n, R = p.n, args.nrhs
    d_val = torch.from_numpy(up.val).cuda()
    d_ptr = torch.from_numpy(p.csr.ptr).cuda()
    d_idx = torch.from_numpy(p.csr.idx).cuda()
    d_kv = torch.from_numpy(p.csr.val).cuda()
    d_f = torch.from_numpy(np.ascontiguousarray(p.rhs.T)).cuda()  # [R, n]: column j of the n x R block
    d_x = torch.empty_like(d_f)
    d_r = torch.empty_like(d_f)
    fnorm = torch.linalg.vector_norm(d_f, dim=1)
    st = Status()

    def step():
        with torch.cuda.stream(stream):
            rc = lib.fc_chol_factor_device_async(f.handle, C.c_void_p(d_val.data_ptr()), up.val.size)
            assert rc == 0
            d_x.copy_(d_f)
            rc = lib.fc_chol_solve_device_async(f.handle, C.c_void_p(d_x.data_ptr()), R, n)
            assert rc == 0
            lib.fc_csr_spmv_device(n, C.c_void_p(d_ptr.data_ptr()), C.c_void_p(d_idx.data_ptr()),
                                   C.c_void_p(d_kv.data_ptr()), C.c_void_p(d_x.data_ptr()),
                                   C.c_void_p(d_r.data_ptr()), R, n, C.c_void_p(stream.cuda_stream))
            d_r.sub_(d_f)
            return torch.linalg.vector_norm(d_r, dim=1) / fnorm

    if args.profile_only:
        # the launch counts per step (for choosing which launches a profiler captures), then the
        # warm-up steps and nothing else
        kinds = 32
        ms_k = np.zeros(kinds)
        cnt_k = np.zeros(kinds, np.int64)
        lib.fc_chol_profile(f.handle, 1)
        relres = step()
        lib.fc_chol_profile_read(f.handle, ms_k.ctypes.data, cnt_k.ctypes.data, kinds)
        lib.fc_chol_profile(f.handle, 0)
        for _ in range(args.warmup):
            relres = step()
        stream.synchronize()
        lib.fc_chol_check(f.handle, C.byref(st))
        raise_for(st)
        if rank == 0:
            print(json.dumps({"profile_only": True, "n": n, "gemm_factor_launches": int(cnt_k[3]),
                              "gemm_big_ordinal": f.stat(11), "gemm_trail_ordinal": f.stat(12),
                              "gemm_solve_launches": int(cnt_k[19]), "panel_launches": int(cnt_k[1]),
                              "gemm_useful_flops_factor": f.stat(9) + f.stat(10),
                              "relres_max": float(relres.max().item())}), flush=True)
        f.close()
        if world > 1:
            dist.destroy_process_group()
        return
    for _ in range(args.warmup):
        relres = step()
    stream.synchronize()
    lib.fc_chol_check(f.handle, C.byref(st))
    raise_for(st)
    launches_per_step = f.stat(7) + f.stat(8) + 1
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with Clocks(local) as clk:
        e0.record(stream)
        for _ in range(args.steps):
            relres = step()
        e1.record(stream)
        e1.synchronize()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / args.steps
    lib.fc_chol_check(f.handle, C.byref(st))
    raise_for(st)
    worst = float(relres.max().item())
    x64_host = d_x.cpu().numpy().T.copy()  # the timed steps' FP64 solutions, n x R
    if world > 1:
        t = torch.tensor([ms], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
        dist.barrier()
    clocks = clk.summary()
    if rank != 0:
        if world > 1:
            dist.destroy_process_group()
        return

    # per-kernel times on the same stream (events around every launch), one profiled step
    kinds = 32
    ms_k = np.zeros(kinds)
    cnt_k = np.zeros(kinds, np.int64)
    lib.fc_chol_profile(f.handle, 1)
    step()
    lib.fc_chol_profile_read(f.handle, ms_k.ctypes.data, cnt_k.ctypes.data, kinds)
    lib.fc_chol_profile(f.handle, 0)
    gemm_ms = ms_k[3]
    gemm_flops = float(f.stat(15))  # the update GEMM launches' tasks alone (profile kind 3)
    peak = dgemm_peak(torch)
    achieved = gemm_flops / (gemm_ms * 1e-3) / 1e12
    factor_ms = float(ms_k[0:4].sum() + ms_k[10:13].sum() + ms_k[15])
    solve_ms = float(ms_k[16:32].sum())
    traffic, traffic_note = recorded_traffic("gemm_kernel", gemm_flops / max(1, int(cnt_k[3])))
    # the solve and the residual product alone, on the same stream (graph replay, CUDA events)
    solve_graph_ms = stream_time(torch, stream, lambda: solve_only(lib, f, d_x, d_f, R, n, stream), reps=5)
    spmv_ms = stream_time(torch, stream, lambda: lib.fc_csr_spmv_device(
        n, C.c_void_p(d_ptr.data_ptr()), C.c_void_p(d_idx.data_ptr()), C.c_void_p(d_kv.data_ptr()),
        C.c_void_p(d_x.data_ptr()), C.c_void_p(d_r.data_ptr()), R, n, C.c_void_p(stream.cuda_stream)), reps=5)
    kernel_roofline = roofline_table(p, f, ms_k, cnt_k, gemm_flops, peak, solve_graph_ms, spmv_ms, R, hbm_peak())

    # end to end through the public API with pinned host buffers
    hv = torch.from_numpy(up.val).pin_memory()
    hb = torch.from_numpy(np.asfortranarray(p.rhs).T.copy()).pin_memory()  # [R, n] contiguous = column-major n x R
    hx = torch.empty_like(hb).pin_memory()
    e2e = []
    for it in range(2 + args.steps):
        hx.copy_(hb)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        rc = lib.fc_chol_factor(f.handle, C.c_void_p(hv.data_ptr()), up.val.size, None, C.byref(st))
        raise_for(st)
        rc = lib.fc_chol_solve(f.handle, C.c_void_p(hx.data_ptr()), R, n, C.byref(st))
        raise_for(st)
        t1 = time.perf_counter()
        if it >= 2:
            e2e.append(t1 - t0)
    e2e_s = float(np.mean(e2e))
    xr = hx.numpy()
    rr = np.stack([np.linalg.norm(p.rhs[:, j]) for j in range(R)])
    # residual of the e2e result on the device (the same SpMV)
    d_x.copy_(hx.cuda())
    lib.fc_csr_spmv_device(n, C.c_void_p(d_ptr.data_ptr()), C.c_void_p(d_idx.data_ptr()), C.c_void_p(d_kv.data_ptr()),
                           C.c_void_p(d_x.data_ptr()), C.c_void_p(d_r.data_ptr()), R, n, None)
    torch.cuda.synchronize()
    e2e_res = float(((d_r - d_f).norm(dim=1) / fnorm).max().item())

    stats = {"supernodes": f.stat(4), "levels": f.stat(0), "l_bytes": f.stat(2)}
    # the learned preconditioner: on a plate with on-policy training (nn_plate_block), or on the
    # same K (a short training; see nn_fcg_block)
    nn = None
    if not args.no_nn and args.nn_plate:
        f.set_stream(None)
        nn = nn_plate_block(args.nn_plate, torch, lib)
        f.set_stream(stream.cuda_stream)
    elif not args.no_nn:
        b1 = d_f[0:1].clone()
        tt = []
        for it in range(3):
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            with torch.cuda.stream(stream):
                lib.fc_chol_factor_device_async(f.handle, C.c_void_p(d_val.data_ptr()), up.val.size)
                lib.fc_chol_solve_device_async(f.handle, C.c_void_p(b1.data_ptr()), 1, n)
            e1.record(stream)
            e1.synchronize()
            tt.append(e0.elapsed_time(e1))
        f.set_stream(None)
        nn = nn_fcg_block(p, f, (d_ptr, d_idx, d_kv), torch, pairs=args.nn_pairs, epochs=args.nn_epochs, cols=[0],
                          cap=1500, chol_ms=float(np.min(tt[1:])))
        f.set_stream(stream.cuda_stream)
    # FP32 (3xTF32) factorisation of S A S + FP64 refinement to the same rel-res, same system
    fp32 = None
    if not args.no_fp32:
        from fieldcraft_b200 import FP32_IR
        f.close()
        torch.cuda.empty_cache()
        g32 = Factor(sym, precision=FP32_IR, device=local)
        g32.set_stream(stream.cuda_stream)
        csr_dev = (d_ptr, d_idx, d_kv)
        x32 = torch.zeros_like(d_f)
        times, its, rels = [], [], []
        for it in range(2 + args.steps):
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            rc = lib.fc_chol_factor_device_async(g32.handle, C.c_void_p(d_val.data_ptr()), up.val.size)
            assert rc == 0
            rel, nit = g32.refine_solve_device(csr_dev, d_f, x32, R, n, tol=1e-10, max_iter=30)
            e1.record(stream)
            e1.synchronize()
            if it >= 2:
                times.append(e0.elapsed_time(e1))
                its.append(nit)
                rels.append(float(np.max(rel)))
        lib.fc_chol_check(g32.handle, C.byref(st))
        raise_for(st)
        x32_host = x32.cpu().numpy().T.copy()
        fp32 = {"value": float(np.mean(times)) / 1e3, "unit": UNIT, "refinement_solves": int(max(its)),
                "relres_max": max(rels), "speedup_vs_fp64": (ms / 1e3) / (float(np.mean(times)) / 1e3),
                "what": "FP32 factor of S A S (3xTF32 updates on the tensor pipe, FP64 diagonal blocks) + FP64 "
                        "iterative refinement to rel-res 1e-10 for every right-hand side"}
        g32.close()
    cb = None
    err_oracle = {}
    if not args.no_cpu_baseline:
        # the oracle on the whole workload, once, from its own builder (bit for bit this K and f):
        # the CPU reference's time, and the oracle's solutions for every right-hand side's error
        from oracle import workloads
        owl = workloads.lognormal_block(args.n_el, nrhs=R, seed=SEED + rank)
        same_input = same_system(owl, p.csr, p.rhs)
        threads = os.cpu_count() or 1
        r = oracle_full_run(owl, threads, 0.0, max_runs=1)
        xo = r["x"]
        cb = {"value": r["factor_s"][0] + r["solve_s"][0], "unit": UNIT, "cores": threads, "kind": "port",
              "cpu_model": cpu_model(),
              "sample": f"the whole workload once (built by the oracle's own builder, bit for bit this K and f: "
                        f"{same_input}): numeric factorisation {r['factor_s'][0]:.2f} s on {threads} threads + "
                        f"solve of {R} RHS {r['solve_s'][0]:.2f} s (sequential groups of 6, as the reference); "
                        f"analysis {r['symbolic_s']:.2f} s untimed"}
        err_oracle["fp64"] = per_rhs_error(x64_host, xo)
        if fp32 is not None:
            err_oracle["fp32_ir"] = per_rhs_error(x32_host, xo)
            fp32["err_vs_oracle_per_rhs"] = [float(v) for v in err_oracle["fp32_ir"]]
            fp32["err_vs_oracle_max"] = float(np.max(err_oracle["fp32_ir"]))
        del xo, owl
    line = {
        "metric": METRIC, "value": ms / 1e3, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": False, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded lognormal E, Gaussian loads)",
        "config": {"workload": f"FP64 direct solve, hex8 block {args.n_el}^3 lognormal E (sigma 0.5), z=0 clamped, "
                               f"{R} Gaussian top-face RHS", "n": n, "nnz": int(p.csr.idx.size), "nrhs": R,
                   "factor_entries": entries, "factor_flops": full_flops, "supernodes": stats["supernodes"],
                   "levels": stats["levels"], "l2": "inputs larger than L2 (L alone is %.1f GB)" % (stats["l_bytes"] / 1e9),
                   "parallelism": f"replicas x{world}" if world > 1 else "1 GPU"},
        "relres_max": worst, "relres_target": 1e-10, "solved": worst <= 1e-10,
        "err_vs_oracle_per_rhs": [float(v) for v in err_oracle["fp64"]] if "fp64" in err_oracle else None,
        "err_vs_oracle_max": float(np.max(err_oracle["fp64"])) if "fp64" in err_oracle else None,
        "factor_tflops": full_flops / (factor_ms * 1e-3) / 1e12 if factor_ms > 0 else None,
        "phase_ms": {"factor": factor_ms, "solve": solve_ms,
                     "by_kernel": {name: round(float(ms_k[k]), 3) for k, name in KERNEL_KINDS},
                     "launches": {name: int(cnt_k[k]) for k, name in KERNEL_KINDS}},
        "roofline": {"kernel": "gemm_kernel (FP64 DMMA, factor updates)", "bound": "tensor",
                     "achieved": achieved, "peak": peak, "unit": "TFLOP/s", "frac": achieved / peak,
                     "traffic": traffic, "traffic_source": traffic_note,
                     "peak_source": "cuBLAS DGEMM 8192^3 measured in this run (MEASURED_PEAKS.json has no FP64 "
                                    "figure)",
                     "algorithmic": "useful flops of the factor's GEMM tasks (2 K per lower-triangle output)",
                     "flops_per_step": gemm_flops, "ms_per_step": float(gemm_ms), "launches": int(cnt_k[3]),
                     "kernels": kernel_roofline},
        "e2e": {"value": e2e_s, "unit": UNIT, "h2d_bytes_per_step": int(up.val.nbytes + hb.numel() * 8),
                "d2h_bytes_per_step": int(hx.numel() * 8 + 32), "relres_max": e2e_res},
        "gpu_launches": int(launches_per_step * args.steps),
        "clocks": clocks,
    }
    if cb is not None:
        line["cpu_baseline"] = cb
    if fp32 is not None:
        line["fp32_ir"] = fp32
    if nn is not None:
        line["nn_fcg"] = nn
    print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()

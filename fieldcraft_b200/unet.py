"""The learned preconditioner and flexible CG (include/fieldcraft_unet.h), for the same K u = f the
Cholesky factor solves. No reference counterpart: the reference is a direct solver only
(docs/linear-solvers.md:375-376). The Cholesky factor produces the training pairs (r, K^-1 r), is
the fallback when FCG does not converge, and the reference against which FCG's error is measured.

Device arrays are CUDA tensors (torch is only the allocator here); the network's forward and
backward passes, Adam and FCG run on this library's kernels."""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from .cholesky import Factor, Status, raise_for
from .problems import Problem, node_feature


def _p(t) -> C.c_void_p:
    return C.c_void_p(t.data_ptr())


class UNet:
    """The 32-channel 3D-convolution U-Net on the node grid of a box problem (`levels` levels, 3 by
    default). With `operator` = (ptr, idx, val) CUDA tensors of K, the preconditioner is the nodal
    block-Jacobi inverse of K plus the network, which then learns the rest of K^-1 r."""

    def __init__(self, problem: Problem, seed: int = 0, device: int = 0, kref: float | None = None, levels: int = 3,
                 operator=None):
        lib = _lib.load()
        nx, ny, nz = problem.dims
        if kref is None:
            csr = problem.csr
            rows = np.repeat(np.arange(csr.n), np.diff(csr.ptr))
            kref = float(np.mean(csr.val[csr.idx == rows]))
        self.kref = float(kref)
        eq = np.ascontiguousarray(problem.eq, np.int64)
        feat = node_feature(problem)
        st = Status()
        h = C.c_void_p()
        lib.fc_unet_create_levels(nx, ny, nz, problem.n, _lib.ptr(eq), _lib.ptr(feat), self.kref, int(levels), seed,
                                  device, C.byref(h), C.byref(st))
        raise_for(st)
        self.handle = h
        self.n = problem.n
        self.levels = int(levels)
        self.voxels = (nx + 1) * (ny + 1) * (nz + 1)
        if operator is not None:
            self.set_operator(operator)

    def set_operator(self, csr_device):
        """Adds the nodal block-Jacobi part of K (CUDA tensors ptr, idx, val) to the preconditioner;
        None removes it."""
        args = [_p(a) for a in csr_device] if csr_device is not None else [None, None, None]
        rc = _lib.load().fc_unet_set_operator(self.handle, *args)
        if rc != 0:
            raise ValueError(f"fc_unet_set_operator ({rc})")

    def enable(self, on, safeguard: bool = True):
        """False: the preconditioner is the block-Jacobi part alone (the network is not run);
        True: B r + net(r), FCG's safeguard on unless `safeguard` is False."""
        code = 0 if not on else (1 if safeguard else 2)
        if _lib.load().fc_unet_enable(self.handle, code) != 0:
            raise ValueError("fc_unet_enable needs the operator set")

    def set_odd(self, odd: bool):
        """True (the default): the network part of M is (net(r) - net(-r)) / 2 (M odd in r)."""
        if _lib.load().fc_unet_set_odd(self.handle, int(bool(odd))) != 0:
            raise ValueError("fc_unet_set_odd")

    def stat(self, what: int) -> int:
        """0 levels, 1 iterations of the last FCG with the network, 2 whether its safeguard dropped
        the network, 3 whether the block-Jacobi part is set."""
        return int(_lib.load().fc_unet_stat(self.handle, int(what)))

    def set_stream(self, stream_ptr: int | None):
        _lib.load().fc_unet_set_stream(self.handle, C.c_void_p(stream_ptr) if stream_ptr else None)

    def param_count(self) -> int:
        return int(_lib.load().fc_unet_param_count(self.handle))

    def params(self) -> np.ndarray:
        out = np.empty(self.param_count(), np.float32)
        if _lib.load().fc_unet_get_params(self.handle, _lib.ptr(out)) != 0:
            raise RuntimeError("fc_unet_get_params")
        return out

    def set_params(self, flat: np.ndarray):
        v = np.ascontiguousarray(flat, np.float32)
        if v.size != self.param_count() or _lib.load().fc_unet_set_params(self.handle, _lib.ptr(v)) != 0:
            raise ValueError("parameter vector")

    def grads(self) -> np.ndarray:
        out = np.empty(self.param_count(), np.float32)
        if _lib.load().fc_unet_get_grads(self.handle, _lib.ptr(out)) != 0:
            raise RuntimeError("fc_unet_get_grads")
        return out

    def forward_grid(self, x, y):
        """y = net(x) on device FP32 grids [voxels, 16]."""
        if _lib.load().fc_unet_forward_grid(self.handle, _p(x), _p(y)) != 0:
            raise RuntimeError("fc_unet_forward_grid")

    def backward_grid(self, dy):
        if _lib.load().fc_unet_backward_grid(self.handle, _p(dy)) != 0:
            raise RuntimeError("fc_unet_backward_grid")

    def apply(self, r, z):
        """z = M(r) for device FP64 equation vectors."""
        if _lib.load().fc_unet_apply(self.handle, _p(r), _p(z)) != 0:
            raise RuntimeError("fc_unet_apply")

    def train_step(self, r, e, lr: float, step: int, loss=None, csr_device=None):
        """One Adam step on the pair (r, e = K^-1 r); with csr_device = (ptr, idx, val) of K the loss
        is the energy norm of the error, else its Euclidean norm (both relative)."""
        k = [_p(a) for a in csr_device] if csr_device is not None else [None, None, None]
        if _lib.load().fc_unet_train_step(self.handle, _p(r), _p(e), *k, C.c_float(lr), int(step),
                                          _p(loss) if loss is not None else None) != 0:
            raise RuntimeError("fc_unet_train_step")

    def train_batch(self, R, E, lr: float, step: int, loss=None, csr_device=None):
        """One Adam step on the mean gradient of the pairs (rows of R, rows of E: CUDA tensors
        [count, n]); `loss` (a device double) gets the sum of their losses."""
        k = [_p(a) for a in csr_device] if csr_device is not None else [None, None, None]
        rc = _lib.load().fc_unet_train_batch(self.handle, _p(R), _p(E), int(R.shape[0]), int(R.stride(0)), *k,
                                             C.c_float(lr), int(step), _p(loss) if loss is not None else None)
        if rc != 0:
            raise RuntimeError("fc_unet_train_batch")

    def close(self):
        h = getattr(self, "handle", None)
        if h:
            try:
                _lib.load().fc_unet_destroy(h)
            except TypeError:
                pass
            self.handle = None

    def __del__(self):
        self.close()


def fcg(csr_device, b, x, net: UNet | None = None, fallback: Factor | None = None, tol: float = 1e-10,
        max_iter: int = 1000, keep: int = 4):
    """Flexible CG on K x = b (device FP64 vectors; csr_device = (ptr, idx, val) CUDA tensors),
    preconditioned by `net` (None: plain CG), with the Cholesky `fallback`. Returns (iterations,
    relative residual, used_fallback); raises Timeout when neither reached tol."""
    ptr, idx, val = csr_device
    it, rel, fb = C.c_int32(0), C.c_double(0.0), C.c_int32(0)
    st = Status()
    _lib.load().fc_fcg_solve(net.handle if net else None, fallback.handle if fallback else None, int(b.numel()),
                             _p(ptr), _p(idx), _p(val), _p(b), _p(x), float(tol), int(max_iter), int(keep),
                             C.byref(it), C.byref(rel), C.byref(fb), C.byref(st))
    raise_for(st)
    return it.value, rel.value, bool(fb.value)


def training_pairs(factor: Factor, problem: Problem, count: int, seed: int, torch, block: int = 64):
    """`count` pairs (r, K^-1 r) from the Cholesky solve: half white-noise residuals, half random
    top-face pressures, each r of unit norm. Returns two CUDA tensors [count, n] (FP64)."""
    from .problems import top_pressures
    n = problem.n
    g = torch.Generator(device="cuda")
    g.manual_seed(seed)
    R = torch.empty((count, n), dtype=torch.float64, device="cuda")
    half = count // 2
    R[:half] = torch.randn((half, n), dtype=torch.float64, device="cuda", generator=g)
    R[half:] = torch.from_numpy(np.ascontiguousarray(top_pressures(problem, count - half, seed + 7).T)).cuda()
    R /= torch.linalg.vector_norm(R, dim=1, keepdim=True)
    E = R.clone()
    for s in range(0, count, block):
        e = min(count, s + block)
        factor.solve_device(E[s:e], e - s, n)  # rows of E are column-major right-hand sides
    torch.cuda.synchronize()
    return R, E


def block_jacobi(problem: Problem, torch):
    """The inverses of K's nodal 3 x 3 diagonal blocks (equations node by node, three a node), as a
    CUDA tensor [n / 3, 3, 3]."""
    csr = problem.csr
    n = csr.n
    rows = np.repeat(np.arange(n), np.diff(csr.ptr))
    keep = (csr.idx // 3) == (rows // 3)
    blocks = np.zeros((n // 3, 3, 3))
    blocks[rows[keep] // 3, rows[keep] % 3, csr.idx[keep] % 3] = csr.val[keep]
    return torch.from_numpy(np.linalg.inv(blocks)).cuda()


def krylov_pairs(factor: Factor, problem: Problem, csr_device, count: int, seed: int, torch,
                 snapshots=(0, 2, 5, 10, 20, 40, 80, 160), block: int = 32):
    """`count` pairs (r, K^-1 r) whose r are the residuals that block-Jacobi preconditioned CG
    leaves on random right-hand sides (random top-face pressures and white noise, half each) at the
    iterations `snapshots`: the inputs a preconditioner meets inside the Krylov solve, in which
    the smooth, slowly converging parts dominate more and more. Each r is scaled to unit norm; e =
    K^-1 r from the Cholesky solve. Returns two CUDA tensors [count, n] (FP64)."""
    from .problems import top_pressures
    lib = _lib.load()
    n = problem.n
    per = len(snapshots)
    rhs_count = (count + per - 1) // per
    g = torch.Generator(device="cuda")
    g.manual_seed(seed)
    Binv = block_jacobi(problem, torch)
    ptr, idx, val = csr_device
    out = torch.empty((rhs_count * per, n), dtype=torch.float64, device="cuda")
    at = 0
    for b0 in range(0, rhs_count, block):
        k = min(block, rhs_count - b0)
        half = k // 2
        B = torch.empty((k, n), dtype=torch.float64, device="cuda")
        B[:half] = torch.randn((half, n), dtype=torch.float64, device="cuda", generator=g)
        B[half:] = torch.from_numpy(np.ascontiguousarray(top_pressures(problem, k - half, seed + 31 + b0).T)).cuda()
        X = torch.zeros_like(B)
        Rr = B.clone()
        prec = lambda r: torch.einsum("kab,jkb->jka", Binv, r.view(r.shape[0], n // 3, 3)).reshape(r.shape)  # noqa
        Z = prec(Rr)
        P = Z.clone()
        rz = (Rr * Z).sum(dim=1)
        Q = torch.empty_like(B)
        for it in range(max(snapshots) + 1):
            if it in snapshots:
                out[at:at + k] = Rr / torch.linalg.vector_norm(Rr, dim=1, keepdim=True)
                at += k
            if it == max(snapshots):
                break
            lib.fc_csr_spmv_device(n, C.c_void_p(ptr.data_ptr()), C.c_void_p(idx.data_ptr()),
                                   C.c_void_p(val.data_ptr()), C.c_void_p(P.data_ptr()), C.c_void_p(Q.data_ptr()), k,
                                   n, None)
            alpha = rz / (P * Q).sum(dim=1)
            X += alpha[:, None] * P
            Rr -= alpha[:, None] * Q
            Z = prec(Rr)
            rz_new = (Rr * Z).sum(dim=1)
            P = Z + (rz_new / rz)[:, None] * P
            rz = rz_new
    R = out[:count].contiguous()
    E = R.clone()
    for s in range(0, count, 64):
        e = min(count, s + 64)
        factor.solve_device(E[s:e], e - s, n)
    torch.cuda.synchronize()
    return R, E


def policy_pairs(net: UNet, factor: Factor, problem: Problem, csr_device, nrhs: int, seed: int, torch,
                 snapshots=(1, 2, 3, 5, 8, 12, 20, 30, 45)):
    """Pairs (r, K^-1 r) whose r are the residuals that conjugate gradients preconditioned by the
    network's current M (block Jacobi plus the network) leaves at the iterations `snapshots` on
    `nrhs` random top-face pressures: the inputs the network meets inside its own Krylov solve,
    which change as it learns. Each r of unit norm; e from the Cholesky solve. Returns two CUDA
    tensors [nrhs * len(snapshots), n] (FP64)."""
    from .problems import top_pressures
    lib = _lib.load()
    n = problem.n
    ptr, idx, val = csr_device
    B = torch.from_numpy(np.ascontiguousarray(top_pressures(problem, nrhs, seed).T)).cuda()
    rec = []
    z = torch.empty(n, dtype=torch.float64, device="cuda")
    q = torch.empty_like(z)
    for j in range(nrhs):
        r = B[j].clone()
        net.apply(r, z)
        d = z.clone()
        rz = float(r @ z)
        for it in range(1, max(snapshots) + 1):
            lib.fc_csr_spmv_device(n, _p(ptr), _p(idx), _p(val), _p(d), _p(q), 1, n, None)
            r -= (rz / float(d @ q)) * q
            if it in snapshots:
                rec.append(r / torch.linalg.vector_norm(r))
            net.apply(r, z)
            rz_new = float(r @ z)
            d = z + (rz_new / rz) * d
            rz = rz_new
    R = torch.stack(rec)
    E = R.clone()
    for s in range(0, R.shape[0], 64):
        e = min(R.shape[0], s + 64)
        factor.solve_device(E[s:e], e - s, n)
    torch.cuda.synchronize()
    return R, E


def train_on_policy(net: UNet, factor: Factor, problem: Problem, csr_device, R, E, rounds: int, nrhs: int,
                    epochs: int, lr: float, torch, batch: int = 16, seed: int = 0):
    """`rounds` rounds of: pairs from the network's own Krylov residuals (policy_pairs) added to the
    training set (R, E), then `epochs` passes over the whole set. A network trained on the
    Cholesky pairs alone can make flexible CG diverge on the residuals it meets after a few
    iterations; these rounds teach it those. Returns (R, E, each round's last-epoch loss)."""
    losses = []
    for rd in range(rounds):
        Rn, En = policy_pairs(net, factor, problem, csr_device, nrhs, seed + 100 + rd, torch)
        R = torch.cat([R, Rn])
        E = torch.cat([E, En])
        losses.append(train(net, R, E, epochs=epochs, lr=lr, torch=torch, csr_device=csr_device, batch=batch,
                            warmup=20, seed=seed + 1 + rd)[-1])
    return R, E, losses


def output_scale(R, E) -> float:
    """The network's output scale for pairs (r, K^-1 r): the median of ||r|| / ||e||, so that the
    network's outputs are of order one."""
    import torch
    return float(torch.median(torch.linalg.vector_norm(R, dim=1) / torch.linalg.vector_norm(E, dim=1)).item())


def train(net: UNet, R, E, epochs: int, lr: float, torch, seed: int = 0, lr_decay: float = 0.3, csr_device=None,
          warmup: int = 200, batch: int = 1):
    """Adam over the pairs for `epochs` passes in a seeded order, `batch` pairs per step (their
    mean gradient); the learning rate ramps up over the first `warmup` steps and steps down by
    lr_decay for the last epoch. Returns the mean loss of each epoch."""
    loss = torch.zeros(1, dtype=torch.float64, device="cuda")
    losses = []
    rng = np.random.default_rng(seed)
    step = 0
    count = R.shape[0]
    for ep in range(epochs):
        acc = torch.zeros(1, dtype=torch.float64, device="cuda")
        rate = lr * (lr_decay if epochs > 1 and ep == epochs - 1 else 1.0)
        order = rng.permutation(count)
        for b0 in range(0, count, batch):
            step += 1
            pick = order[b0:b0 + batch]
            lr_now = rate * min(1.0, step / warmup)
            if batch == 1:
                net.train_step(R[pick[0]], E[pick[0]], lr_now, step, loss, csr_device)
            else:
                idx = torch.from_numpy(np.ascontiguousarray(pick)).cuda()
                net.train_batch(R.index_select(0, idx), E.index_select(0, idx), lr_now, step, loss, csr_device)
            acc += loss
        losses.append(float(acc.item()) / count)
    return losses

"""Row-partitioned eigsh of one symmetry sector across ranks (one process per GPU).

A sector too large for one device, or solved faster on several, is split into
contiguous slabs of rows (rows follow the sorted representatives). Every rank
keeps its slab of each Lanczos vector. An operator application all-gathers
the input vector into a full-length buffer in the rank's own memory (one
collective over NVLink), then computes its own rows with the matrix-free
slab kernel (qmbed_gpu_operator_apply_rows_device). Inner products are local
partial sums followed by one all-reduce of a few numbers, so every rank sees
bitwise the same projected matrices and takes the same decisions.

The method is thick-restart Lanczos with full classical Gram-Schmidt
reorthogonalisation done twice (Wu and Simon, SIAM J. Matrix Anal. Appl. 22,
2000), the algorithm family of the reference's thick_restarted_eigsh_real
(src/solve/mod.rs:1651-1912): a cycle extends the kept Ritz vectors and the
residual direction to the Krylov dimension, takes the Rayleigh-Ritz pairs of
the projected matrix, and keeps the lowest ones. Every reported pair passes
the reference's acceptance test r <= tol * max(|lambda|, 1)
(src/solve/mod.rs:1252-1263) with r = ||H x - lambda x|| computed by one more
distributed application. The reference itself is single-rank: its runtime
rejects distributed profiles (src/runtime.rs:224-228).

The slab operator is any callable apply(x_full, y_slab); gpu_slab() gives the
one that runs this library's kernel on a GpuOperator with matrix-free
storage. Collectives go through torch.distributed (NCCL between GPUs, gloo on
CPU), with the process group passed in or the default one.
"""

from __future__ import annotations

import ctypes
from dataclasses import dataclass

import numpy as np


@dataclass
class RowPartition:
    """Contiguous row slabs of equal size `block` (the last may be shorter or empty).

    Rank q owns rows q * block .. q * block + rows(q) - 1, so the all-gather of
    equal-size slabs lays the full vector out in order: the first `dim`
    entries of the gathered buffer are x."""
    dim: int
    world: int

    def __post_init__(self):
        if self.world < 1 or self.dim < 1:
            raise ValueError("a partition needs at least one rank and one row")
        self.block = -(-self.dim // self.world)

    def range(self, rank: int) -> tuple[int, int]:
        row0 = min(rank * self.block, self.dim)
        return row0, min(self.block, self.dim - row0)


def gpu_slab(op, part: RowPartition, rank: int, precision: int = 64):
    """Slab action y_slab = (H x)[rows of `rank`] on device tensors through the
    library's matrix-free kernel (the operator must use matrix-free storage)."""
    import torch
    from ._lib import check, lib

    from .engine import _device_operands

    row0, rows = part.range(rank)
    scalar = 8 if precision == 64 else 4

    def apply(x_full, y_slab):
        _device_operands(("the gathered vector", x_full, part.dim * scalar), ("the slab output", y_slab, rows * scalar),
                         device=getattr(getattr(op, "basis", None), "device", None))
        stream = torch.cuda.current_stream(x_full.device).cuda_stream
        check(lib().qmbed_gpu_operator_apply_rows_device(op.handle, precision, row0, rows,
                                                         ctypes.c_void_p(x_full.data_ptr()),
                                                         ctypes.c_void_p(y_slab.data_ptr()),
                                                         ctypes.c_void_p(stream)))
    return apply


@dataclass
class DistributedEigsh:
    eigenvalues: np.ndarray
    residuals: np.ndarray
    vectors: object        # slab of the eigenvectors on this rank (rows x eigenpairs) or None
    applications: int      # operator applications (every rank applies its slab each time)
    restarts: int
    converged: bool


class _Comm:
    def __init__(self, group):
        import torch.distributed as dist
        self.dist = dist
        self.group = group
        self.active = dist.is_available() and dist.is_initialized()
        self.world = dist.get_world_size(group) if self.active else 1
        self.rank = dist.get_rank(group) if self.active else 0

    def allreduce(self, t):
        if self.active and self.world > 1:
            self.dist.all_reduce(t, group=self.group)
        return t

    def allgather(self, full, slab):
        if self.active and self.world > 1:
            self.dist.all_gather_into_tensor(full, slab, group=self.group)
        else:
            full[: slab.numel()].copy_(slab)


def distributed_eigsh(apply_slab, part: RowPartition, eigenpairs: int, krylov_dimension: int = 40,
                      tolerance: float = 1e-10, max_restarts: int = 1000, start=None, restart_keep: int = 0,
                      group=None, device=None, want_vectors: bool = False) -> DistributedEigsh:
    """Lowest `eigenpairs` eigenvalues of a Hermitian real operator given by slabs.

    apply_slab(x_full, y_slab): this rank's rows of H x (x_full has part.world *
    part.block entries; only the first part.dim are read). start: this rank's
    slab of the start vector (the reference deterministic start of the full
    vector, sliced), or None for a constant vector. restart_keep: Ritz vectors
    kept per restart (at least `eigenpairs`, at most half the Krylov
    dimension)."""
    import torch

    comm = _Comm(group)
    if comm.world != part.world:
        raise ValueError("the partition's rank count differs from the process group's")
    rank = comm.rank
    row0, rows = part.range(rank)
    n, m, k = part.dim, int(krylov_dimension), int(eigenpairs)
    if not 0 < k < m <= n:
        raise ValueError("need 0 < eigenpairs < krylov_dimension <= dimension")
    dev = torch.device(device) if device is not None else torch.device("cpu")
    f64 = torch.float64
    full = torch.zeros(part.world * part.block, dtype=f64, device=dev)
    slab_in = torch.zeros(part.block, dtype=f64, device=dev)
    w = torch.zeros(rows, dtype=f64, device=dev)
    V = torch.zeros((m + 1, rows), dtype=f64, device=dev)   # basis rows: V[j] is vector j's slab
    applications = 0

    def apply(x_slab, out):
        nonlocal applications
        slab_in.zero_()
        slab_in[:rows].copy_(x_slab)
        comm.allgather(full, slab_in)
        apply_slab(full, out)
        applications += 1

    def gdot(a, b):  # global inner products of the rows of a with b
        return comm.allreduce(a @ b)

    def gnorm(x):
        return float(torch.sqrt(comm.allreduce((x * x).sum().reshape(1)))[0])

    v0 = (torch.as_tensor(start, dtype=f64, device=dev).reshape(rows).clone() if start is not None
          else torch.ones(rows, dtype=f64, device=dev))
    norm0 = gnorm(v0)
    if not norm0 > 0.0:
        raise ValueError("start vector has zero norm")
    V[0] = v0 / norm0
    keep_wanted = max(k, min(int(restart_keep), m // 2)) if restart_keep else k
    T = np.zeros((m, m))
    kept = 0            # Ritz vectors carried into this cycle (their T block is diagonal)
    theta_kept = np.zeros(0)
    restarts = 0
    eig = res = None
    converged = False
    while restarts < max_restarts:
        T[:, :] = 0.0
        if kept:
            T[np.arange(kept), np.arange(kept)] = theta_kept
        beta = 0.0
        j = kept
        while j < m:
            apply(V[j], w)
            # two classical Gram-Schmidt passes against every basis vector
            h = gdot(V[: j + 1], w)
            w -= h @ V[: j + 1]
            h2 = gdot(V[: j + 1], w)
            w -= h2 @ V[: j + 1]
            col = (h + h2).cpu().numpy()
            T[: j + 1, j] = col
            T[j, : j + 1] = col
            beta = gnorm(w)
            if not beta > 1e-14 * max(1.0, abs(col[j])):
                m_eff = j + 1
                break
            V[j + 1] = w / beta
            j += 1
        else:
            m_eff = m
        theta, Y = np.linalg.eigh(T[:m_eff, :m_eff])
        estimates = np.abs(beta * Y[m_eff - 1, :k])
        if np.all(estimates <= 0.5 * tolerance * np.maximum(np.abs(theta[:k]), 1.0)) or m_eff < m:
            X = torch.as_tensor(Y[:, :k].T.copy(), dtype=f64, device=dev) @ V[:m_eff]
            residuals = np.zeros(k)
            for i in range(k):
                apply(X[i], w)
                w -= float(theta[i]) * X[i]
                residuals[i] = gnorm(w) / gnorm(X[i])
            eig, res = theta[:k].copy(), residuals
            if np.all(residuals <= tolerance * np.maximum(np.abs(eig), 1.0)):
                converged = True
                vectors = X.T.contiguous() if want_vectors else None
                return DistributedEigsh(eig, res, vectors, applications, restarts, converged)
            if m_eff < m:
                break
        # thick restart: the lowest Ritz vectors, then the residual direction
        kept = min(keep_wanted, m_eff - 1)
        Yk = torch.as_tensor(Y[:, :kept].T.copy(), dtype=f64, device=dev)
        last = V[m_eff].clone()
        V[:kept] = Yk @ V[:m_eff]
        V[kept] = last
        theta_kept = theta[:kept].copy()
        restarts += 1
    return DistributedEigsh(eig if eig is not None else np.full(k, np.nan), res if res is not None else np.full(k, np.inf),
                            None, applications, restarts, False)

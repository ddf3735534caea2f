"""Target-range sharding of the direct KDK step over ranks (one process per GPU).

Mirrors the reference's MPI decomposition (cpp/mpi/distributed_solver.cpp:68-79 ownership
ranges, :114-123 MPI_Allgatherv of the state, cpp/core/main.cpp:240-253 step order): every
rank holds all positions, owns the contiguous target range of ``ownership_range``, kicks
and drifts only its own bodies, and the ranks exchange the drifted positions once per step.
The reference gathers the full 11-double state three times a step; here one all-gather of
the 3 FP64 position components of the owned bodies suffices (masses never change, and
velocities/accelerations are only read by their owner).  The exchange is a
``torch.distributed.all_gather_into_tensor`` (NCCL over NVLink on GPUs, gloo on CPU);
ranges are padded to the largest one so the collective has equal chunks.

The force is injected: on GPUs it is the engine's target-range kernel; the CPU tests pass
a CPU function and a gloo group.
"""
from __future__ import annotations

from typing import Callable

import torch
import torch.distributed as dist


def ownership_range(count: int, rank: int, size: int) -> tuple[int, int]:
    """ownership_for_rank (cpp/mpi/distributed_solver.cpp:68-79)."""
    if size <= 1:
        return 0, count
    base, rem = divmod(count, size)
    begin = rank * base + min(rank, rem)
    return begin, begin + base + (1 if rank < rem else 0)


def partition_instances(sizes, world: int) -> list[list[int]]:
    """Independent encounters of a batched ensemble over ranks, with no exchange between
    them: instances in decreasing cost (N_b (N_b - 1) pair terms per force evaluation; ties
    by index) each go to the rank with the least cost so far (lowest rank on ties).  Every
    rank computes the same answer.  Returns each rank's instance indices, ascending."""
    sizes = [int(v) for v in sizes]
    order = sorted(range(len(sizes)), key=lambda i: (-sizes[i] * (sizes[i] - 1), i))
    load = [0] * max(1, world)
    parts: list[list[int]] = [[] for _ in range(max(1, world))]
    for i in order:
        r = min(range(len(load)), key=lambda q: (load[q], q))
        load[r] += sizes[i] * (sizes[i] - 1)
        parts[r].append(i)
    return [sorted(q) for q in parts]


def ensemble_shard(offsets, rank: int, world: int):
    """This rank's part of a batched ensemble given as concatenated bodies with instance
    offsets (n_instances + 1): (instance ids, offsets of the rank's sub-batch, body indices
    into the full arrays), from partition_instances."""
    import numpy as np

    off = np.asarray(offsets, dtype=np.int64)
    sizes = np.diff(off)
    ids = np.asarray(partition_instances(sizes, world)[rank] if world > 1 else range(len(sizes)), dtype=np.int64)
    sub = np.zeros(len(ids) + 1, dtype=np.int64)
    sub[1:] = np.cumsum(sizes[ids])
    body = np.concatenate([np.arange(off[i], off[i + 1]) for i in ids]) if len(ids) else np.zeros(0, np.int64)
    return ids, sub, body


# force(X_full (3, n), m (n,), begin, end) -> A_owned (3, end - begin)
ForceFn = Callable[[torch.Tensor, torch.Tensor, int, int], torch.Tensor]


class ShardedLeapfrog:
    def __init__(self, n: int, force: ForceFn, rank: int | None = None, world: int | None = None, group=None):
        self.n = n
        self.force = force
        self.group = group
        self.rank = dist.get_rank(group) if rank is None else rank
        self.world = dist.get_world_size(group) if world is None else world
        self.begin, self.end = ownership_range(n, self.rank, self.world)
        self.chunk = max(ownership_range(n, r, self.world)[1] - ownership_range(n, r, self.world)[0]
                         for r in range(self.world))
        self.ranges = [ownership_range(n, r, self.world) for r in range(self.world)]

    def gather_positions(self, X: torch.Tensor) -> None:
        """All ranks' owned columns of X (3, n) -> everyone's full X, in place."""
        if self.world == 1:
            return
        send = torch.zeros(3, self.chunk, dtype=X.dtype, device=X.device)
        send[:, : self.end - self.begin] = X[:, self.begin:self.end]
        recv = torch.empty(self.world, 3, self.chunk, dtype=X.dtype, device=X.device)
        dist.all_gather_into_tensor(recv, send.unsqueeze(0).contiguous(), group=self.group)
        for r, (b, e) in enumerate(self.ranges):
            X[:, b:e] = recv[r, :, : e - b]

    def initial_accelerations(self, X: torch.Tensor, m: torch.Tensor) -> torch.Tensor:
        return self.force(X, m, self.begin, self.end)

    def step(self, X: torch.Tensor, V: torch.Tensor, A: torch.Tensor, m: torch.Tensor, dt: float) -> None:
        """One KDK step.  X (3, n) full; V, A (3, n_owned) for the owned range; in place."""
        h = 0.5 * dt
        b, e = self.begin, self.end
        V.add_(A * h)
        X[:, b:e] += V * dt
        self.gather_positions(X)
        A.copy_(self.force(X, m, b, e))
        V.add_(A * h)


def direct_force(params, precision=None) -> ForceFn:
    """The engine's direct sum over all bodies for the owned targets (GPU tensors)."""
    from . import _ffi
    from .adjoint import _rows
    prec = _ffi.PRECISION_F64 if precision is None else precision

    def force(X: torch.Tensor, m: torch.Tensor, b: int, e: int) -> torch.Tensor:
        A = torch.empty(3, e - b, dtype=X.dtype, device=X.device)
        _ffi.call("gx_direct_accel_targets", X.shape[1], *_rows(X), m.data_ptr(), b, e, None, 0, params.ffi(),
                  _ffi.precision_code(prec), *_rows(A), torch.cuda.current_stream().cuda_stream)
        return A

    return force


def fmm_force(params, options=None, precision=None) -> ForceFn:
    """The engine's FMM for the owned targets -- the reference's MPI FMM path
    (compute_fmm_accelerations_for_targets, cpp/fmm/fmm_solver.cpp:324-333): every rank builds
    the whole tree and evaluates its own range."""
    from . import _ffi
    from .fmm import FmmOptions, fmm_accelerations
    prec = _ffi.PRECISION_F64 if precision is None else precision
    opt = options or FmmOptions()

    def force(X: torch.Tensor, m: torch.Tensor, b: int, e: int) -> torch.Tensor:
        n = X.shape[1]
        A = torch.zeros(3, n, dtype=X.dtype, device=X.device)
        Xc = X.contiguous()
        fmm_accelerations(Xc[0], Xc[1], Xc[2], m, A[0], A[1], A[2], params, opt, prec, b, e,
                          stream=torch.cuda.current_stream().cuda_stream)
        return A[:, b:e].clone()

    return force

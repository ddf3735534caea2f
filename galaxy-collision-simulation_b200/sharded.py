"""Target-range sharding of the direct KDK step over ranks (one process per GPU).

Mirrors the reference's MPI decomposition (cpp/mpi/distributed_solver.cpp:68-79 ownership
ranges, :114-123 MPI_Allgatherv of the state, cpp/core/main.cpp:240-253 step order): every
rank holds all positions, owns the contiguous target range of ``ownership_range``, kicks
and drifts only its own bodies, and the ranks exchange the drifted positions once per step.
The reference gathers the full 11-double state three times a step; here one all-gather of
the 3 FP64 position components of the owned bodies suffices (masses never change, and
velocities/accelerations are only read by their owner).

``ShardedSession`` keeps each rank's state resident in an engine session and exchanges the
positions in place (see its docstring for the layout); ``ShardedLeapfrog`` is the same step
over torch tensors with an injected force (the FMM force of the reference's MPI FMM path).
Collectives are ``torch.distributed`` (NCCL over NVLink on GPUs, gloo on CPU).
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


class ShardLayout:
    """Padded, rank-major slot order of n bodies over `world` ranks: rank r's owned bodies
    (ownership_range) occupy slots [r * chunk, r * chunk + count_r), chunk = the largest
    count, and the rest of each chunk is padding (zero mass, at the origin)."""

    def __init__(self, n: int, world: int):
        import numpy as np

        self.n, self.world = n, world
        self.ranges = [ownership_range(n, r, world) for r in range(world)]
        self.chunk = max(e - b for b, e in self.ranges) if n else 0
        self.slots = self.chunk * world
        self.body_slot = np.concatenate([np.arange(b, e) - b + r * self.chunk
                                         for r, (b, e) in enumerate(self.ranges)]).astype(np.int64)

    def pad(self, a):
        import numpy as np

        out = np.zeros(self.slots, dtype=np.float64)
        out[self.body_slot] = np.asarray(a, dtype=np.float64)
        return out

    def unpad(self, a):
        import numpy as np

        return np.asarray(a)[self.body_slot].copy()


class ShardedSession:
    """The reference's MPI direct step (cpp/core/main.cpp:240-253) with each rank's state
    resident in an engine session.

    Bodies are held in ShardLayout's padded rank-major slot order.  A padding slot has zero
    mass, so its term in any sum is +-0 -- and a running sum that starts at +0.0 never
    becomes -0.0 in round-to-nearest -- so padded sums equal the unpadded ones bit for bit in
    every arithmetic form, and the real bodies keep their order (the exact form still sums in
    the reference's source order).  Every rank's session holds all slots and owns the first
    count_r slots of its chunk (gx_session_set_targets).  A step is the session's opening half
    (kick and drift of the owned bodies), then one in-place all-gather per position component
    -- each rank's chunk is already where the collective puts it, so NCCL writes straight
    into the arrays the force kernel reads and nothing is copied or scattered -- then the
    closing half (forces on the owned bodies from all slots and the kick).

    `backend` carries the state and the two half steps: ``EngineShard`` on a GPU; tests pass a
    CPU stand-in with the same methods."""

    def __init__(self, n: int, params, backend=None, group=None, rank: int | None = None, world: int | None = None):
        self.n = n
        self.group = group
        self.rank = dist.get_rank(group) if rank is None else rank
        self.world = dist.get_world_size(group) if world is None else world
        self.layout = ShardLayout(n, self.world)
        b, e = self.layout.ranges[self.rank]
        self.begin, self.end = b, e
        self.slot0 = self.rank * self.layout.chunk
        self.backend = backend if backend is not None else EngineShard(self.layout.slots, params)
        self.backend.set_targets(self.slot0, e - b)

    def set_state(self, x, y, z, vx, vy, vz, m, ax=None, ay=None, az=None) -> None:
        L = self.layout
        acc = [ax, ay, az] if ax is not None else [None, None, None]
        self.backend.set_state({k: L.pad(v) for k, v in zip(("x", "y", "z", "vx", "vy", "vz", "m"),
                                                               (x, y, z, vx, vy, vz, m))},
                               None if acc[0] is None else [L.pad(a) for a in acc])

    def compute_accelerations(self, precision=None) -> None:
        self.backend.force_kick(0.0, precision)

    def _exchange(self) -> None:
        if self.world == 1:
            return
        c = self.layout.chunk
        for t in self.backend.position_tensors():
            dist.all_gather_into_tensor(t, self.backend.send_view(t[self.slot0:self.slot0 + c]), group=self.group)

    def step(self, n_steps: int, dt: float, precision=None) -> None:
        h = 0.5 * dt
        for _ in range(int(n_steps)):
            self.backend.kick_drift(h, dt)
            self._exchange()
            self.backend.force_kick(h, precision)

    def get_state(self) -> dict:
        """The whole system's state (unpadded, body order) on every rank: positions are
        already global; velocities and accelerations are gathered from their owners."""
        st = self.backend.state()
        c = self.layout.chunk
        dev = self.backend.position_tensors()[0].device
        out = {k: self.layout.unpad(st[k]) for k in ("x", "y", "z")}
        for k in ("vx", "vy", "vz", "ax", "ay", "az"):
            full = st[k]
            if self.world > 1:
                t = torch.as_tensor(full).to(dev)
                pieces = [torch.empty_like(t[:c]) for _ in range(self.world)]
                dist.all_gather(pieces, t[self.slot0:self.slot0 + c].contiguous(), group=self.group)
                full = torch.cat(pieces).cpu().numpy()
            out[k] = self.layout.unpad(full)
        return out


class _DeviceVector:
    """A device array of the engine seen by torch without a copy (__cuda_array_interface__)."""

    def __init__(self, ptr: int, n: int):
        self.__cuda_array_interface__ = {"shape": (n,), "typestr": "<f8", "data": (int(ptr), False),
                                         "version": 3, "strides": None, "stream": None}


class EngineShard:
    """ShardedSession's backend on a GPU: one engine session over all slots on the current
    device and stream."""

    def __init__(self, slots: int, params, device: int | None = None):
        from .session import Session

        dev = torch.cuda.current_device() if device is None else device
        self.session = Session(slots, params, dev)
        self.session.set_stream(torch.cuda.current_stream(dev))
        ptrs = self.session.device_arrays()
        self._pos = [torch.as_tensor(_DeviceVector(ptrs[k], slots), device=f"cuda:{dev}") for k in ("x", "y", "z")]

    def set_targets(self, begin: int, count: int) -> None:
        self.session.set_targets(begin, count)

    def set_state(self, arrays: dict, acc) -> None:
        a = [None, None, None] if acc is None else acc
        self.session.set_state(arrays["x"], arrays["y"], arrays["z"], arrays["vx"], arrays["vy"], arrays["vz"],
                               arrays["m"], *a)

    def position_tensors(self):
        return self._pos

    @staticmethod
    def send_view(t):
        return t  # NCCL gathers in place: the send buffer is the rank's own chunk of the output

    def kick_drift(self, h: float, dt: float) -> None:
        self.session.kick_drift(h, dt)

    def force_kick(self, h: float, precision=None) -> None:
        from ._ffi import PRECISION_F64
        self.session.force_kick(h, PRECISION_F64 if precision is None else precision)

    def state(self) -> dict:
        return self.session.get_state()

    def close(self) -> None:
        self.session.close()


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

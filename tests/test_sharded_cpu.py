"""The multi-rank KDK step on CPU: world_size 2 over gloo, forces from the oracle.

The sharded run (ownership ranges + one position all-gather per step) must reproduce the
single-process per-target leapfrog of the oracle bit for bit.
"""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

import conftest  # noqa: F401  (registers the engine package as `gx` in spawned ranks too)
import oracle
from gx.sharded import ShardedLeapfrog, ensemble_shard, ownership_range, partition_instances


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _oracle_force(X, m, b, e):
    Xn = X.numpy()
    a = oracle.direct_targets(Xn[0], Xn[1], Xn[2], m.numpy(), 1.0, 0.05, b, e)
    return torch.from_numpy(np.ascontiguousarray(a.T))


def _worker(rank, world, port, n, steps, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=__import__("datetime").timedelta(seconds=60))
    try:
        import gx
        p = gx.ics.two_disk_encounter(n // 2, n - n // 2, 42, 0.05)
        X = torch.from_numpy(np.stack([p.x, p.y, p.z]))
        m = torch.from_numpy(p.m)
        sh = ShardedLeapfrog(n, _oracle_force)
        V = torch.from_numpy(np.stack([p.vx, p.vy, p.vz])[:, sh.begin:sh.end].copy())
        A = sh.initial_accelerations(X, m)
        for _ in range(steps):
            sh.step(X, V, A, m, 0.005)
        Vfull = [torch.zeros(3, sh.chunk, dtype=torch.float64) for _ in range(world)]
        pad = torch.zeros(3, sh.chunk, dtype=torch.float64)
        pad[:, : sh.end - sh.begin] = V
        dist.all_gather(Vfull, pad)
        if rank == 0:
            v = np.concatenate([Vfull[r][:, : e - b].numpy() for r, (b, e) in enumerate(sh.ranges)], 1)
            np.save(out, np.concatenate([X.numpy(), v]))
    finally:
        dist.destroy_process_group()


def test_ownership_matches_reference():
    for n in (0, 1, 7, 10, 1001):
        for size in (1, 2, 3, 8):
            rs = [ownership_range(n, r, size) for r in range(size)]
            assert rs == [oracle.ownership(n, r, size) for r in range(size)]
            assert rs[0][0] == 0 and rs[-1][1] == n


@pytest.mark.parametrize("n", [101])
def test_two_rank_step_matches_single_process(tmp_path, n):
    steps = 3
    out = str(tmp_path / "state.npy")
    mp.start_processes(_worker, args=(2, _free_port(), n, steps, out), nprocs=2, start_method="spawn")
    got = np.load(out)
    import gx
    p = gx.ics.two_disk_encounter(n // 2, n - n // 2, 42, 0.05)
    a0 = oracle.direct_targets(p.x, p.y, p.z, p.m, 1.0, 0.05)
    st = dict(x=p.x, y=p.y, z=p.z, vx=p.vx, vy=p.vy, vz=p.vz, ax=a0[:, 0], ay=a0[:, 1], az=a0[:, 2])
    ref = oracle.leapfrog(st, p.m, 1.0, 0.05, 0.005, steps, solver=1)
    expect = np.stack([ref[k] for k in ("x", "y", "z", "vx", "vy", "vz")])
    assert np.array_equal(got, expect)


def test_partition_instances_cover_and_balance():
    import gx
    off, _, _ = gx.ics.ensemble(512, seed=7)
    sizes = np.diff(off)
    cost = sizes * (sizes - 1)
    for world in (1, 2, 3, 8):
        parts = partition_instances(sizes, world)
        assert len(parts) == world
        flat = sorted(i for q in parts for i in q)
        assert flat == list(range(512)) and all(q == sorted(q) for q in parts)
        loads = [int(cost[q].sum()) for q in parts]
        assert max(loads) <= 1.01 * sum(loads) / world
    assert partition_instances([5, 5, 9], 2) == [[2], [0, 1]]


def _ensemble_worker(rank, world, port, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=__import__("datetime").timedelta(seconds=60))
    try:
        import gx
        off, p, _ = gx.ics.ensemble(6, seed=3, n_min=64, n_max=160)
        ids, sub, body = ensemble_shard(off, rank, world)
        # each rank steps its own encounters (oracle forces, per instance), no exchange
        res = np.zeros((6, len(p.x)))
        for q, i in enumerate(ids):
            b = body[sub[q]:sub[q + 1]]
            a = oracle.direct_targets(p.x[b], p.y[b], p.z[b], p.m[b], 1.0, 0.05)
            st = dict(x=p.x[b], y=p.y[b], z=p.z[b], vx=p.vx[b], vy=p.vy[b], vz=p.vz[b], ax=a[:, 0], ay=a[:, 1],
                      az=a[:, 2])
            r = oracle.leapfrog(st, p.m[b], 1.0, 0.05, 0.005, 2, solver=1)
            for k, name in enumerate(("x", "y", "z", "vx", "vy", "vz")):
                res[k, b] = r[name]
        t = torch.from_numpy(res)
        dist.all_reduce(t)  # bodies are owned by exactly one rank: the sum assembles the state
        if rank == 0:
            np.save(out, t.numpy())
    finally:
        dist.destroy_process_group()


def test_two_rank_ensemble_by_instance(tmp_path):
    """Instances split over two gloo ranks and stepped independently equal the whole
    ensemble stepped in one process."""
    out = str(tmp_path / "ens.npy")
    mp.start_processes(_ensemble_worker, args=(2, _free_port(), out), nprocs=2, start_method="spawn")
    got = np.load(out)
    import gx
    off, p, _ = gx.ics.ensemble(6, seed=3, n_min=64, n_max=160)
    for i in range(6):
        b = np.arange(off[i], off[i + 1])
        a = oracle.direct_targets(p.x[b], p.y[b], p.z[b], p.m[b], 1.0, 0.05)
        st = dict(x=p.x[b], y=p.y[b], z=p.z[b], vx=p.vx[b], vy=p.vy[b], vz=p.vz[b], ax=a[:, 0], ay=a[:, 1], az=a[:, 2])
        r = oracle.leapfrog(st, p.m[b], 1.0, 0.05, 0.005, 2, solver=1)
        for k, name in enumerate(("x", "y", "z", "vx", "vy", "vz")):
            assert np.array_equal(got[k, b], r[name]), (i, name)


class CpuShard:
    """The engine-shard interface of ShardedSession on the CPU: the padded slot arrays as
    torch tensors, the reference's kick/drift rounding (separate multiply and add), and the
    oracle's per-target sum over all slots for the owned ones."""

    def __init__(self, slots, eps):
        self.slots, self.eps = slots, eps

    def set_targets(self, begin, count):
        self.sl = slice(begin, begin + count)

    def set_state(self, arrays, acc):
        self.s = {k: torch.from_numpy(np.array(arrays[k], dtype=np.float64)) for k in arrays}
        for k, a in zip(("ax", "ay", "az"), acc or [np.zeros(self.slots)] * 3):
            self.s[k] = torch.from_numpy(np.array(a, dtype=np.float64))

    def position_tensors(self):
        return [self.s["x"], self.s["y"], self.s["z"]]

    @staticmethod
    def send_view(t):
        return t.clone()  # gloo's all-gather does not take a slice of its output as input

    def kick_drift(self, h, dt):
        s, sl = self.s, self.sl
        for v, a, x in (("vx", "ax", "x"), ("vy", "ay", "y"), ("vz", "az", "z")):
            s[v][sl] = s[v][sl] + s[a][sl] * h
            s[x][sl] = s[x][sl] + s[v][sl] * dt

    def force_kick(self, h, precision=None):
        s, sl = self.s, self.sl
        a = oracle.direct_targets(*(s[k].numpy() for k in ("x", "y", "z", "m")), 1.0, self.eps, sl.start, sl.stop)
        for c, (ak, vk) in enumerate((("ax", "vx"), ("ay", "vy"), ("az", "vz"))):
            s[ak][sl] = torch.from_numpy(np.ascontiguousarray(a[:, c]))
            if h != 0.0:
                s[vk][sl] = s[vk][sl] + s[ak][sl] * h

    def state(self):
        return {k: v.numpy().copy() for k, v in self.s.items()}


def _session_worker(rank, world, port, n, steps, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=__import__("datetime").timedelta(seconds=60))
    try:
        import gx
        from gx.sharded import ShardLayout, ShardedSession
        p = gx.ics.two_disk_encounter(n // 2, n - n // 2, 42, 0.05)
        sh = ShardedSession(n, None, backend=CpuShard(ShardLayout(n, world).slots, 0.05))
        sh.set_state(p.x, p.y, p.z, p.vx, p.vy, p.vz, p.m)
        sh.compute_accelerations()
        sh.step(steps, 0.005)
        st = sh.get_state()
        if rank == 0:
            np.save(out, np.stack([st[k] for k in ("x", "y", "z", "vx", "vy", "vz", "ax", "ay", "az")]))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("n,world", [(101, 2), (7, 3)])
def test_sharded_session_padded_layout_matches_single_process(tmp_path, n, world):
    """ShardedSession's padded rank-major layout (zero-mass padding slots, in-place
    all-gathers of x, y, z) reproduces the single-process per-target leapfrog of the oracle
    bit for bit, accelerations included, with uneven ownership ranges."""
    steps = 3
    out = str(tmp_path / "state.npy")
    mp.start_processes(_session_worker, args=(world, _free_port(), n, steps, out), nprocs=world, start_method="spawn")
    got = np.load(out)
    import gx
    p = gx.ics.two_disk_encounter(n // 2, n - n // 2, 42, 0.05)
    a0 = oracle.direct_targets(p.x, p.y, p.z, p.m, 1.0, 0.05)
    st = dict(x=p.x, y=p.y, z=p.z, vx=p.vx, vy=p.vy, vz=p.vz, ax=a0[:, 0], ay=a0[:, 1], az=a0[:, 2])
    ref = oracle.leapfrog(st, p.m, 1.0, 0.05, 0.005, steps, solver=1)
    expect = np.stack([ref[k] for k in ("x", "y", "z", "vx", "vy", "vz", "ax", "ay", "az")])
    assert np.array_equal(got, expect)


def test_shard_layout_round_trip():
    from gx.sharded import ShardLayout
    for n, world in ((0, 1), (1, 1), (10, 3), (101, 2), (1000, 8)):
        L = ShardLayout(n, world)
        a = np.arange(n, dtype=np.float64) + 0.5
        padded = L.pad(a)
        assert len(padded) == L.slots == L.chunk * world
        assert np.array_equal(L.unpad(padded), a)
        assert np.count_nonzero(padded) == n  # padding slots stay zero (zero mass)

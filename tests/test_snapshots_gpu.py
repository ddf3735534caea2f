"""Snapshots of device-resident state (B200): a session snapshot taken while the session keeps
stepping is the state of the step it was taken at, byte for byte, and device arrays give the
same files as host arrays."""
import numpy as np
import pytest
import torch

import gx

pytestmark = pytest.mark.gpu


def test_session_snapshot_does_not_wait_and_is_exact(tmp_path):
    p = gx.ics.two_disk_encounter(3000, 2000, 21, 0.02)
    g = (np.arange(len(p)) % 2).astype(np.uint32)
    params = gx.PhysicsParams(1.0, 0.02)
    with gx.Session(len(p), params) as s, gx.SnapshotWriter(tmp_path / "async", len(p), g, binary=True) as w:
        s.set_particles(p)
        s.compute_accelerations(gx.PRECISION_F64)
        s.step(5, 0.001, gx.PRECISION_F64)
        s.snapshot(w, 5, 0.005)
        s.step(5, 0.001, gx.PRECISION_F64)   # overwrites the state while the snapshot is in flight
        s.snapshot(w, 10, 0.010)
        w.flush()
        late = s.get_state()
    with gx.Session(len(p), params) as s2:
        s2.set_particles(p)
        s2.compute_accelerations(gx.PRECISION_F64)
        s2.step(5, 0.001, gx.PRECISION_F64)
        st = s2.get_state()
    with gx.SnapshotWriter(tmp_path / "host", len(p), g) as w2:
        w2.write(5, 0.005, m=p.m, **st)
    name = "snapshot_000005.csv"
    assert (tmp_path / "async" / name).read_bytes() == (tmp_path / "host" / name).read_bytes()
    b = gx.read_binary(tmp_path / "async" / "snapshot_000010.bin")
    assert all(np.array_equal(b[k], late[k]) for k in late) and b["step"] == 10


def test_device_arrays_match_host_arrays(tmp_path):
    n = 4099
    rng = np.random.default_rng(4)
    host = {k: rng.normal(size=n) for k in gx.snapshots.FIELDS}
    dev = {k: torch.tensor(v, device="cuda") for k, v in host.items()}
    stream = torch.cuda.Stream()
    with gx.SnapshotWriter(tmp_path / "d", n, slots=3) as w:
        w.write(7, 1.5, stream=stream, **dev)
    with gx.SnapshotWriter(tmp_path / "h", n) as w:
        w.write(7, 1.5, **host)
    assert (tmp_path / "d" / "snapshot_000007.csv").read_bytes() == (tmp_path / "h" / "snapshot_000007.csv").read_bytes()

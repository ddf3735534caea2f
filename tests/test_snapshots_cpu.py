"""Snapshot output vs the reference's own SnapshotWriter (cpp/io/snapshot_writer.cpp:38-128),
built from its sources: the CSV snapshot and diagnostics.csv are byte-identical; the binary
form round-trips.  Host arrays only -- no GPU needed."""
import numpy as np
import pytest

import gx
import oracle

need_ref = pytest.mark.skipif(not oracle.ref_available(), reason="reference build absent")


def state(n, seed):
    rng = np.random.default_rng(seed)
    s = {k: rng.normal(size=n) * 10.0 ** rng.integers(-8, 8, size=n) for k in
         ("x", "y", "z", "vx", "vy", "vz", "ax", "ay", "az")}
    s["x"][:3] = [0.0, -0.0, 1e-310]          # signed zero, subnormal
    s["vx"][:2] = [1.0 / 3.0, 123456789.0]
    m = rng.random(n) * 1e-3
    return s, m


@need_ref
@pytest.mark.parametrize("n,step,time", [(1000, 20, 0.2), (37, 0, 0.0), (5000, 123456, 1.0 / 3.0)])
def test_csv_matches_reference_writer(tmp_path, n, step, time):
    s, m = state(n, n)
    g = (np.arange(n) % 3).astype(np.uint32)
    diag = np.array([1.0, 0.25, -0.5, -0.25, 1e-17, -2e-17, 3.0, 0.1, 0.2, 0.3, -1e-5, 2e-5, 1.0 / 7.0])
    oracle.ref_write_outputs(tmp_path / "ref", s, m, g, step, time, diag)
    with gx.SnapshotWriter(tmp_path / "ours", n, g) as w:
        w.write(step, time, m=m, **s)
        w.write_diagnostics(step, time, gx.Diagnostics(total_mass=diag[0], kinetic_energy=diag[1],
                                                       potential_energy=diag[2], total_energy=diag[3],
                                                       momentum=tuple(diag[4:7]), center_of_mass=tuple(diag[7:10]),
                                                       angular_momentum=tuple(diag[10:13])))
    name = f"snapshot_{step:06d}.csv"
    assert (tmp_path / "ours" / name).read_bytes() == (tmp_path / "ref" / name).read_bytes()
    assert (tmp_path / "ours" / "diagnostics.csv").read_bytes() == (tmp_path / "ref" / "diagnostics.csv").read_bytes()


def test_binary_round_trip_and_several_snapshots(tmp_path):
    n = 777
    s, m = state(n, 3)
    with gx.SnapshotWriter(tmp_path, n, np.arange(n) % 5, csv=False, binary=True, slots=1) as w:
        for k in range(3):
            w.write(k, 0.5 * k, m=m, **{f: v + k for f, v in s.items()})
    for k in range(3):
        b = gx.read_binary(tmp_path / f"snapshot_{k:06d}.bin")
        assert b["step"] == k and b["time"] == 0.5 * k
        assert np.array_equal(b["x"], s["x"] + k) and np.array_equal(b["m"], m)
        assert np.array_equal(b["group_id"], np.arange(n) % 5)
    assert not (tmp_path / "diagnostics.csv").exists()


def test_writer_errors(tmp_path):
    with pytest.raises(gx.GxError):
        gx.SnapshotWriter(tmp_path, 10, csv=False, binary=False)
    f = tmp_path / "a_file"
    f.write_text("x")
    with pytest.raises(gx.GxError):
        gx.SnapshotWriter(f / "sub", 10)


@need_ref
@pytest.mark.parametrize("md", [
    dict(name="benchmark_direct_1000", solver="cuda-direct", particle_count=1000, steps=20, dt=0.01,
         snapshot_every=20, dim=3, G=1.0, eps=0.025, theta=0.58, leaf_capacity=16, order=4),
    dict(name='quote " and back\\slash', solver="fmm", particle_count=1 << 20, steps=123456, dt=1.0 / 3.0,
         snapshot_every=7, dim=2, G=6.674e-11, eps=1e-300, theta=0.6, leaf_capacity=64, order=0),
    dict(name="", solver="direct", particle_count=0, steps=0, dt=1e22, snapshot_every=1, dim=3, G=-0.0,
         eps=123456789.0, theta=1e-5, leaf_capacity=1, order=3),
])
def test_metadata_matches_reference_writer(tmp_path, md):
    """metadata.json (SnapshotWriter::write_metadata, snapshot_writer.cpp:49-69) byte for byte:
    escaped strings, integers and doubles in the default six-digit ostream format."""
    oracle.ref_write_metadata(tmp_path / "ref", md["name"], md["solver"], md["particle_count"], md["steps"], md["dt"],
                              md["snapshot_every"], md["dim"], md["G"], md["eps"], md["theta"], md["leaf_capacity"],
                              md["order"])
    with gx.SnapshotWriter(tmp_path / "ours", 1) as w:
        w.write_metadata(md["name"], md["solver"], md["particle_count"], md["steps"], md["dt"], md["snapshot_every"],
                         md["dim"], md["G"], md["eps"], md["theta"], md["leaf_capacity"], md["order"])
    assert (tmp_path / "ours" / "metadata.json").read_bytes() == (tmp_path / "ref" / "metadata.json").read_bytes()

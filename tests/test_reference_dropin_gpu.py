"""The reference itself with the engine dropped in (B200).

oracle/_ref/ holds the reference's unmodified sources built with the engine's shim in place
of cpp/cuda/cuda_solver.cu (oracle/Makefile): its own smoke tests must pass, and its CLI with
`solver = "cuda-direct"` must reproduce the reference's golden direct run.
"""
import os
import subprocess

import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu

# The benchmark configuration of experiments/benchmarks/local_cpu/configs/direct_1000_r1.toml
# with the solver switched to the drop-in (all other values as in that run).
CONFIG = """[simulation]
name = "dropin_direct_1000"
dim = 3
solver = "cuda-direct"
seed = 20260502
n_particles = 1000
steps = 20
dt = 0.01
snapshot_every = 20
[physics]
G = 1.0
softening = 0.025
[galaxy.primary]
n_particles = 500
mass = 1.0
radius = 0.85
position = [-0.72, -0.10, 0.06]
velocity = [0.34, 0.10, -0.015]
orientation = 0.25
group_id = 0
thickness = 0.045
inclination = 0.62
[galaxy.secondary]
n_particles = 500
mass = 1.0
radius = 0.85
position = [0.72, 0.10, -0.06]
velocity = [-0.34, -0.10, 0.015]
orientation = 3.42
group_id = 1
thickness = 0.045
inclination = -0.72
[output]
directory = "{out}"
format = "csv"
"""


def _need(path):
    if not path.exists():
        pytest.skip(f"{path.name} was not built (the reference tree was absent at build time)")


def test_reference_smoke_tests_pass_with_engine(tmp_path):
    _need(oracle.REF_SMOKE_B200)
    r = subprocess.run([str(oracle.REF_SMOKE_B200)], cwd=tmp_path, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "smoke_tests passed" in r.stdout


def _load_snapshot(path):
    a = np.loadtxt(path, delimiter=",", comments="#", skiprows=2)
    return a[:, 3:12]


@pytest.mark.parametrize("precision", ["f64", "f64-exact"])
def test_reference_cli_cuda_direct(tmp_path, golden, precision):
    _need(oracle.REF_SIM_B200)
    out = tmp_path / "out"
    cfg = tmp_path / "cfg.toml"
    cfg.write_text(CONFIG.format(out=out))
    env = dict(os.environ, GX_PRECISION=precision)
    r = subprocess.run([str(oracle.REF_SIM_B200), "--config", str(cfg)], capture_output=True, text=True, timeout=300,
                       env=env)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "CUDA direct available: yes" in r.stdout
    g = golden("direct_snapshots.npz")
    s0 = _load_snapshot(out / "snapshot_000000.csv")
    s20 = _load_snapshot(out / "snapshot_000020.csv")
    keys = ("x", "y", "z", "vx", "vy", "vz", "ax", "ay", "az")
    want0 = np.stack([g[f"direct_1000_r1/s0/{k}"] for k in keys], 1)
    want20 = np.stack([g[f"direct_1000_r1/s20/{k}"] for k in keys], 1)
    # initial conditions are the reference generator's; the golden files were written on
    # another platform's libm, so they agree to the last bit or two only
    assert np.max(np.abs(s0[:, :6] - want0[:, :6])) <= 1e-14
    assert np.max(np.abs(s20[:, :3] - want20[:, :3])) <= 1e-10
    assert np.max(np.abs(s20[:, 6:] - want20[:, 6:]) / np.abs(want20[:, 6:]).max()) <= 1e-9
    if precision == "f64-exact":
        # per-target order: step 0 equals the reference's _for_targets sum
        a3 = oracle.direct_targets(s0[:, 0], s0[:, 1], s0[:, 2], g["direct_1000_r1/s0/m"], 1.0, 0.025)
        assert np.max(np.abs(s0[:, 6:] - a3)) <= 1e-15 * np.abs(a3).max()


def _run(exe, cfg, env_extra):
    env = dict(os.environ, **env_extra)
    r = subprocess.run([str(exe), "--config", str(cfg)], capture_output=True, text=True, timeout=300, env=env)
    assert r.returncode == 0, r.stdout + r.stderr
    return r


def test_resident_step_loop_matches_the_reference_cli(tmp_path):
    """The reference's step loop on the resident session (csrc/shim/resident_main.cpp, built
    with the reference's config loader, generator and SnapshotWriter against
    include/gx_session.hpp): one upload, gx_session_step between snapshot steps, one download
    per snapshot.  In the exact form, with the reference's host diagnostics, every file it
    writes -- metadata.json, the snapshots at steps 0, 5, 10, 15, 20 and diagnostics.csv --
    is byte-identical to the reference CLI running the per-step drop-in."""
    _need(oracle.REF_SIM_RESIDENT)
    _need(oracle.REF_SIM_B200)
    outs = {}
    for name, exe, extra in (("cli", oracle.REF_SIM_B200, {"GX_PRECISION": "f64-exact"}),
                             ("resident", oracle.REF_SIM_RESIDENT, {"GX_PRECISION": "f64-exact",
                                                                     "GX_DIAGNOSTICS": "host"})):
        out = tmp_path / name
        cfg = tmp_path / f"{name}.toml"
        cfg.write_text(CONFIG.format(out=out).replace("snapshot_every = 20", "snapshot_every = 5"))
        _run(exe, cfg, extra)
        outs[name] = out
    files = sorted(p.name for p in outs["cli"].iterdir())
    assert files == sorted(p.name for p in outs["resident"].iterdir())
    assert [f for f in files if f.startswith("snapshot_")] == [f"snapshot_{s:06d}.csv" for s in (0, 5, 10, 15, 20)]
    assert "metadata.json" in files and "diagnostics.csv" in files
    for f in files:
        assert (outs["cli"] / f).read_bytes() == (outs["resident"] / f).read_bytes(), f


def test_resident_step_loop_matches_the_golden_run(tmp_path, golden):
    """FP64 form with device diagnostics against the reference's committed direct_1000_r1 run
    (CPU symmetric direct sum): snapshots 0 and 20 and both diagnostics rows."""
    _need(oracle.REF_SIM_RESIDENT)
    out = tmp_path / "out"
    cfg = tmp_path / "cfg.toml"
    cfg.write_text(CONFIG.format(out=out))
    r = _run(oracle.REF_SIM_RESIDENT, cfg, {"GX_PRECISION": "f64"})
    assert "resident session" in r.stdout
    g = golden("direct_snapshots.npz")
    keys = ("x", "y", "z", "vx", "vy", "vz", "ax", "ay", "az")
    assert sorted(p.name for p in out.glob("snapshot_*.csv")) == ["snapshot_000000.csv", "snapshot_000020.csv"]
    s20 = _load_snapshot(out / "snapshot_000020.csv")
    want20 = np.stack([g[f"direct_1000_r1/s20/{k}"] for k in keys], 1)
    assert np.max(np.abs(s20[:, :3] - want20[:, :3])) <= 1e-10
    assert np.max(np.abs(s20[:, 6:] - want20[:, 6:]) / np.abs(want20[:, 6:]).max()) <= 1e-9
    d = np.loadtxt(out / "diagnostics.csv", delimiter=",", skiprows=1)
    gd = g["direct_1000_r1/diagnostics"]
    assert d.shape == gd.shape and np.array_equal(d[:, :3], gd[:, :3])  # step, time, n
    scale = np.maximum(np.abs(gd[:, 3:]).max(0), 1e-300)
    assert np.max(np.abs(d[:, 3:] - gd[:, 3:]) / scale) <= 1e-10

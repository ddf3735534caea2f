"""Device kick-drift-kick, the resident session (CUDA graphs) and FP64 diagnostics (B200).

Tolerances: the 20-step trajectories of the reference's golden snapshots and of the N=1000
workload within max |dx| <= 1e-10 (FP64); the exact form reproduces the oracle's per-target
leapfrog bit for bit; diagnostics within 1e-12 relative.
"""
import ctypes

import numpy as np
import pytest

import gx
import oracle
from conftest import rel_err

pytestmark = pytest.mark.gpu

F64, MIX, EXACT = gx.PRECISION_F64, gx.PRECISION_MIXED, gx.PRECISION_F64_EXACT
STATE = ("x", "y", "z", "vx", "vy", "vz", "ax", "ay", "az")


def snapshot(g, name, step):
    s = {k: g[f"{name}/s{step}/{k}"] for k in STATE}
    s["m"] = g[f"{name}/s{step}/m"]
    return s


def as_particles(s):
    return gx.ParticleSet(s["x"], s["y"], s["z"], s["vx"], s["vy"], s["vz"], s["m"], s["ax"], s["ay"], s["az"])


@pytest.mark.parametrize("name", ["direct_250_r1", "direct_1000_r1"])
def test_golden_snapshot_trajectory(golden, name):
    g = golden("direct_snapshots.npz")
    s0, s20 = snapshot(g, name, 0), snapshot(g, name, 20)
    params = gx.PhysicsParams(1.0, 0.025)
    # resident session
    with gx.Session(len(s0["m"]), params) as s:
        s.set_particles(as_particles(s0))
        s.step(20, 0.01, F64)
        st = s.get_state()
    for k in ("x", "y", "z"):
        assert np.max(np.abs(st[k] - s20[k])) <= 1e-10
    assert rel_err(np.stack([st["ax"], st["ay"], st["az"]], 1), np.stack([s20["ax"], s20["ay"], s20["az"]], 1)).max() < 1e-9
    # the drop-in step on host arrays (cuda_direct_leapfrog_step semantics)
    p = as_particles(s0)
    for _ in range(20):
        gx.cuda_direct_leapfrog_step(p, 0.01, params)
    for k in ("x", "y", "z"):
        assert np.max(np.abs(getattr(p, k) - s20[k])) <= 1e-10
    # the exact form is the oracle's per-target leapfrog, bit for bit
    with gx.Session(len(s0["m"]), params) as s:
        s.set_particles(as_particles(s0))
        s.step(20, 0.01, EXACT)
        st = s.get_state()
    ref = oracle.leapfrog(s0, s0["m"], 1.0, 0.025, 0.01, 20, solver=1)
    for k in STATE:
        assert np.array_equal(st[k], ref[k]), k


def test_workload_n1000_fixture(golden):
    g = golden("cfg0_n1000.npz")
    eps, dt = float(g["softening"]), float(g["dt"])
    p = gx.ParticleSet(g["x0"], g["y0"], g["z0"], g["vx0"], g["vy0"], g["vz0"], g["m"])
    with gx.Session(len(p), gx.PhysicsParams(1.0, eps)) as s:
        s.set_particles(p)
        s.compute_accelerations(F64)
        a0 = s.get_state()
        assert rel_err(np.stack([a0["ax"], a0["ay"], a0["az"]], 1), g["a0"]).max() < 1e-11
        d0 = s.diagnostics()
        s.step(20, dt, F64)
        st = s.get_state()
        d20 = s.diagnostics()
    for k in ("x", "y", "z"):
        assert np.max(np.abs(st[k] - g[f"{k}20"])) <= 1e-10
    np.testing.assert_allclose(d0.as_row(), g["diag0"], rtol=1e-12, atol=1e-14)
    np.testing.assert_allclose(d20.as_row(), g["diag20"], rtol=1e-11, atol=1e-13)


@pytest.mark.parametrize("prec", [F64, MIX])
def test_graph_replay_equals_eager(prec):
    p = gx.ics.two_disk_encounter(900, 700, 3, 0.02)
    params = gx.PhysicsParams(1.0, 0.02)
    out = []
    for timing in (False, True):
        with gx.Session(len(p), params) as s:
            s.set_persistent(False)  # graph replay vs eager launches of the same kernels
            s.set_particles(p)
            s.compute_accelerations(prec)
            s.enable_timing(timing)
            s.step(45, 0.002, prec)  # graphs: 32 + 13; eager when timing is on
            s.synchronize()
            if timing:
                ms, launches = s.force_timing()
                assert launches == 45 and ms > 0
            out.append(s.get_state())
    for k in STATE:
        assert np.array_equal(out[0][k], out[1][k]), k


def test_session_set_state_from_device_and_arrays():
    import torch
    p = gx.ics.two_disk_encounter(500, 500, 8, 0.05)
    with gx.Session(len(p), gx.PhysicsParams(1.0, 0.05)) as s:
        t = {k: torch.from_numpy(getattr(p, k)).cuda() for k in ("x", "y", "z", "vx", "vy", "vz", "m")}
        s.set_state(t["x"], t["y"], t["z"], t["vx"], t["vy"], t["vz"], t["m"])
        st = s.get_state()
        assert np.array_equal(st["x"], p.x) and np.all(st["ax"] == 0)
        ptrs = s.device_arrays()
        assert all(v for v in ptrs.values())


@pytest.mark.parametrize("eps", [0.02, 0.0])
def test_diagnostics_vs_oracle(eps):
    p = gx.ics.two_disk_encounter(1500, 1500, 21, 0.02)
    if eps == 0.0:
        p.x[7], p.y[7], p.z[7] = p.x[8], p.y[8], p.z[8]  # a coincident pair is skipped
    d = gx.compute_diagnostics(p, gx.PhysicsParams(1.0, eps))
    ref = oracle.diagnostics(p.x, p.y, p.z, p.vx, p.vy, p.vz, p.m, 1.0, eps)
    np.testing.assert_allclose(d.as_row(), ref, rtol=1e-12, atol=1e-13)


def test_energy_drift_mixed_vs_f64():
    p = gx.ics.two_disk_encounter(2048, 2048, 12, 0.05)
    params = gx.PhysicsParams(1.0, 0.05)
    drift = {}
    for prec in (F64, MIX):
        with gx.Session(len(p), params) as s:
            s.set_particles(p)
            s.compute_accelerations(prec)
            e0 = s.diagnostics().total_energy
            s.step(200, 0.005, prec)
            drift[prec] = abs(s.diagnostics().total_energy - e0) / abs(e0)
    assert drift[F64] < 1e-4 and drift[MIX] < 1e-4
    assert abs(drift[MIX] - drift[F64]) < 1e-5


def test_bounded_wait_times_out_then_recovers():
    """A host wait with a short limit gives GX_ERR_TIMEOUT while work is in flight; the
    context stays usable (no GPU fault is involved)."""
    p = gx.ics.two_disk_encounter(32768, 32768, 2, 0.02)
    with gx.Session(len(p), gx.PhysicsParams(1.0, 0.02)) as s:
        s.set_particles(p)
        s.step(3, 0.001, EXACT)  # tens of milliseconds of work
        with pytest.raises(gx.GxError) as e:
            s.synchronize(timeout_ms=0.01)
        assert e.value.status == gx.GX_ERR_TIMEOUT
        s.synchronize(timeout_ms=60000.0)
        assert np.all(np.isfinite(s.get_state()["x"]))


def test_allocation_failure_is_reported():
    gx._ffi.call("gx_debug_fail_allocations", 1)
    with pytest.raises(gx.GxError) as e:
        gx.Session(1000, gx.PhysicsParams())
    assert e.value.status == gx.GX_ERR_OUT_OF_MEMORY
    with gx.Session(1000, gx.PhysicsParams()) as s:  # the next allocation works again
        s.synchronize()
    gx._ffi.call("gx_debug_fail_allocations", 0)


def test_autotune_keeps_results():
    p = gx.ics.two_disk_encounter(3000, 3000, 31, 0.02)
    with gx.Session(len(p), gx.PhysicsParams(1.0, 0.02)) as s:
        s.set_particles(p)
        s.compute_accelerations(MIX)
        before = s.get_state()
        ms = s.autotune(MIX)
        assert ms > 0
        after = s.get_state()
        assert np.array_equal(before["ax"], after["ax"])  # tuning restores the state
        v, js = s.get_config(MIX)
        assert "mixed" in gx.describe_variant(MIX, v) and js >= 1


@pytest.mark.parametrize("n,steps", [(1, 3), (2, 5), (33, 7), (1000, 20), (1185, 6), (4096, 3)])
def test_single_launch_step_loop(n, steps):
    """Small systems step in one cooperative launch (csrc/small.cu).  The exact form is the
    oracle's per-target leapfrog bit for bit (and equals the graph-replayed step loop); the
    FP64 form stays within the FP64 tolerance of the graph loop.  Sizes cover one, two and
    four targets per warp (1185 > 148 SMs x 8 warps)."""
    eps, dt = 0.05, 0.005
    p = gx.ics.two_disk_encounter(n // 2, n - n // 2, 700 + n, eps)
    params = gx.PhysicsParams(1.0, eps)
    out = {}
    for persistent in (True, False):
        for prec in (EXACT, F64):
            with gx.Session(n, params) as s:
                s.set_persistent(persistent)
                s.set_particles(p)
                s.compute_accelerations(prec)
                s.step(steps, dt, prec)
                s.step(1, dt, prec)  # a second launch continues from the first one's state
                out[persistent, prec] = s.get_state()
    a0 = oracle.direct_targets(p.x, p.y, p.z, p.m, 1.0, eps)
    st0 = dict(x=p.x, y=p.y, z=p.z, vx=p.vx, vy=p.vy, vz=p.vz, ax=a0[:, 0], ay=a0[:, 1], az=a0[:, 2])
    want = oracle.leapfrog(st0, p.m, 1.0, eps, dt, steps + 1, solver=1)
    for k in STATE:
        assert np.array_equal(out[True, EXACT][k], want[k]), k
        assert np.array_equal(out[False, EXACT][k], want[k]), k
    for k in ("x", "y", "z"):
        assert np.max(np.abs(out[True, F64][k] - out[False, F64][k])) <= 1e-12
    acc = lambda st: np.stack([st["ax"], st["ay"], st["az"]], 1)
    if n > 1:
        assert rel_err(acc(out[True, F64]), acc(out[False, F64])).max() <= 1e-11


def test_single_launch_step_loop_zero_softening():
    """Coincident bodies with softening 0: the pair is skipped (s2 == 0) in both forms."""
    n = 300
    p = gx.ics.two_disk_encounter(150, 150, 77, 0.05)
    p.x[5], p.y[5], p.z[5] = p.x[6], p.y[6], p.z[6]
    params = gx.PhysicsParams(1.0, 0.0)
    got = {}
    for prec in (EXACT, F64):
        with gx.Session(n, params) as s:
            s.set_particles(p)
            s.compute_accelerations(prec)
            s.step(4, 1e-4, prec)
            got[prec] = s.get_state()
    a0 = oracle.direct_targets(p.x, p.y, p.z, p.m, 1.0, 0.0)
    st0 = dict(x=p.x, y=p.y, z=p.z, vx=p.vx, vy=p.vy, vz=p.vz, ax=a0[:, 0], ay=a0[:, 1], az=a0[:, 2])
    want = oracle.leapfrog(st0, p.m, 1.0, 0.0, 1e-4, 4, solver=1)
    for k in STATE:
        assert np.array_equal(got[EXACT][k], want[k]), k
        assert np.all(np.isfinite(got[F64][k]))


def test_single_launch_barrier_timeout_is_reported():
    """A participant that leaves before a grid barrier (test hook) makes the others' bounded
    waits run out: the launch ends early, the state stays that of the previous call, the next
    synchronising call reports GX_ERR_TIMEOUT, and the session keeps working afterwards."""
    n, eps, dt = 1000, 0.05, 0.005
    p = gx.ics.two_disk_encounter(500, 500, 12, eps)
    with gx.Session(n, gx.PhysicsParams(1.0, eps)) as s:
        s.set_particles(p)
        s.compute_accelerations(EXACT)
        s.step(3, dt, EXACT)
        before = s.get_state()
        gx._ffi.call("gx_debug_stall_barrier", 2)
        s.step(5, dt, EXACT)
        with pytest.raises(gx.GxError) as ei:
            s.synchronize()
        assert ei.value.status == gx.GX_ERR_TIMEOUT
        after = s.get_state()
        for k in STATE:
            assert np.array_equal(after[k], before[k]), k
        s.step(2, dt, EXACT)  # the session still steps
        s.synchronize()

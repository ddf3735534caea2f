"""Persistent batched-ensemble kernel (B200): each instance against the oracle run on its own
bodies; ragged sizes including single-body instances."""
import numpy as np
import pytest

import gx
import oracle
from conftest import rel_err

pytestmark = pytest.mark.gpu

F64, MIX = gx.PRECISION_F64, gx.PRECISION_MIXED


def ragged(sizes, seed=0, eps=0.05):
    parts = [gx.ics.two_disk_encounter(max(1, s // 2), s - max(1, s // 2), seed + i, eps) if s > 1 else
             gx.ParticleSet([0.5], [0.1], [0.0], [0.0], [0.0], [0.0], [1.0]) for i, s in enumerate(sizes)]
    off = np.concatenate([[0], np.cumsum([len(p) for p in parts])]).astype(np.int64)
    cat = lambda f: np.concatenate([getattr(p, f) for p in parts])
    return off, gx.ParticleSet(cat("x"), cat("y"), cat("z"), cat("vx"), cat("vy"), cat("vz"), cat("m"))


@pytest.mark.parametrize("prec", [F64, MIX])
def test_batch_accel_vs_oracle(prec):
    off, p = ragged([1, 2, 37, 1000, 3000, 513, 1025, 4100])
    a = np.stack(gx.batch_accelerations(off, p.x, p.y, p.z, p.m, gx.PhysicsParams(1.0, 0.05), prec), 1)
    for b in range(len(off) - 1):
        s, e = off[b], off[b + 1]
        ref = oracle.direct_targets(p.x[s:e], p.y[s:e], p.z[s:e], p.m[s:e], 1.0, 0.05)
        if e - s == 1:
            assert np.array_equal(a[s:e], np.zeros((1, 3)))
            continue
        err = rel_err(a[s:e], ref)
        lim = (1e-13, 1e-11) if prec == F64 else (1e-6, 1e-4)
        assert np.median(err) <= lim[0] and err.max() <= lim[1], (b, np.median(err), err.max())


@pytest.mark.parametrize("prec", [F64, MIX])
def test_batch_steps_vs_sessions(prec):
    off, p = ragged([700, 1800, 64, 2500], seed=40)
    params = gx.PhysicsParams(1.0, 0.05)
    with gx.Batch(off, params) as b:
        b.set_state(p.x, p.y, p.z, p.vx, p.vy, p.vz, p.m)
        b.compute_accelerations(prec)
        b.step(25, 0.005, prec)
        st = b.get_state()
    for i in range(len(off) - 1):
        s, e = off[i], off[i + 1]
        q = gx.ParticleSet(p.x[s:e], p.y[s:e], p.z[s:e], p.vx[s:e], p.vy[s:e], p.vz[s:e], p.m[s:e])
        with gx.Session(e - s, params) as ses:
            ses.set_particles(q)
            ses.compute_accelerations(prec)
            ses.step(25, 0.005, prec)
            ref = ses.get_state()
        tol = 1e-11 if prec == F64 else 1e-5
        for k in ("x", "y", "z"):
            assert np.max(np.abs(st[k][s:e] - ref[k])) <= tol * max(1.0, np.abs(ref[k]).max()), (i, k)


def test_batch_autotune_and_diagnostics():
    off, p = ragged([1500, 900, 2048, 3], seed=60)
    params = gx.PhysicsParams(1.0, 0.05)
    with gx.Batch(off, params) as b:
        b.set_state(p.x, p.y, p.z, p.vx, p.vy, p.vz, p.m)
        ms = b.autotune(MIX)
        assert ms > 0 and b.get_config(MIX) >= 0
        b.step(5, 0.005, MIX)
        st = b.get_state()
        diags = b.diagnostics()
    for i, d in enumerate(diags):
        s, e = off[i], off[i + 1]
        ref = oracle.diagnostics(st["x"][s:e], st["y"][s:e], st["z"][s:e], st["vx"][s:e], st["vy"][s:e],
                                 st["vz"][s:e], p.m[s:e], 1.0, 0.05)
        np.testing.assert_allclose(d.as_row(), ref, rtol=1e-11, atol=1e-13)


def test_ensemble_graph_multi_step_timing():
    off, p, _ = gx.ics.ensemble(24, seed=3)
    with gx.Batch(off, gx.PhysicsParams(1.0, 0.05)) as b:
        b.set_state(p.x, p.y, p.z, p.vx, p.vy, p.vz, p.m)
        b.compute_accelerations(MIX)
        b.step(10, 0.005, MIX)  # one captured graph of 10 steps
        g = b.get_state()
        b.set_state(p.x, p.y, p.z, p.vx, p.vy, p.vz, p.m)
        b.compute_accelerations(MIX)
        b.enable_timing(True)
        b.step(10, 0.005, MIX)
        ms, launches = b.force_timing()
        e = b.get_state()
    assert launches == 10 and ms > 0
    assert np.array_equal(g["x"], e["x"])

"""Direct-sum kernels vs the oracle and the reference's known answers (B200).

Tolerances: GX_PRECISION_F64_EXACT bit-identical to compute_direct_accelerations_for_targets;
GX_PRECISION_F64 median relative error <= 1e-13 and max <= 1e-11; GX_PRECISION_MIXED median
<= 1e-6 (the engine's stated target) and max <= 1e-4.
"""
import numpy as np
import pytest
import torch

import gx
import oracle
from conftest import rel_err

pytestmark = pytest.mark.gpu

F64, MIX, EXACT = gx.PRECISION_F64, gx.PRECISION_MIXED, gx.PRECISION_F64_EXACT
TOL = {F64: (1e-13, 1e-11), MIX: (1e-6, 1e-4)}


def accel(p, eps, prec, G=1.0):
    q = p.copy()
    gx.compute_cuda_direct_accelerations(q, gx.PhysicsParams(G, eps), prec)
    return q.accelerations


def ref_a3(p, eps, G=1.0):
    return oracle.direct_targets(p.x, p.y, p.z, p.m, G, eps)


def check(a, ref, prec):
    if prec == EXACT:
        assert np.array_equal(a, ref)
        return
    e = rel_err(a, ref)
    med, mx = TOL[prec]
    assert np.median(e) <= med and e.max() <= mx, (prec, np.median(e), e.max())


def test_device_available():
    assert gx.cuda_solver_available()


def test_smoke80_known_answer(golden):
    """cpp/tests/smoke_tests.cpp:83-123: mean relative error vs the direct solver < 1e-10."""
    g = golden("smoke80.npz")
    p = gx.ParticleSet(g["x"], g["y"], g["z"], np.zeros(80), np.zeros(80), np.zeros(80), g["m"])
    for prec in (F64, EXACT):
        assert rel_err(accel(p, 0.03, prec), g["a_direct"]).mean() < 1e-10
    assert np.array_equal(accel(p, 0.03, EXACT), g["a_targets"])
    assert rel_err(accel(p, 0.03, MIX), g["a_direct"]).mean() < 1e-6


def test_two_body_zero_softening(golden):
    g = golden("smoke80.npz")
    p = gx.ParticleSet(g["two_body_x"], g["two_body_y"], g["two_body_z"], np.zeros(2), np.zeros(2), np.zeros(2),
                       g["two_body_m"])
    for prec in (F64, EXACT, MIX):
        a = accel(p, 0.0, prec)
        assert a[0, 0] > 0 and a[1, 0] < 0
        assert abs(2.0 * a[0, 0] + 3.0 * a[1, 0]) < (1e-12 if prec != MIX else 1e-6)
    assert np.array_equal(accel(p, 0.0, EXACT), oracle.direct_targets(p.x, p.y, p.z, p.m, 1.0, 0.0))
    assert rel_err(accel(p, 0.0, F64), g["two_body_a"]).max() < 1e-15


@pytest.mark.parametrize("n", [1, 2, 3, 31, 33, 255, 257, 1000, 1025, 4097])
@pytest.mark.parametrize("prec", [F64, MIX, EXACT])
def test_sizes_vs_oracle(n, prec):
    p = gx.ics.two_disk_encounter(n // 2, n - n // 2, 1000 + n, 0.05)
    a = accel(p, 0.05, prec)
    if n == 1:
        assert np.array_equal(a, np.zeros((1, 3)))
        return
    check(a, ref_a3(p, 0.05), prec)


@pytest.mark.parametrize("prec", [F64, MIX, EXACT])
def test_zero_softening_coincident_bodies(prec):
    p = gx.ics.two_disk_encounter(300, 300, 5, 0.05)
    for j in (10, 11, 12):  # three coincident copies of body 3
        p.x[j], p.y[j], p.z[j] = p.x[3], p.y[3], p.z[3]
    a = accel(p, 0.0, prec)
    assert np.all(np.isfinite(a))
    ref = ref_a3(p, 0.0)
    if prec == MIX:
        # close pairs amplify FP32 offset rounding without softening: check the bulk only
        assert np.median(rel_err(a, ref)) <= 1e-5
    else:
        check(a, ref, prec)


@pytest.mark.parametrize("prec", [F64, MIX])
def test_every_variant_and_split(prec):
    n = 3001
    p = gx.ics.two_disk_encounter(1500, 1501, 77, 0.02)
    ref = ref_a3(p, 0.02)
    count = 0
    with gx.Session(n, gx.PhysicsParams(1.0, 0.02)) as s:
        s.set_particles(p)
        for v in range(64):
            try:
                desc = gx.describe_variant(prec, v)
            except gx.GxError:
                continue
            if "eps0" in desc:
                continue
            for js in (1, 2, 3, 7):
                s.set_config(prec, v, js)
                s.compute_accelerations(prec)
                st = s.get_state()
                a = np.stack([st["ax"], st["ay"], st["az"]], 1)
                check(a, ref, prec)
                count += 1
    assert count >= 12


@pytest.mark.parametrize("prec", [F64, EXACT, MIX])
def test_target_ranges_and_lists(prec):
    p = gx.ics.two_disk_encounter(1200, 800, 9, 0.03)
    params = gx.PhysicsParams(1.0, 0.03)
    full = accel(p, 0.03, prec)
    q = p.copy()
    q.ax[:] = 0
    gx.compute_direct_accelerations_for_targets(q, params, 150, 1333, prec)
    assert np.all(q.ax[:150] == 0) and np.all(q.ax[1333:] == 0)
    idx = np.random.default_rng(1).choice(len(p), 257, replace=False)
    a = gx.indexed_accelerations(p, params, idx, prec)
    for got, want in ((q.accelerations[150:1333], full[150:1333]), (a, full[idx])):
        if prec == MIX:  # a different target tile has a different FP64 origin
            e = rel_err(got, want)
            assert np.median(e) <= 1e-6 and e.max() <= 1e-4
        else:
            assert np.max(rel_err(got, want)) <= (0 if prec == EXACT else 1e-14)


@pytest.mark.parametrize("prec", [F64, MIX])
def test_device_pointers_and_streams(prec):
    p = gx.ics.two_disk_encounter(700, 700, 4, 0.02)
    host = accel(p, 0.02, prec)
    dev = {k: torch.from_numpy(getattr(p, k)).cuda() for k in ("x", "y", "z", "m")}
    out = [torch.empty_like(dev["x"]) for _ in range(3)]
    s = torch.cuda.Stream()
    with torch.cuda.stream(s):
        gx._ffi.call("gx_direct_accel", len(p), *(gx._ffi.ptr(dev[k]) for k in ("x", "y", "z", "m")),
                     gx._ffi.physics(1.0, 0.02), prec, *(gx._ffi.ptr(o) for o in out), s.cuda_stream)
    s.synchronize()
    got = torch.stack(out, 1).cpu().numpy()
    assert np.max(rel_err(got, host)) <= (1e-14 if prec == F64 else 1e-6)


def test_mixed_host_device_mismatch_rejected():
    x = np.zeros(8)
    d = torch.zeros(8, dtype=torch.float64, device="cuda")
    st = gx._ffi.load().gx_direct_accel(8, x.ctypes.data, d.data_ptr(), x.ctypes.data, x.ctypes.data,
                                        gx._ffi.physics(1, 0.1), 0, x.ctypes.data, x.ctypes.data, x.ctypes.data, None)
    assert st == gx.GX_ERR_INVALID_ARGUMENT


def test_mixed_precision_error_at_scale():
    """The mixed form on a 131072-body 3:1 encounter (softening 0.01) against the FP64
    oracle on 512 sampled targets: median <= 1e-6."""
    p = gx.ics.two_disk_encounter(65536, 65536, 20260502, 0.01, mass2=1.0 / 3.0)
    idx = np.random.default_rng(0).choice(len(p), 512, replace=False)
    a = gx.indexed_accelerations(p, gx.PhysicsParams(1.0, 0.01), idx, MIX)
    ref = oracle.direct_indexed(p.x, p.y, p.z, p.m, 1.0, 0.01, idx, threads=oracle.default_threads())
    e = rel_err(a, ref)
    assert np.median(e) <= 1e-6 and e.max() <= 1e-4, (np.median(e), e.max())
    exact = gx.indexed_accelerations(p, gx.PhysicsParams(1.0, 0.01), idx, EXACT)
    assert np.array_equal(exact, ref)

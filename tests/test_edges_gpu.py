"""Edge cases of the engine on B200: empty and single-body inputs, zero softening in the
batched and adjoint kernels, run-to-run determinism, the device-only kick/drift entry points
and diagnostics on device arrays."""
import ctypes

import numpy as np
import pytest
import torch

import gx
import oracle
from gx import _ffi, adjoint
from conftest import rel_err

pytestmark = pytest.mark.gpu

F64, MIX, EXACT = gx.PRECISION_F64, gx.PRECISION_MIXED, gx.PRECISION_F64_EXACT
P = _ffi.ptr


def test_empty_inputs_are_no_ops():
    lib = _ffi.load()
    z = np.zeros(1)
    phys = _ffi.physics(1.0, 0.1)
    assert lib.gx_direct_accel(0, P(z), P(z), P(z), P(z), phys, F64, P(z), P(z), P(z), None) == 0
    assert lib.gx_direct_vjp(0, *(P(z) for _ in range(7)), phys, F64, *(P(z) for _ in range(4)), None) == 0
    assert lib.gx_p2p_leaves(0, *(P(z) for _ in range(4)), 0, None, None, None, None, phys, F64, P(z), P(z), P(z),
                             None) == 0
    d = _ffi.DiagnosticsStruct()
    assert lib.gx_diagnostics_compute(0, *(P(z) for _ in range(7)), phys, ctypes.byref(d), None) == 0
    assert d.total_mass == 0.0 and d.potential_energy == 0.0
    assert lib.gx_direct_accel_targets(5, P(np.zeros(5)), P(np.zeros(5)), P(np.zeros(5)), P(np.ones(5)), 2, 2, None, 0,
                                       phys, F64, P(z), P(z), P(z), None) == 0


@pytest.mark.parametrize("prec", [F64, MIX, EXACT])
def test_single_body_session(prec):
    p = gx.ParticleSet([0.3], [-0.2], [0.1], [1.0], [0.5], [0.0], [2.0])
    with gx.Session(1, gx.PhysicsParams(1.0, 0.05)) as s:
        s.set_particles(p)
        s.compute_accelerations(prec)
        s.step(3, 0.01, prec)
        st = s.get_state()
        d = s.diagnostics()
    assert st["ax"][0] == 0.0 and st["x"][0] == pytest.approx(0.3 + 3 * 0.01)
    assert d.potential_energy == 0.0 and d.kinetic_energy == pytest.approx(0.5 * 2.0 * 1.25)


@pytest.mark.parametrize("prec", [F64, MIX])
def test_batch_zero_softening(prec):
    parts = [gx.ics.two_disk_encounter(200, 200, 70 + i, 0.05) for i in range(3)]
    for q in parts:
        q.x[5], q.y[5], q.z[5] = q.x[6], q.y[6], q.z[6]  # a coincident pair in every instance
    off = np.array([0, 400, 800, 1200], np.int64)
    cat = lambda f: np.concatenate([getattr(q, f) for q in parts])
    a = np.stack(gx.batch_accelerations(off, cat("x"), cat("y"), cat("z"), cat("m"), gx.PhysicsParams(1.0, 0.0), prec), 1)
    assert np.all(np.isfinite(a))
    for b, q in enumerate(parts):
        ref = oracle.direct_targets(q.x, q.y, q.z, q.m, 1.0, 0.0)
        e = rel_err(a[off[b]:off[b + 1]], ref)
        assert np.median(e) <= (1e-13 if prec == F64 else 1e-5)


def test_vjp_zero_softening_skips_coincident_pairs():
    rng = np.random.default_rng(8)
    p = gx.ics.two_disk_encounter(150, 150, 9, 0.05)
    p.x[3], p.y[3], p.z[3] = p.x[4], p.y[4], p.z[4]
    lam = rng.normal(size=(300, 3))
    gpos, gm = oracle.direct_vjp(p.x, p.y, p.z, p.m, lam[:, 0], lam[:, 1], lam[:, 2], 1.0, 0.0)
    X = torch.tensor(np.stack([p.x, p.y, p.z]), device="cuda")
    GX, GM = adjoint.direct_vjp(X, torch.tensor(p.m, device="cuda"), torch.tensor(lam.T.copy(), device="cuda"),
                                gx.PhysicsParams(1.0, 0.0), F64)
    got = GX.t().cpu().numpy()
    assert np.all(np.isfinite(got))
    assert np.median(rel_err(got, gpos)) <= 1e-12


def first_variant(prec):
    for v in range(64):
        try:
            if "eps0" not in gx.describe_variant(prec, v):
                return v
        except gx.GxError:
            continue
    raise AssertionError("no variant")


@pytest.mark.parametrize("prec", [F64, MIX])
def test_repeated_runs_are_bitwise_identical(prec):
    p = gx.ics.two_disk_encounter(3000, 2500, 14, 0.02)
    out = []
    for _ in range(2):
        with gx.Session(len(p), gx.PhysicsParams(1.0, 0.02)) as s:
            s.set_particles(p)
            s.set_config(prec, first_variant(prec), 5)  # partial sums reduced in chunk order
            s.compute_accelerations(prec)
            s.step(7, 0.002, prec)
            out.append(s.get_state())
    for k in out[0]:
        assert np.array_equal(out[0][k], out[1][k]), k


def test_device_kick_drift_match_reference_rounding():
    rng = np.random.default_rng(3)
    n = 4097
    x, v, a = (rng.normal(size=(3, n)) for _ in range(3))
    X = torch.tensor(x, device="cuda")
    V = torch.tensor(v, device="cuda")
    A = torch.tensor(a, device="cuda")
    st = torch.cuda.current_stream().cuda_stream
    rows = lambda t: (t[0].data_ptr(), t[1].data_ptr(), t[2].data_ptr())
    _ffi.call("gx_kick_drift", n, *rows(X), *rows(V), *rows(A), 0.005, 0.01, st)
    vv = v + a * 0.005          # kick: v += a*dt (cpp/core/integrator.cpp:7-11)
    xx = x + vv * 0.01          # drift: x += v*dt (integrator.cpp:13-17)
    assert np.array_equal(V.cpu().numpy(), vv) and np.array_equal(X.cpu().numpy(), xx)
    _ffi.call("gx_kick", n, *rows(V), *rows(A), 0.005, st)
    _ffi.call("gx_drift", n, *rows(X), *rows(V), 0.01, st)
    vv = vv + a * 0.005
    xx = xx + vv * 0.01
    assert np.array_equal(V.cpu().numpy(), vv) and np.array_equal(X.cpu().numpy(), xx)
    host = np.zeros(4)
    assert _ffi.load().gx_kick(4, P(host), P(host), P(host), P(host), P(host), P(host), 0.1, None) == \
        gx.GX_ERR_INVALID_ARGUMENT


def test_diagnostics_on_device_arrays():
    p = gx.ics.two_disk_encounter(1000, 1000, 2, 0.03)
    T = {k: torch.tensor(getattr(p, k), device="cuda") for k in ("x", "y", "z", "vx", "vy", "vz", "m")}
    d = _ffi.DiagnosticsStruct()
    _ffi.call("gx_diagnostics_compute", len(p), *(T[k].data_ptr() for k in ("x", "y", "z", "vx", "vy", "vz", "m")),
              _ffi.physics(1.0, 0.03), ctypes.byref(d), torch.cuda.current_stream().cuda_stream)
    ref = oracle.diagnostics(p.x, p.y, p.z, p.vx, p.vy, p.vz, p.m, 1.0, 0.03)
    np.testing.assert_allclose(gx.Diagnostics.from_struct(d).as_row(), ref, rtol=1e-12, atol=1e-13)


def test_session_step_graph_cache_over_many_lengths():
    p = gx.ics.two_disk_encounter(300, 300, 19, 0.05)
    with gx.Session(len(p), gx.PhysicsParams(1.0, 0.05)) as s:
        s.set_particles(p)
        s.compute_accelerations(F64)
        for k in (1, 2, 33, 64, 5, 1, 70):
            s.step(k, 0.001, F64)
        st = s.get_state()
    q = p.copy()
    gx.compute_cuda_direct_accelerations(q, gx.PhysicsParams(1.0, 0.05), F64)
    for _ in range(176):
        gx.cuda_direct_leapfrog_step(q, 0.001, gx.PhysicsParams(1.0, 0.05), F64)
    assert np.max(np.abs(st["x"] - q.x)) <= 1e-12


@pytest.mark.parametrize("prec", [F64, MIX, EXACT])
def test_device_target_indices_out_of_range_give_nan(prec):
    """Device index arrays are not checked on the host: an entry outside [0, n) is never read
    through (no out-of-bounds access) and its row of the result is NaN; the other rows are
    the normal per-target sums."""
    p = gx.ics.two_disk_encounter(300, 300, 31, 0.05)
    n = len(p)
    d = {k: torch.from_numpy(getattr(p, k)).cuda() for k in ("x", "y", "z", "m")}
    idx = np.array([5, -1, 17, n, 599, -(2 ** 40), 0], np.int64)
    di = torch.from_numpy(idx).cuda()
    out = [torch.zeros(len(idx), dtype=torch.float64, device="cuda") for _ in range(3)]
    lib = _ffi.load()
    st = lib.gx_direct_accel_targets(n, *(d[k].data_ptr() for k in ("x", "y", "z", "m")), 0, 0, di.data_ptr(),
                                     len(idx), _ffi.physics(1.0, 0.05), prec, *(o.data_ptr() for o in out),
                                     torch.cuda.current_stream().cuda_stream)
    assert st == 0, _ffi.last_error()
    got = torch.stack(out, 1).cpu().numpy()
    bad = (idx < 0) | (idx >= n)
    assert np.all(np.isnan(got[bad]))
    ok = idx[~bad]
    want = oracle.direct_indexed(p.x, p.y, p.z, p.m, 1.0, 0.05, ok)
    e = rel_err(got[~bad], want)
    assert e.max() <= (0.0 if prec == EXACT else 1e-11 if prec == F64 else 1e-4)

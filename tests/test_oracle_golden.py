"""The oracle (oracle/gx_oracle.c) pinned against the reference's own outputs (CPU only).

Golden vectors: the reference's committed snapshots and diagnostics
(experiments/benchmarks/local_cpu/outputs/direct_*_r1, fmm_1000_r1) and the outputs of the
reference's sources compiled here (the smoke-test case of cpp/tests/smoke_tests.cpp:54-123,
a 20-step direct run, the FMM leaf lists); see tests/golden/make_golden.py.
"""
import numpy as np
import pytest

import oracle
from conftest import rel_err

STATE = ("x", "y", "z", "vx", "vy", "vz", "ax", "ay", "az")


def test_smoke80_direct_bitwise(golden):
    g = golden("smoke80.npz")
    a2 = oracle.direct_symmetric(g["x"], g["y"], g["z"], g["m"], 1.0, 0.03)
    a3 = oracle.direct_targets(g["x"], g["y"], g["z"], g["m"], 1.0, 0.03)
    assert np.array_equal(a2, g["a_direct"])
    assert np.array_equal(a3, g["a_targets"])
    # the two orders agree to rounding only (the reference KAT allows 1e-10 mean)
    assert rel_err(a3, a2).mean() < 1e-14


def test_two_body_zero_softening(golden):
    g = golden("smoke80.npz")
    a = oracle.direct_symmetric(g["two_body_x"], g["two_body_y"], g["two_body_z"], g["two_body_m"], 1.0, 0.0)
    assert np.array_equal(a, g["two_body_a"])
    assert a[0, 0] > 0 and a[1, 0] < 0
    assert abs(2.0 * a[0, 0] + 3.0 * a[1, 0]) < 1e-12  # smoke_tests.cpp:66-69


@pytest.mark.parametrize("name", ["direct_250_r1", "direct_1000_r1"])
def test_reference_snapshot_trajectory(golden, name):
    """20 KDK steps of the symmetric direct solver reproduce the reference's snapshot."""
    g = golden("direct_snapshots.npz")
    s0 = {k: g[f"{name}/s0/{k}"] for k in STATE}
    m = g[f"{name}/s0/m"]
    # step-0 accelerations are the reference's symmetric direct sum
    a0 = oracle.direct_symmetric(s0["x"], s0["y"], s0["z"], m, 1.0, 0.025)
    assert np.max(np.abs(a0 - np.stack([s0["ax"], s0["ay"], s0["az"]], 1))) <= 1e-13 * np.abs(a0).max()
    s20 = oracle.leapfrog(s0, m, 1.0, 0.025, 0.01, 20, solver=0)
    for k in STATE:
        ref = g[f"{name}/s20/{k}"]
        assert np.max(np.abs(s20[k] - ref)) <= 1e-12 * max(1.0, np.abs(ref).max()), k
    diag = g[f"{name}/diagnostics"]
    d0 = oracle.diagnostics(s0["x"], s0["y"], s0["z"], s0["vx"], s0["vy"], s0["vz"], m, 1.0, 0.025)
    d20 = oracle.diagnostics(*(s20[k] for k in STATE[:6]), m, 1.0, 0.025)
    np.testing.assert_allclose(d0, diag[0, 3:], rtol=1e-13, atol=1e-15)
    np.testing.assert_allclose(d20, diag[1, 3:], rtol=1e-12, atol=1e-15)


def test_cfg0_fixture_bitwise(golden):
    g = golden("cfg0_n1000.npz")
    eps, dt = float(g["softening"]), float(g["dt"])
    a0 = oracle.direct_symmetric(g["x0"], g["y0"], g["z0"], g["m"], 1.0, eps)
    assert np.array_equal(a0, g["a0"])
    st = dict(x=g["x0"], y=g["y0"], z=g["z0"], vx=g["vx0"], vy=g["vy0"], vz=g["vz0"], ax=a0[:, 0], ay=a0[:, 1], az=a0[:, 2])
    s20 = oracle.leapfrog(st, g["m"], 1.0, eps, dt, 20, solver=0)
    for k in STATE:
        assert np.array_equal(s20[k], g[f"{k}20"]), k
    d0 = oracle.diagnostics(g["x0"], g["y0"], g["z0"], g["vx0"], g["vy0"], g["vz0"], g["m"], 1.0, eps)
    assert np.array_equal(d0, g["diag0"])


def test_fmm_leaf_lists_and_p2p(golden):
    """Restated octree == the reference's tree; far field + restated P2P == reference FMM."""
    g = golden("fmm1000.npz")
    L = oracle.leaf_lists(g["x"], g["y"], g["z"], g["m"], float(g["softening"]), float(g["theta"]),
                          int(g["leaf_capacity"]))
    for k in ("leaf_offsets", "leaf_particles", "near_offsets", "near_leaves"):
        assert np.array_equal(L[k], g[k]), k
    acc = oracle.p2p_near(g["x"], g["y"], g["z"], g["m"], 1.0, float(g["softening"]), L, acc=g["far"])
    golden_acc = np.stack([g["ax"], g["ay"], g["az"]], 1)
    assert np.array_equal(acc, golden_acc)


def test_readme_run_diagnostics(golden):
    """experiments/validation/readme_1000_body_collision: the oracle's diagnostics of the
    reference's step-0 and step-10 states equal rows 0 and 10 of its diagnostics.csv, and
    (where the reference library is built) its FMM of the step-0 state equals the snapshot's
    accelerations."""
    g = golden("readme1000.npz")
    eps, diag = float(g["softening"]), g["diagnostics"]
    for k in (0, 10):
        d = oracle.diagnostics(*(g[f"{v}{k}"] for v in STATE[:6]), g["m"], 1.0, eps)
        np.testing.assert_allclose(d, diag[k, 3:], rtol=1e-13, atol=1e-15)
    if oracle.ref_available():
        theta, cap = float(g["theta"]), int(g["leaf_capacity"])
        a = oracle.ref_fmm(g["x0"], g["y0"], g["z0"], g["m"], 1.0, eps, theta, cap)
        assert np.array_equal(a, np.stack([g["ax0"], g["ay0"], g["az0"]], 1))
        # the reference's own KDK + FMM, rebuilt here, reproduces its published step 10 to a
        # few ulps (the run is chaotic: the gap grows about tenfold every 20 steps)
        s = oracle.ref_leapfrog_fmm({k: g[f"{k}0"] for k in STATE}, g["m"], 1.0, eps, float(g["dt"]), 10, theta, cap)
        assert max(np.abs(s[k] - g[f"{k}10"]).max() for k in STATE) <= 1e-15


@pytest.mark.skipif(not oracle.ref_available(), reason="reference library not built in this tree")
def test_oracle_vs_reference_random():
    rng = np.random.default_rng(11)
    n = 700
    x, y, z = rng.normal(size=(3, n))
    m = rng.uniform(0.5, 1.5, n) / n
    x[5], y[5], z[5] = x[9], y[9], z[9]  # a coincident pair
    for eps in (0.0, 0.01):
        a2o = oracle.direct_symmetric(x, y, z, m, 1.3, eps)
        a2r = oracle.ref_direct(x, y, z, m, 1.3, eps)
        assert np.array_equal(a2o, a2r)
        a3o = oracle.direct_targets(x, y, z, m, 1.3, eps, 100, 400)
        a3r = oracle.ref_direct_targets(x, y, z, m, 1.3, eps, 100, 400, threads=3)
        assert np.array_equal(a3o, a3r)
    v = rng.normal(size=(3, n))
    assert np.array_equal(oracle.diagnostics(x, y, z, *v, m, 1.0, 0.02), oracle.ref_diagnostics(x, y, z, *v, m, 1.0, 0.02))
    Lr, far = oracle.ref_fmm_split(x, y, z, m, 1.0, 0.02, 0.5, 8)
    Lo = oracle.leaf_lists(x, y, z, m, 0.02, 0.5, 8)
    for k in ("leaf_offsets", "leaf_particles", "near_offsets", "near_leaves"):
        assert np.array_equal(Lo[k], Lr[k]), k
    full = oracle.ref_fmm(x, y, z, m, 1.0, 0.02, 0.5, 8)
    assert np.array_equal(oracle.p2p_near(x, y, z, m, 1.0, 0.02, Lo, acc=far), full)


def test_vjp_oracle_finite_difference():
    rng = np.random.default_rng(3)
    n = 24
    x, y, z = rng.normal(size=(3, n))
    m = rng.uniform(0.5, 1.5, n)
    lam = rng.normal(size=(n, 3))
    eps = 0.1
    gpos, gm = oracle.direct_vjp(x, y, z, m, lam[:, 0], lam[:, 1], lam[:, 2], 1.0, eps)

    def L(xx, yy, zz, mm):
        return float(np.sum(lam * oracle.direct_targets(xx, yy, zz, mm, 1.0, eps)))

    h = 1e-6
    for k in (0, 7, 19):
        for c, arr in enumerate((x, y, z)):
            p, q = arr.copy(), arr.copy()
            p[k] += h
            q[k] -= h
            args_p = [x, y, z]
            args_q = [x, y, z]
            args_p[c], args_q[c] = p, q
            fd = (L(*args_p, m) - L(*args_q, m)) / (2 * h)
            assert abs(fd - gpos[k, c]) <= 1e-6 * max(1.0, abs(fd))
        mp, mq = m.copy(), m.copy()
        mp[k] += h
        mq[k] -= h
        fd = (L(x, y, z, mp) - L(x, y, z, mq)) / (2 * h)
        assert abs(fd - gm[k]) <= 1e-6 * max(1.0, abs(fd))


def test_ownership_ranges():
    # distributed_solver.cpp:68-79: contiguous ranges, remainder on the low ranks
    assert oracle.ownership(10, 0, 1) == (0, 10)
    assert [oracle.ownership(10, r, 3) for r in range(3)] == [(0, 4), (4, 7), (7, 10)]

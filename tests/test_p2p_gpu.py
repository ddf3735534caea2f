"""FMM near-field leaf kernel (B200) vs the reference FMM and the oracle.

The exact form started from the reference's far field reproduces the reference's FMM
accelerations (fmm_1000_r1 step 0) bit for bit; the FP64 form within 1e-12 relative.
"""
import numpy as np
import pytest
import torch

import gx
import oracle
from conftest import rel_err

pytestmark = pytest.mark.gpu

F64, MIX, EXACT = gx.PRECISION_F64, gx.PRECISION_MIXED, gx.PRECISION_F64_EXACT


def run_p2p(x, y, z, m, lists, eps, prec, far=None):
    a = [np.zeros(len(x)) for _ in range(3)] if far is None else [np.ascontiguousarray(far[:, c]).copy() for c in range(3)]
    gx.p2p_leaves(x, y, z, m, lists, gx.PhysicsParams(1.0, eps), a[0], a[1], a[2], prec)
    return np.stack(a, 1)


def test_reference_fmm_fixture(golden):
    g = golden("fmm1000.npz")
    eps = float(g["softening"])
    lists = gx.build_leaf_lists(g["x"], g["y"], g["z"], g["m"], eps, float(g["theta"]), int(g["leaf_capacity"]))
    ref = np.stack([g["ax"], g["ay"], g["az"]], 1)
    assert np.array_equal(run_p2p(g["x"], g["y"], g["z"], g["m"], lists, eps, EXACT, g["far"]), ref)
    assert rel_err(run_p2p(g["x"], g["y"], g["z"], g["m"], lists, eps, F64, g["far"]), ref).max() <= 1e-12
    assert np.median(rel_err(run_p2p(g["x"], g["y"], g["z"], g["m"], lists, eps, MIX, g["far"]), ref)) <= 1e-6


@pytest.mark.parametrize("n,cap,theta", [(20000, 64, 0.6), (5000, 16, 0.35), (3000, 300, 0.6)])
@pytest.mark.parametrize("prec", [F64, MIX, EXACT])
def test_near_field_vs_oracle(n, cap, theta, prec):
    p = gx.ics.two_disk_encounter(n // 2, n - n // 2, n + cap, 0.02)
    lists = gx.build_leaf_lists(p.x, p.y, p.z, p.m, 0.02, theta, cap)
    L = dict(leaf_offsets=lists.leaf_offsets, leaf_particles=lists.leaf_particles, near_offsets=lists.near_offsets,
             near_leaves=lists.near_leaves)
    ref = oracle.p2p_near(p.x, p.y, p.z, p.m, 1.0, 0.02, L)
    got = run_p2p(p.x, p.y, p.z, p.m, lists, 0.02, prec)
    if prec == EXACT:
        assert np.array_equal(got, ref)
    else:
        e = rel_err(got, ref)
        lim = (1e-13, 1e-11) if prec == F64 else (1e-6, 1e-4)
        assert np.median(e) <= lim[0] and e.max() <= lim[1], (np.median(e), e.max())


def test_zero_softening_and_deep_coincident_leaves():
    n = 600
    p = gx.ics.two_disk_encounter(300, 300, 13, 0.02)
    p.x[:40] = p.x[0]
    p.y[:40] = p.y[0]
    p.z[:40] = p.z[0]  # 40 coincident bodies end in one max-depth leaf
    lists = gx.build_leaf_lists(p.x, p.y, p.z, p.m, 0.0, 0.6, 8, max_depth=10)
    L = dict(leaf_offsets=lists.leaf_offsets, leaf_particles=lists.leaf_particles, near_offsets=lists.near_offsets,
             near_leaves=lists.near_leaves)
    ref = oracle.p2p_near(p.x, p.y, p.z, p.m, 1.0, 0.0, L)
    for prec in (F64, EXACT):
        got = run_p2p(p.x, p.y, p.z, p.m, lists, 0.0, prec)
        assert np.all(np.isfinite(got))
        if prec == EXACT:
            assert np.array_equal(got, ref)
        else:
            assert rel_err(got, ref).max() <= 1e-11


def window_lists(n, per_leaf, k, seed):
    """Synthetic leaf lists: the bodies in a random order cut into leaves of per_leaf, each
    leaf's near list the leaves within k of it, ascending."""
    perm = np.random.default_rng(seed).permutation(n).astype(np.int32)
    nl = (n + per_leaf - 1) // per_leaf
    lo = np.minimum(np.arange(nl + 1) * per_leaf, n).astype(np.int32)
    near = [np.arange(max(0, l - k), min(nl, l + k + 1), dtype=np.int32) for l in range(nl)]
    no = np.zeros(nl + 1, np.int32)
    no[1:] = np.cumsum([len(v) for v in near])
    return gx.LeafLists(lo, perm, no, np.concatenate(near))


@pytest.mark.parametrize("per_leaf,k", [(12, 900), (64, 150)])
def test_heavy_leaves_split_into_groups_and_chunks(per_leaf, k):
    """Leaves with ~20,000 sources each: the plan cuts them into target groups and source
    chunks (partial sums merged in chunk order), with one-warp blocks (12 bodies per leaf) and
    four-warp blocks (64 per leaf)."""
    n = 24000
    rng = np.random.default_rng(per_leaf)
    x, y, z = (rng.uniform(-1, 1, n) for _ in range(3))
    m = rng.uniform(0.5, 1.5, n) / n
    lists = window_lists(n, per_leaf, k, 7)
    L = dict(leaf_offsets=lists.leaf_offsets, leaf_particles=lists.leaf_particles, near_offsets=lists.near_offsets,
             near_leaves=lists.near_leaves)
    ref = oracle.p2p_near(x, y, z, m, 1.0, 0.02, L)
    assert np.array_equal(run_p2p(x, y, z, m, lists, 0.02, EXACT), ref)
    e = rel_err(run_p2p(x, y, z, m, lists, 0.02, F64), ref)
    assert np.median(e) <= 1e-13 and e.max() <= 1e-11
    e = rel_err(run_p2p(x, y, z, m, lists, 0.02, MIX), ref)
    assert np.median(e) <= 1e-6 and e.max() <= 1e-4


def test_host_lists_with_a_repeated_body_are_rejected():
    p = gx.ics.two_disk_encounter(500, 500, 29, 0.02)
    lists = gx.build_leaf_lists(p.x, p.y, p.z, p.m, 0.02, 0.6, 16)
    lp = lists.leaf_particles.copy()
    lp[5] = lp[0]
    bad = gx.LeafLists(lists.leaf_offsets, lp, lists.near_offsets, lists.near_leaves)
    with pytest.raises(gx.GxError, match="two leaf slots"):
        run_p2p(p.x, p.y, p.z, p.m, bad, 0.02, F64)


def test_device_arrays():
    p = gx.ics.two_disk_encounter(4000, 4000, 17, 0.02)
    lists = gx.build_leaf_lists(p.x, p.y, p.z, p.m, 0.02, 0.6, 64)
    host = run_p2p(p.x, p.y, p.z, p.m, lists, 0.02, F64)
    T = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
    dl = gx.LeafLists(T(lists.leaf_offsets), T(lists.leaf_particles), T(lists.near_offsets), T(lists.near_leaves))
    a = [torch.zeros(len(p), dtype=torch.float64, device="cuda") for _ in range(3)]
    gx.p2p_leaves(T(p.x), T(p.y), T(p.z), T(p.m), dl, gx.PhysicsParams(1.0, 0.02), *a, F64)
    torch.cuda.synchronize()
    assert np.array_equal(torch.stack(a, 1).cpu().numpy(), host)


def test_reference_fmm_split_random():
    if not oracle.ref_available():
        pytest.skip("reference library not built in this tree")
    p = gx.ics.two_disk_encounter(3000, 3000, 23, 0.02)
    L, far = oracle.ref_fmm_split(p.x, p.y, p.z, p.m, 1.0, 0.02, 0.6, 64)
    lists = gx.build_leaf_lists(p.x, p.y, p.z, p.m, 0.02, 0.6, 64)
    full = oracle.ref_fmm(p.x, p.y, p.z, p.m, 1.0, 0.02, 0.6, 64)
    assert np.array_equal(run_p2p(p.x, p.y, p.z, p.m, lists, 0.02, EXACT, far), full)


def test_fmm_trajectory_with_gpu_near_field(golden):
    """20 KDK steps of the reference's FMM solver with the near field on the GPU: every step
    rebuilds the tree, takes the far field from the reference's own code (oracle/_ref) and adds
    the engine's exact-form P2P.  The trajectory must equal the reference's pure-CPU FMM run bit
    for bit, and the reference's committed fmm_1000_r1 step-20 snapshot to 1e-12."""
    if not oracle.ref_available():
        pytest.skip("reference library not built in this tree")
    g = golden("fmm1000.npz")
    eps, theta, cap, dt = float(g["softening"]), float(g["theta"]), int(g["leaf_capacity"]), float(g["dt"])
    st = {k: np.array(g[k], dtype=np.float64) for k in ("x", "y", "z", "vx", "vy", "vz", "ax", "ay", "az")}
    m = g["m"]
    ref = oracle.ref_leapfrog_fmm(st, m, 1.0, eps, dt, int(g["steps"]), theta, cap)
    h = 0.5 * dt
    for _ in range(int(g["steps"])):
        for c in "xyz":  # kick(dt/2), drift(dt): cpp/core/integrator.cpp:7-17, same rounding
            st["v" + c] = st["v" + c] + st["a" + c] * h
        for c in "xyz":
            st[c] = st[c] + st["v" + c] * dt
        _, far = oracle.ref_fmm_split(st["x"], st["y"], st["z"], m, 1.0, eps, theta, cap)
        lists = gx.build_leaf_lists(st["x"], st["y"], st["z"], m, eps, theta, cap)
        acc = run_p2p(st["x"], st["y"], st["z"], m, lists, eps, EXACT, far)
        st["ax"], st["ay"], st["az"] = (np.ascontiguousarray(acc[:, c]) for c in range(3))
        for c in "xyz":
            st["v" + c] = st["v" + c] + st["a" + c] * h
    for k in st:
        assert np.array_equal(st[k], ref[k]), k
        want = g[f"{k}20"]
        assert np.max(np.abs(st[k] - want)) <= 1e-12 * max(1.0, np.abs(want).max()), k


@pytest.fixture
def p2p_shape():
    """Forces the P2P kernel's targets per thread for one test, then restores the default."""
    def force(tpt):
        gx._ffi.call("gx_debug_p2p_targets_per_thread", tpt)
    yield force
    gx._ffi.call("gx_debug_p2p_targets_per_thread", 0)


@pytest.mark.parametrize("tpt", [2, 4])
@pytest.mark.parametrize("n,cap,theta,eps", [(20000, 64, 0.6, 0.02), (6000, 16, 0.5, 0.02), (3000, 200, 0.6, 0.02),
                                             (2000, 32, 0.6, 0.0)])
@pytest.mark.parametrize("prec", [F64, MIX])
def test_near_field_both_thread_shapes(p2p_shape, tpt, n, cap, theta, eps, prec):
    """Two and four targets per thread (rows of a leaf's targets; the mixed form packs target
    pairs into f32x2 lanes) give the oracle's near field within each form's tolerance, with
    one-warp and four-warp blocks (small and large leaves), split leaves and zero softening."""
    p = gx.ics.two_disk_encounter(n // 2, n - n // 2, n + cap + tpt, 0.02)
    if eps == 0.0:
        p.x[7], p.y[7], p.z[7] = p.x[8], p.y[8], p.z[8]
    lists = gx.build_leaf_lists(p.x, p.y, p.z, p.m, eps, theta, cap)
    L = dict(leaf_offsets=lists.leaf_offsets, leaf_particles=lists.leaf_particles, near_offsets=lists.near_offsets,
             near_leaves=lists.near_leaves)
    ref = oracle.p2p_near(p.x, p.y, p.z, p.m, 1.0, eps, L)
    p2p_shape(tpt)
    got = run_p2p(p.x, p.y, p.z, p.m, lists, eps, prec)
    assert np.all(np.isfinite(got))
    e = rel_err(got, ref)
    lim = (1e-13, 1e-11) if prec == F64 else (1e-6, 1e-4)
    assert np.median(e) <= lim[0] and e.max() <= lim[1], (np.median(e), e.max())

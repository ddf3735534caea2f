"""Disk initial conditions (cpp/core/initial_conditions.cpp:37-114).

CPU: the oracle's restatement of the disk model (fed the engine's counter-based draws)
follows the same distributions as the reference's own generator (mt19937_64).  GPU: the
device generator equals the restatement body for body."""
import numpy as np
import pytest

import gx
import oracle

need_ref = pytest.mark.skipif(not oracle.ref_available(), reason="reference build absent")

GALAXIES = [
    dict(n_particles=120000, mass=1.0, radius=1.0, thickness=0.05, orientation=0.3, inclination=0.0, group_id=0),
    dict(n_particles=80000, mass=0.25, radius=0.6, position=(6.0, 1.5, -0.5), velocity=(-0.4, 0.1, 0.05),
         orientation=1.1, inclination=0.7, thickness=0.02, group_id=1),
    dict(n_particles=0, mass=1.0, radius=1.0),       # makes no bodies (initial_conditions.cpp:46-48)
    dict(n_particles=10, mass=-1.0, radius=1.0),
]


def frame(d, g):
    """Body positions and velocities in the galaxy's own disk frame (rotations undone)."""
    ci, si = np.cos(g.get("inclination", 0.0)), np.sin(g.get("inclination", 0.0))
    co, so = np.cos(g.get("orientation", 0.0)), np.sin(g.get("orientation", 0.0))
    Rz = np.array([[co, -so, 0], [so, co, 0], [0, 0, 1]])
    Rx = np.array([[1, 0, 0], [0, ci, -si], [0, si, ci]])
    R = Rz @ Rx
    p = np.stack([d["x"], d["y"], d["z"]], 1) - np.array(g.get("position", (0, 0, 0)))
    v = np.stack([d["vx"], d["vy"], d["vz"]], 1) - np.array(g.get("velocity", (0, 0, 0)))
    return p @ R, v @ R


@need_ref
def test_restatement_follows_reference_distributions():
    eps = 0.02
    ref = oracle.ref_generate_galaxies(GALAXIES, 1.0, eps, 20260502)
    ours = oracle.generate_galaxies(GALAXIES, 1.0, eps, 99)
    assert len(ref["x"]) == len(ours["x"]) == 200000
    assert np.array_equal(ref["m"], ours["m"]) and np.array_equal(ref["group_id"], ours["group_id"])
    off = 0
    for g in GALAXIES[:2]:
        n = g["n_particles"]
        sl = slice(off, off + n)
        off += n
        (pr, vr), (po, vo) = (frame({k: v[sl] for k, v in d.items()}, g) for d in (ref, ours))
        rr, ro = np.hypot(pr[:, 0], pr[:, 1]), np.hypot(po[:, 0], po[:, 1])
        R = g["radius"]
        # radius: truncated exponential of scale R/3 -> quantiles agree to sampling error
        for q in (0.1, 0.25, 0.5, 0.75, 0.9, 0.99):
            assert abs(np.quantile(rr, q) - np.quantile(ro, q)) < 0.01 * R, q
        assert rr.max() <= R and ro.max() <= R
        # height ~ N(0, thickness^2); in-plane angle uniform
        assert abs(pr[:, 2].std() - po[:, 2].std()) < 0.02 * g["thickness"]
        assert abs(np.mean(np.cos(np.arctan2(po[:, 1], po[:, 0])))) < 0.01
        # tangential speed profile and dispersion
        vt = lambda p, v: (p[:, 0] * v[:, 1] - p[:, 1] * v[:, 0]) / np.hypot(p[:, 0], p[:, 1])
        bins = np.quantile(rr, np.linspace(0, 1, 11))
        for lo_, hi_ in zip(bins[:-1], bins[1:]):
            a, b = (rr >= lo_) & (rr < hi_), (ro >= lo_) & (ro < hi_)
            assert abs(vt(pr[a], vr[a]).mean() - vt(po[b], vo[b]).mean()) < 0.01 * np.sqrt(g["mass"] / R)
        assert abs(vr[:, 2].std() - vo[:, 2].std()) < 0.05 * vr[:, 2].std()


@pytest.mark.gpu
def test_device_generator_equals_restatement():
    import torch
    eps = 0.02
    params = gx.PhysicsParams(1.0, eps)
    want = oracle.generate_galaxies(GALAXIES, 1.0, eps, 12345)
    got = gx.ics.generate_galaxies(GALAXIES, params, 12345)
    for f in ("x", "y", "z", "vx", "vy", "vz"):
        np.testing.assert_allclose(getattr(got, f), want[f], rtol=1e-12, atol=1e-13, err_msg=f)
    assert np.array_equal(got.m, want["m"]) and np.array_equal(got.group_id, want["group_id"])
    dev = gx.ics.generate_galaxies(GALAXIES, params, 12345, device="cuda")
    torch.cuda.synchronize()
    for f in ("x", "y", "z", "vx", "vy", "vz", "m"):
        assert np.array_equal(dev[f].cpu().numpy(), getattr(got, f)), f


@pytest.mark.gpu
def test_galaxy_bodies_do_not_depend_on_other_galaxies():
    params = gx.PhysicsParams(1.0, 0.02)
    a = [dict(GALAXIES[0], n_particles=1000), GALAXIES[1]]
    b = [dict(GALAXIES[0], n_particles=3333), GALAXIES[1]]
    pa, pb = (gx.ics.generate_galaxies(g, params, 7) for g in (a, b))
    assert np.array_equal(pa.x[1000:], pb.x[3333:]) and np.array_equal(pa.vz[1000:], pb.vz[3333:])
    assert np.array_equal(pa.x[:1000], pb.x[:1000])
    pc = gx.ics.generate_galaxies(a, params, 8)
    assert not np.array_equal(pa.x, pc.x)

"""Seeded two-disk encounter initial conditions.

The workloads are specified as: each disk draws radii from an exponential surface density
(scale length 1, truncated at 5), heights from N(0, 0.05^2), and circular speeds from the
enclosed mass of the sampled disk with softening; disk 1 sits at the origin at rest, disk 2
at (10, b, 0) moving at (-0.5, 0, 0) and inclined about x.

This is not the reference generator (cpp/core/initial_conditions.cpp:28-114 uses scale
radius/3, a uniform-disk enclosed fraction and a 2.5% velocity dispersion), whose
parameters cannot express these disks.  Parity is therefore always taken on identical
particle arrays fed to both the reference and the engine.  The RNG is numpy's PCG64 seeded
with `seed`; draws happen disk by disk in the order radius, angle, height.
"""
from __future__ import annotations

import numpy as np

from .engine import ParticleSet


def _truncated_exponential_radii(u: np.ndarray, scale: float, rmax: float) -> np.ndarray:
    """Inverse CDF of p(r) ~ r exp(-r/scale) on [0, rmax], by bisection (exact to 2^-55 rmax)."""
    cdf = lambda r: 1.0 - (1.0 + r / scale) * np.exp(-r / scale)
    target = u * cdf(rmax)
    lo = np.zeros_like(u)
    hi = np.full_like(u, rmax)
    for _ in range(56):
        mid = 0.5 * (lo + hi)
        below = cdf(mid) < target
        lo = np.where(below, mid, lo)
        hi = np.where(below, hi, mid)
    return 0.5 * (lo + hi)


def exponential_disk(n: int, mass: float, rng: np.random.Generator, softening: float, G: float = 1.0,
                     scale: float = 1.0, rmax: float = 5.0, sigma_z: float = 0.05):
    """Positions (n,3), velocities (n,3), masses (n,) of one face-on disk centred at 0."""
    if n <= 0:
        return np.zeros((0, 3)), np.zeros((0, 3)), np.zeros(0)
    r = _truncated_exponential_radii(rng.random(n), scale, rmax)
    th = 2.0 * np.pi * rng.random(n)
    z = sigma_z * rng.standard_normal(n)
    m = np.full(n, mass / n)
    # enclosed mass of the sampled disk: bodies at radius <= r (itself included)
    rank = np.empty(n)
    rank[np.argsort(r, kind="stable")] = np.arange(1, n + 1)
    menc = rank * (mass / n)
    vc = np.sqrt(G * menc * r * r / (r * r + softening * softening) ** 1.5)
    pos = np.stack([r * np.cos(th), r * np.sin(th), z], 1)
    vel = np.stack([-np.sin(th) * vc, np.cos(th) * vc, np.zeros(n)], 1)
    return pos, vel, m


def _rot_x(deg: float) -> np.ndarray:
    a = np.deg2rad(deg)
    c, s = np.cos(a), np.sin(a)
    return np.array([[1.0, 0.0, 0.0], [0.0, c, -s], [0.0, s, c]])


def two_disk_encounter(n1: int, n2: int, seed: int, softening: float, mass1: float = 1.0,
                       mass2: float = 1.0, separation: float = 10.0, impact: float = 2.0,
                       approach_speed: float = 0.5, inclination_deg: float = 30.0,
                       G: float = 1.0) -> ParticleSet:
    """Disk 1 at rest at the origin; disk 2 at (separation, impact, 0) with velocity
    (-approach_speed, 0, 0), rotated by inclination_deg about x."""
    rng = np.random.Generator(np.random.PCG64(seed))
    p1, v1, m1 = exponential_disk(n1, mass1, rng, softening, G)
    p2, v2, m2 = exponential_disk(n2, mass2, rng, softening, G)
    R = _rot_x(inclination_deg)
    p2 = p2 @ R.T + np.array([separation, impact, 0.0])
    v2 = v2 @ R.T + np.array([-approach_speed, 0.0, 0.0])
    pos = np.concatenate([p1, p2])
    vel = np.concatenate([v1, v2])
    m = np.concatenate([m1, m2])
    gid = np.concatenate([np.zeros(n1, np.uint32), np.ones(n2, np.uint32)])
    return ParticleSet.from_arrays(pos, vel, m, group_id=gid)


# The workloads (sizes, softening, step) of the benchmark configurations.
WORKLOADS = {
    "direct-n1000-f64": dict(n1=500, n2=500, mass1=1.0, mass2=1.0, softening=0.05, dt=0.005, steps=20),
    "direct-n65536": dict(n1=32768, n2=32768, mass1=1.0, mass2=1.0, softening=0.02, dt=0.002, steps=100),
    "mixed-n1048576": dict(n1=524288, n2=524288, mass1=1.0, mass2=1.0 / 3.0, softening=0.01, dt=0.001, steps=10),
}


def workload(name: str, seed: int = 20260502) -> tuple[ParticleSet, dict]:
    w = dict(WORKLOADS[name])
    p = two_disk_encounter(w["n1"], w["n2"], seed, w["softening"], w["mass1"], w["mass2"])
    return p, w


def ensemble(n_instances: int = 512, seed: int = 7, n_min: int = 1024, n_max: int = 16384,
             softening: float = 0.05):
    """Independent encounters: N ~ U[n_min, n_max] (even, two equal-count disks), mass ratio
    ~ U[1, 10] (disk 2 lighter), impact parameter ~ U[0.5, 4], inclination ~ U[0, 90] deg.
    Returns (offsets, ParticleSet of the concatenation, per-instance parameter dict)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    sizes = 2 * rng.integers(n_min // 2, n_max // 2 + 1, n_instances)
    ratio = rng.uniform(1.0, 10.0, n_instances)
    impact = rng.uniform(0.5, 4.0, n_instances)
    incl = rng.uniform(0.0, 90.0, n_instances)
    seeds = rng.integers(0, 2**62, n_instances)
    parts = []
    for b in range(n_instances):
        h = int(sizes[b]) // 2
        parts.append(two_disk_encounter(h, h, int(seeds[b]), softening, 1.0, 1.0 / ratio[b], impact=impact[b],
                                        inclination_deg=incl[b]))
    offsets = np.zeros(n_instances + 1, np.int64)
    offsets[1:] = np.cumsum(sizes)
    cat = lambda f: np.concatenate([getattr(p, f) for p in parts])
    ps = ParticleSet(cat("x"), cat("y"), cat("z"), cat("vx"), cat("vy"), cat("vz"), cat("m"),
                     group_id=cat("group_id"))
    return offsets, ps, dict(sizes=sizes, mass_ratio=ratio, impact=impact, inclination_deg=incl)


def _galaxy_struct(g: dict):
    from . import _ffi
    gs = _ffi.GalaxyStruct()
    gs.n_particles = int(g["n_particles"])
    gs.mass = float(g["mass"])
    gs.radius = float(g["radius"])
    gs.position[:] = [float(v) for v in g.get("position", (0.0, 0.0, 0.0))]
    gs.velocity[:] = [float(v) for v in g.get("velocity", (0.0, 0.0, 0.0))]
    gs.orientation = float(g.get("orientation", 0.0))
    gs.group_id = int(g.get("group_id", 0))
    gs.thickness = float(g.get("thickness", 0.0))
    gs.inclination = float(g.get("inclination", 0.0))
    return gs


def generate_galaxies(galaxies, params, seed: int, device=None, stream=None):
    """The reference's generate_galaxies (cpp/core/initial_conditions.cpp:92-114) computed on
    the GPU: each galaxy is a dict of GalaxyConfig fields (n_particles, mass, radius,
    position, velocity, orientation, group_id, thickness, inclination).  Returns a
    ParticleSet (host) or, with device="cuda", a dict of CUDA tensors.  Same disk model as
    the reference; the random numbers come from a counter-based generator, so the bodies
    differ from the reference's mt19937_64 draws but follow the same distributions."""
    import ctypes
    from . import _ffi
    from .engine import ParticleSet
    arr = (_ffi.GalaxyStruct * max(1, len(galaxies)))(*[_galaxy_struct(g) for g in galaxies])
    n = int(_ffi.load().gx_galaxies_body_count(len(galaxies), ctypes.addressof(arr)))
    fields = ("x", "y", "z", "vx", "vy", "vz", "m")
    if device is not None:
        import torch
        out = {f: torch.empty(n, dtype=torch.float64, device=device) for f in fields}
        grp = torch.empty(n, dtype=torch.int32, device=device)
        _ffi.call("gx_generate_galaxies", len(galaxies), ctypes.addressof(arr), params.ffi(), int(seed),
                  *(out[f].data_ptr() for f in fields), grp.data_ptr(), _ffi.stream_ptr(stream))
        out["group_id"] = grp
        return out
    out = {f: np.zeros(n) for f in fields}
    grp = np.zeros(n, np.uint32)
    if n:
        _ffi.call("gx_generate_galaxies", len(galaxies), ctypes.addressof(arr), params.ffi(), int(seed),
                  *(out[f].ctypes.data for f in fields), grp.ctypes.data, _ffi.stream_ptr(stream))
    p = ParticleSet(x=out["x"], y=out["y"], z=out["z"], vx=out["vx"], vy=out["vy"], vz=out["vz"], m=out["m"])
    p.group_id = grp
    return p


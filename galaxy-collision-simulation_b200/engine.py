"""Host-side mirror of the reference's solver interface for the direct path.

Same names, argument meaning and error behaviour as ryan-charette/galaxy-collision-simulation:

* ``cuda_solver_available()``                    -- cpp/cuda/cuda_solver.cu:185-189
* ``compute_cuda_direct_accelerations(p, params)`` -- cpp/cuda/cuda_solver.cu:191-210
* ``compute_direct_accelerations_for_targets``    -- cpp/direct/direct_solver.cpp:59-83
* ``cuda_direct_leapfrog_step(p, dt, params)``    -- cpp/cuda/cuda_solver.cu:212-246
* ``compute_diagnostics(p, params)``              -- cpp/core/diagnostics.cpp:7-37

Differences, by design: the state is structure-of-arrays (``ParticleSet``; the reference's
88-byte ``Particle`` records convert with ``ParticleSet.from_records``/``to_records``), errors
raise ``GxError`` (a ``RuntimeError``, as the reference throws ``std::runtime_error``), and
there is no silent CPU fallback: without a CUDA device every call raises.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

from . import _ffi
from ._ffi import PRECISION_F64, ptr

# The reference Particle (cpp/core/particle.hpp:8-14): Vec3 position, velocity,
# acceleration; double mass; uint32 group_id; padded to 88 bytes.
PARTICLE_DTYPE = np.dtype(
    {
        "names": ["position", "velocity", "acceleration", "mass", "group_id"],
        "formats": [("<f8", 3), ("<f8", 3), ("<f8", 3), "<f8", "<u4"],
        "offsets": [0, 24, 48, 72, 80],
        "itemsize": 88,
    }
)


@dataclass
class PhysicsParams:
    """PhysicsParams (cpp/core/simulation_params.hpp:5-8)."""

    gravitational_constant: float = 1.0
    softening: float = 0.02

    def ffi(self) -> _ffi.Physics:
        return _ffi.physics(self.gravitational_constant, self.softening)


@dataclass
class Diagnostics:
    """Diagnostics (cpp/core/diagnostics.hpp:11-19)."""

    kinetic_energy: float = 0.0
    potential_energy: float = 0.0
    total_energy: float = 0.0
    total_mass: float = 0.0
    momentum: tuple = (0.0, 0.0, 0.0)
    center_of_mass: tuple = (0.0, 0.0, 0.0)
    angular_momentum: tuple = (0.0, 0.0, 0.0)

    @classmethod
    def from_struct(cls, d: _ffi.DiagnosticsStruct) -> "Diagnostics":
        return cls(**_ffi.diagnostics_dict(d))

    def as_row(self) -> list[float]:
        """The 13 values of a diagnostics.csv row after step, time, n."""
        return [self.total_mass, self.kinetic_energy, self.potential_energy, self.total_energy,
                *self.momentum, *self.center_of_mass, *self.angular_momentum]


def _f64(a, n):
    a = np.ascontiguousarray(a, dtype=np.float64)
    if a.shape != (n,):
        raise ValueError(f"expected shape ({n},), got {a.shape}")
    return a


@dataclass
class ParticleSet:
    """Structure-of-arrays particle state (FP64)."""

    x: np.ndarray
    y: np.ndarray
    z: np.ndarray
    vx: np.ndarray
    vy: np.ndarray
    vz: np.ndarray
    m: np.ndarray
    ax: np.ndarray = None
    ay: np.ndarray = None
    az: np.ndarray = None
    group_id: np.ndarray = field(default=None)

    def __post_init__(self):
        n = len(self.x)
        for name in ("x", "y", "z", "vx", "vy", "vz", "m"):
            setattr(self, name, _f64(getattr(self, name), n))
        for name in ("ax", "ay", "az"):
            v = getattr(self, name)
            setattr(self, name, np.zeros(n) if v is None else _f64(v, n))
        self.group_id = np.zeros(n, np.uint32) if self.group_id is None else np.asarray(self.group_id, np.uint32)

    def __len__(self):
        return len(self.x)

    @classmethod
    def from_arrays(cls, pos, vel, mass, acc=None, group_id=None) -> "ParticleSet":
        pos = np.asarray(pos, np.float64)
        vel = np.asarray(vel, np.float64)
        acc = None if acc is None else np.asarray(acc, np.float64)
        return cls(pos[:, 0], pos[:, 1], pos[:, 2], vel[:, 0], vel[:, 1], vel[:, 2], mass,
                   None if acc is None else acc[:, 0], None if acc is None else acc[:, 1],
                   None if acc is None else acc[:, 2], group_id)

    @classmethod
    def from_records(cls, rec: np.ndarray) -> "ParticleSet":
        rec = np.asarray(rec, PARTICLE_DTYPE)
        return cls.from_arrays(rec["position"], rec["velocity"], rec["mass"], rec["acceleration"], rec["group_id"])

    def to_records(self) -> np.ndarray:
        rec = np.zeros(len(self), PARTICLE_DTYPE)
        rec["position"] = self.positions
        rec["velocity"] = self.velocities
        rec["acceleration"] = self.accelerations
        rec["mass"] = self.m
        rec["group_id"] = self.group_id
        return rec

    @property
    def positions(self):
        return np.stack([self.x, self.y, self.z], 1)

    @property
    def velocities(self):
        return np.stack([self.vx, self.vy, self.vz], 1)

    @property
    def accelerations(self):
        return np.stack([self.ax, self.ay, self.az], 1)

    def copy(self) -> "ParticleSet":
        return ParticleSet(*(np.copy(getattr(self, f)) for f in
                             ("x", "y", "z", "vx", "vy", "vz", "m", "ax", "ay", "az", "group_id")))


def cuda_solver_available() -> bool:
    """True when a compute-capability-10.0 device is usable."""
    return _ffi.device_available()


def compute_cuda_direct_accelerations(particles: ParticleSet, params: PhysicsParams,
                                      precision=PRECISION_F64) -> None:
    """Overwrites particles' accelerations with the direct sum (in place, like the reference)."""
    n = len(particles)
    if n == 0:
        return
    _ffi.call("gx_direct_accel", n, ptr(particles.x), ptr(particles.y), ptr(particles.z), ptr(particles.m),
              params.ffi(), _ffi.precision_code(precision), ptr(particles.ax), ptr(particles.ay),
              ptr(particles.az), None)


def compute_direct_accelerations_for_targets(particles: ParticleSet, params: PhysicsParams, begin: int,
                                             end: int, precision=PRECISION_F64) -> None:
    """Accelerations of targets [begin, min(end, n)) against all bodies, written in place."""
    n = len(particles)
    end = min(end, n)
    if begin >= end:
        return
    out = [np.zeros(end - begin) for _ in range(3)]
    _ffi.call("gx_direct_accel_targets", n, ptr(particles.x), ptr(particles.y), ptr(particles.z),
              ptr(particles.m), begin, end, None, 0, params.ffi(), _ffi.precision_code(precision),
              ptr(out[0]), ptr(out[1]), ptr(out[2]), None)
    particles.ax[begin:end], particles.ay[begin:end], particles.az[begin:end] = out


def cuda_direct_leapfrog_step(particles: ParticleSet, dt: float, params: PhysicsParams,
                              precision=PRECISION_F64) -> None:
    """One kick-drift-kick step in place, reusing the stored accelerations for the first kick."""
    n = len(particles)
    if n == 0:
        return
    p = particles
    _ffi.call("gx_leapfrog_step", n, ptr(p.x), ptr(p.y), ptr(p.z), ptr(p.vx), ptr(p.vy), ptr(p.vz),
              ptr(p.ax), ptr(p.ay), ptr(p.az), ptr(p.m), float(dt), params.ffi(),
              _ffi.precision_code(precision), None)


def compute_diagnostics(particles: ParticleSet, params: PhysicsParams) -> Diagnostics:
    """FP64 energy, momentum, centre of mass and angular momentum on the device."""
    d = _ffi.DiagnosticsStruct()
    p = particles
    _ffi.call("gx_diagnostics_compute", len(p), ptr(p.x), ptr(p.y), ptr(p.z), ptr(p.vx), ptr(p.vy),
              ptr(p.vz), ptr(p.m), params.ffi(), _ffi.ctypes.byref(d), None)
    return Diagnostics.from_struct(d)


def indexed_accelerations(particles: ParticleSet, params: PhysicsParams, targets,
                          precision=PRECISION_F64) -> np.ndarray:
    """Accelerations of an explicit target list, shape (len(targets), 3)."""
    t = np.ascontiguousarray(targets, dtype=np.int64)
    out = [np.zeros(len(t)) for _ in range(3)]
    _ffi.call("gx_direct_accel_targets", len(particles), ptr(particles.x), ptr(particles.y), ptr(particles.z),
              ptr(particles.m), 0, 0, ptr(t), len(t), params.ffi(), _ffi.precision_code(precision),
              ptr(out[0]), ptr(out[1]), ptr(out[2]), None)
    return np.stack(out, 1)

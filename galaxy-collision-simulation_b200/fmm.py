"""The reference FMM solver on the GPU.

Mirrors cpp/fmm/fmm_solver.hpp: ``FmmOptions`` (:15-20), ``FmmStats`` (:22-27),
``FastMultipoleSolver`` with ``compute`` / ``compute_targets`` / ``stats`` (:29-37), and the
free functions ``compute_fmm_accelerations`` / ``compute_fmm_accelerations_for_targets``
(fmm_solver.cpp:315-333).  The octree and its interaction lists are the reference's, built
on the host; moments, the multipole far field and the P2P near field run on the device
through ``gx_fmm_accel``.  Accelerations are written in place into the particle set, only
for the target range, as the reference does.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass

from . import _ffi
from ._ffi import PRECISION_F64, ptr
from .engine import ParticleSet, PhysicsParams


@dataclass
class FmmOptions:
    theta: float = 0.6
    leaf_capacity: int = 16
    max_depth: int = 32
    expansion_order: int = 4

    def ffi(self) -> _ffi.FmmOptionsStruct:
        return _ffi.FmmOptionsStruct(float(self.theta), int(self.leaf_capacity), int(self.max_depth),
                                     int(self.expansion_order))


@dataclass
class FmmStats:
    """FmmStats of the reference, plus the body-pair counts of the far and near fields and
    the number of tree levels."""
    node_count: int = 0
    leaf_count: int = 0
    far_interactions: int = 0
    near_interactions: int = 0
    far_pairs: int = 0
    near_pairs: int = 0
    tree_levels: int = 0


PHASES = ("tree", "moments", "lists", "far_field", "near_field")


def fmm_accelerations(x, y, z, m, ax, ay, az, params: PhysicsParams, options: FmmOptions | None = None,
                      precision=PRECISION_F64, begin: int = 0, end: int | None = None, stream=None) -> FmmStats:
    """Array form: host numpy or device torch arrays; writes (ax, ay, az)[begin:end]."""
    options = options or FmmOptions()
    n = len(x)
    st = _ffi.FmmStatsStruct()
    _ffi.call("gx_fmm_accel", n, ptr(x), ptr(y), ptr(z), ptr(m), params.ffi(), options.ffi(),
              _ffi.precision_code(precision), int(begin), int(n if end is None else end), ptr(ax), ptr(ay), ptr(az),
              ctypes.byref(st), _ffi.stream_ptr(stream))
    return _stats(st)


def _stats(st) -> FmmStats:
    return FmmStats(st.node_count, st.leaf_count, st.far_interactions, st.near_interactions, st.far_pairs,
                    st.near_pairs, st.tree_levels)


def fmm_accelerations_timed(x, y, z, m, ax, ay, az, params: PhysicsParams, options: FmmOptions | None = None,
                            precision=PRECISION_F64, begin: int = 0, end: int | None = None, stream=None):
    """fmm_accelerations plus {phase: device milliseconds} for PHASES (synchronizes)."""
    options = options or FmmOptions()
    n = len(x)
    st = _ffi.FmmStatsStruct()
    ms = (ctypes.c_double * len(PHASES))()
    _ffi.call("gx_fmm_accel_timed", n, ptr(x), ptr(y), ptr(z), ptr(m), params.ffi(), options.ffi(),
              _ffi.precision_code(precision), int(begin), int(n if end is None else end), ptr(ax), ptr(ay), ptr(az),
              ctypes.byref(st), _ffi.stream_ptr(stream), ctypes.addressof(ms))
    return _stats(st), dict(zip(PHASES, list(ms)))


class FastMultipoleSolver:
    """FastMultipoleSolver(params, options) with compute / compute_targets / stats."""

    def __init__(self, params: PhysicsParams, options: FmmOptions | None = None, precision=PRECISION_F64):
        self.params = params
        self.options = options or FmmOptions()
        self.precision = precision
        self._stats = FmmStats()

    def compute(self, particles: ParticleSet) -> None:
        self.compute_targets(particles, 0, len(particles))

    def compute_targets(self, particles: ParticleSet, begin: int, end: int) -> None:
        p = particles
        self._stats = fmm_accelerations(p.x, p.y, p.z, p.m, p.ax, p.ay, p.az, self.params, self.options,
                                        self.precision, begin, end)

    def stats(self) -> FmmStats:
        return self._stats


def compute_fmm_accelerations(particles: ParticleSet, params: PhysicsParams, options: FmmOptions | None = None,
                              precision=PRECISION_F64) -> None:
    FastMultipoleSolver(params, options, precision).compute(particles)


def compute_fmm_accelerations_for_targets(particles: ParticleSet, params: PhysicsParams, begin: int, end: int,
                                          options: FmmOptions | None = None, precision=PRECISION_F64) -> None:
    FastMultipoleSolver(params, options, precision).compute_targets(particles, begin, end)

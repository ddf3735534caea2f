"""FMM near-field leaves on the GPU.

``LeafLists`` holds the reference octree's leaf lists as CSR arrays (built on the host by
the engine, FastMultipoleSolver::build semantics, cpp/fmm/fmm_solver.cpp:48-98,210-277);
``p2p_leaves`` adds the P2P near field of evaluate_particle (:295-310) to accelerations
that already hold the far field.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass

import numpy as np

from . import _ffi
from ._ffi import PRECISION_F64, ptr
from .engine import PhysicsParams


@dataclass
class LeafLists:
    leaf_offsets: np.ndarray    # int32, n_leaves + 1
    leaf_particles: np.ndarray  # int32, body indices grouped by leaf (ascending within a leaf)
    near_offsets: np.ndarray    # int32, n_leaves + 1
    near_leaves: np.ndarray     # int32, leaf ids
    n_far: int = 0
    n_pairs: int = 0
    built_on_device: bool = False

    @property
    def n_leaves(self) -> int:
        return len(self.leaf_offsets) - 1


def build_leaf_lists(x, y, z, m, softening: float, theta: float = 0.6, leaf_capacity: int = 16,
                     max_depth: int = 32, on_device: bool = False) -> LeafLists:
    """Leaf lists of the reference octree, built on the host or (on_device) on the GPU;
    ``on_device`` sets ``LeafLists.built_on_device`` to what actually ran (trees deeper
    than 21 levels are always built on the host)."""
    xs = [np.ascontiguousarray(a, np.float64) for a in (x, y, z, m)]
    h = ctypes.c_void_p()
    where = ctypes.c_int(0)
    if on_device:
        _ffi.call("gx_leaf_lists_build_device", len(xs[0]), *(ptr(a) for a in xs), float(softening), float(theta),
                  int(leaf_capacity), int(max_depth), None, ctypes.byref(h), ctypes.byref(where))
    else:
        _ffi.call("gx_leaf_lists_build", len(xs[0]), *(ptr(a) for a in xs), float(softening), float(theta),
                  int(leaf_capacity), int(max_depth), ctypes.byref(h))
    try:
        nl, nlp, nn, nf, npairs = ctypes.c_int32(), ctypes.c_int64(), ctypes.c_int64(), ctypes.c_int64(), ctypes.c_int64()
        _ffi.call("gx_leaf_lists_info", h, ctypes.byref(nl), ctypes.byref(nlp), ctypes.byref(nn), ctypes.byref(nf),
                  ctypes.byref(npairs))
        lo = np.empty(nl.value + 1, np.int32)
        lp = np.empty(nlp.value, np.int32)
        no = np.empty(nl.value + 1, np.int32)
        nlv = np.empty(max(nn.value, 1), np.int32)
        _ffi.call("gx_leaf_lists_export", h, ptr(lo), ptr(lp), ptr(no), ptr(nlv))
    finally:
        _ffi.call("gx_leaf_lists_free", h)
    return LeafLists(lo, lp, no, nlv[: nn.value], nf.value, npairs.value, bool(where.value))


def p2p_leaves(x, y, z, m, lists: LeafLists, params: PhysicsParams, ax, ay, az, precision=PRECISION_F64,
               stream=None) -> None:
    """Adds the near field to (ax, ay, az) in place.  Host numpy or device torch arrays."""
    near = lists.near_leaves if len(lists.near_leaves) else np.zeros(1, np.int32)
    _ffi.call("gx_p2p_leaves", len(x), ptr(x), ptr(y), ptr(z), ptr(m), lists.n_leaves, ptr(lists.leaf_offsets),
              ptr(lists.leaf_particles), ptr(lists.near_offsets), ptr(near), params.ffi(),
              _ffi.precision_code(precision), ptr(ax), ptr(ay), ptr(az), _ffi.stream_ptr(stream))

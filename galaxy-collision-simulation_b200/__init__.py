"""B200 softened-gravity engine for ryan-charette/galaxy-collision-simulation.

Drops in behind the reference's ``solver = "cuda-direct"`` path and the P2P near-field leaves
of its FMM.  Compute runs in hand-written sm_100a CUDA kernels behind the C ABI of
``include/gx.h`` (``_lib/libgx.so``); this package is the Python host side:

* ``engine``   -- the reference solver interface (cuda_solver_available,
                  compute_cuda_direct_accelerations, cuda_direct_leapfrog_step, ...)
* ``session``  -- device-resident sessions and batched ensembles (CUDA graphs)
* ``fmm_p2p``  -- reference-octree leaf lists and the GPU near field
* ``fmm``      -- the reference FMM solver (moments, far field and near field on the GPU)
* ``adjoint``  -- autograd Function over the leapfrog with the adjoint kernel (needs torch)
* ``ics``      -- seeded two-disk initial conditions
* ``snapshots`` -- the reference's CSV snapshot / diagnostics output (+ a binary form), async
"""
from ._ffi import (GX_ERR_CUDA, GX_ERR_INVALID_ARGUMENT, GX_ERR_NO_DEVICE, GX_ERR_OUT_OF_MEMORY, GX_ERR_TIMEOUT,
                   GX_ERR_UNSUPPORTED, GX_OK, LIB_PATH, PRECISION_F64, PRECISION_F64_EXACT, PRECISION_MIXED, GxError,
                   device_available, load)
from .engine import (Diagnostics, ParticleSet, PhysicsParams, compute_cuda_direct_accelerations,
                     compute_diagnostics, compute_direct_accelerations_for_targets, cuda_direct_leapfrog_step,
                     cuda_solver_available, indexed_accelerations)
from .fmm import (FastMultipoleSolver, FmmOptions, FmmStats, compute_fmm_accelerations,
                  compute_fmm_accelerations_for_targets)
from .fmm_p2p import LeafLists, build_leaf_lists, p2p_leaves
from .session import Batch, Session, batch_accelerations, describe_variant
from .snapshots import SnapshotWriter, read_binary
from . import ics

__all__ = [
    "GxError", "PhysicsParams", "ParticleSet", "Diagnostics", "Session", "Batch", "LeafLists",
    "cuda_solver_available", "compute_cuda_direct_accelerations", "compute_direct_accelerations_for_targets",
    "cuda_direct_leapfrog_step", "compute_diagnostics", "indexed_accelerations", "build_leaf_lists", "p2p_leaves",
    "batch_accelerations", "describe_variant", "device_available", "load", "ics",
    "FastMultipoleSolver", "FmmOptions", "FmmStats", "compute_fmm_accelerations",
    "compute_fmm_accelerations_for_targets", "SnapshotWriter", "read_binary",
    "PRECISION_F64", "PRECISION_MIXED", "PRECISION_F64_EXACT",
]

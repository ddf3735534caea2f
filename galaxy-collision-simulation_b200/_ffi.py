"""ctypes binding of the engine's C ABI (include/gx.h).

The shared library ``_lib/libgx.so`` is built in-tree by ``__graft_entry__.build()`` (or
``make -C csrc``).  Loading fails loudly when it is missing: there is no Python or CPU
fallback for any compute call.
"""
from __future__ import annotations

import ctypes
from ctypes import POINTER, c_char_p, c_double, c_int, c_int32, c_int64, c_void_p
from pathlib import Path

PACKAGE_DIR = Path(__file__).resolve().parent
LIB_PATH = PACKAGE_DIR / "_lib" / "libgx.so"
HEADER_PATH = PACKAGE_DIR.parent / "include" / "gx.h"

GX_OK = 0
GX_ERR_INVALID_ARGUMENT = 1
GX_ERR_NO_DEVICE = 2
GX_ERR_CUDA = 3
GX_ERR_TIMEOUT = 4
GX_ERR_OUT_OF_MEMORY = 5
GX_ERR_UNSUPPORTED = 6

PRECISION_F64 = 0
PRECISION_MIXED = 1
PRECISION_F64_EXACT = 2
SNAPSHOT_CSV = 1
SNAPSHOT_BINARY = 2
PRECISIONS = {"f64": PRECISION_F64, "mixed": PRECISION_MIXED, "f64-exact": PRECISION_F64_EXACT}

_STATUS_NAMES = {
    GX_ERR_INVALID_ARGUMENT: "invalid argument",
    GX_ERR_NO_DEVICE: "no device",
    GX_ERR_CUDA: "CUDA error",
    GX_ERR_TIMEOUT: "timeout",
    GX_ERR_OUT_OF_MEMORY: "out of memory",
    GX_ERR_UNSUPPORTED: "unsupported",
}


class GxError(RuntimeError):
    """A non-zero gx_status; ``status`` is the code, the message is gx_last_error()."""

    def __init__(self, status: int, message: str):
        super().__init__(f"[{_STATUS_NAMES.get(status, status)}] {message}")
        self.status = status


class Physics(ctypes.Structure):
    """gx_physics: PhysicsParams of the reference (cpp/core/simulation_params.hpp:5-8)."""

    _fields_ = [("G", c_double), ("softening", c_double)]


class DiagnosticsStruct(ctypes.Structure):
    """gx_diagnostics, fields in the reference's diagnostics.csv column order."""

    _fields_ = [
        ("total_mass", c_double),
        ("kinetic_energy", c_double),
        ("potential_energy", c_double),
        ("total_energy", c_double),
        ("momentum", c_double * 3),
        ("center_of_mass", c_double * 3),
        ("angular_momentum", c_double * 3),
    ]


class FmmOptionsStruct(ctypes.Structure):
    """gx_fmm_options: FmmOptions of the reference (cpp/fmm/fmm_solver.hpp:15-20)."""

    _fields_ = [("theta", c_double), ("leaf_capacity", c_int64), ("max_depth", c_int32),
                ("expansion_order", c_int32)]


class FmmStatsStruct(ctypes.Structure):
    """gx_fmm_stats: FmmStats of the reference (cpp/fmm/fmm_solver.hpp:22-27)."""

    _fields_ = [("node_count", c_int64), ("leaf_count", c_int64), ("far_interactions", c_int64),
                ("near_interactions", c_int64), ("far_pairs", c_int64), ("near_pairs", c_int64),
                ("tree_levels", c_int64)]


class GalaxyStruct(ctypes.Structure):
    """gx_galaxy: GalaxyConfig of the reference (cpp/core/initial_conditions.hpp:14-24)."""

    _fields_ = [("n_particles", c_int64), ("mass", c_double), ("radius", c_double), ("position", c_double * 3),
                ("velocity", c_double * 3), ("orientation", c_double), ("group_id", ctypes.c_uint32),
                ("reserved", ctypes.c_uint32), ("thickness", c_double), ("inclination", c_double)]


class RunMetadataStruct(ctypes.Structure):
    """gx_run_metadata: the SimulationConfig fields SnapshotWriter::write_metadata prints."""

    _fields_ = [("name", c_char_p), ("solver", c_char_p), ("particle_count", c_int64), ("steps", c_int32),
                ("snapshot_every", c_int32), ("dim", c_int32), ("fmm_expansion_order", c_int32), ("dt", c_double),
                ("gravitational_constant", c_double), ("softening", c_double), ("tree_theta", c_double),
                ("tree_leaf_capacity", c_int64)]


P = c_void_p  # any array: numpy .ctypes.data, torch .data_ptr(), or None
PP = POINTER(c_void_p)
I64 = c_int64
D = c_double
S = c_void_p  # cudaStream_t

# name: argument types (all return int gx_status unless listed in _RESTYPES)
_SIGNATURES = {
    "gx_last_error": [],
    "gx_abi_version": [],
    "gx_device_available": [POINTER(c_int)],
    "gx_direct_accel": [I64, P, P, P, P, Physics, c_int, P, P, P, S],
    "gx_direct_accel_targets": [I64, P, P, P, P, I64, I64, P, I64, Physics, c_int, P, P, P, S],
    "gx_leapfrog_step": [I64, P, P, P, P, P, P, P, P, P, P, D, Physics, c_int, S],
    "gx_kick": [I64, P, P, P, P, P, P, D, S],
    "gx_drift": [I64, P, P, P, P, P, P, D, S],
    "gx_kick_drift": [I64, P, P, P, P, P, P, P, P, P, D, D, S],
    "gx_diagnostics_compute": [I64, P, P, P, P, P, P, P, Physics, POINTER(DiagnosticsStruct), S],
    "gx_session_create": [I64, Physics, c_int, PP],
    "gx_session_destroy": [P],
    "gx_session_set_stream": [P, S],
    "gx_session_get_stream": [P, PP],
    "gx_session_set_state": [P, P, P, P, P, P, P, P, P, P, P],
    "gx_session_get_state": [P, P, P, P, P, P, P, P, P, P],
    "gx_session_device_arrays": [P, PP],
    "gx_session_compute_accelerations": [P, c_int],
    "gx_session_step": [P, I64, D, c_int],
    "gx_session_diagnostics": [P, POINTER(DiagnosticsStruct)],
    "gx_session_synchronize": [P],
    "gx_session_set_persistent": [P, c_int],
    "gx_session_set_targets": [P, I64, I64],
    "gx_session_set_fmm": [P, P],
    "gx_session_kick_drift": [P, D, D],
    "gx_session_force_kick": [P, D, c_int],
    "gx_session_synchronize_timeout": [P, D],
    "gx_session_enable_timing": [P, c_int],
    "gx_session_force_timing": [P, POINTER(D), POINTER(I64)],
    "gx_session_get_config": [P, c_int, POINTER(c_int), POINTER(c_int)],
    "gx_session_set_config": [P, c_int, c_int, c_int],
    "gx_session_autotune": [P, c_int, POINTER(D)],
    "gx_p2p_leaves": [I64, P, P, P, P, c_int32, P, P, P, P, Physics, c_int, P, P, P, S],
    "gx_galaxies_body_count": [c_int32, P],
    "gx_generate_galaxies": [c_int32, P, Physics, ctypes.c_uint64, P, P, P, P, P, P, P, P, S],
    "gx_snapshot_writer_create": [c_char_p, I64, P, c_int, c_int, PP],
    "gx_snapshot_writer_flush": [P],
    "gx_snapshot_writer_destroy": [P],
    "gx_snapshot_write": [P, c_int, D, P, P, P, P, P, P, P, P, P, P, S],
    "gx_snapshot_write_diagnostics": [P, c_int, D, POINTER(DiagnosticsStruct)],
    "gx_snapshot_write_metadata": [P, POINTER(RunMetadataStruct)],
    "gx_session_snapshot": [P, P, c_int, D],
    "gx_fmm_accel": [I64, P, P, P, P, Physics, FmmOptionsStruct, c_int, I64, I64, P, P, P, POINTER(FmmStatsStruct),
                     S],
    "gx_fmm_accel_timed": [I64, P, P, P, P, Physics, FmmOptionsStruct, c_int, I64, I64, P, P, P,
                           POINTER(FmmStatsStruct), S, P],
    "gx_fmm_moments": [I64, P, P, P, P, Physics, FmmOptionsStruct, I64, P, POINTER(I64)],
    "gx_leaf_lists_build": [I64, P, P, P, P, D, D, I64, c_int, PP],
    "gx_leaf_lists_build_device": [I64, P, P, P, P, D, D, I64, c_int, S, PP, POINTER(c_int)],
    "gx_leaf_lists_info": [P, POINTER(c_int32), POINTER(I64), POINTER(I64), POINTER(I64), POINTER(I64)],
    "gx_leaf_lists_export": [P, P, P, P, P],
    "gx_leaf_lists_free": [P],
    "gx_batch_accel": [c_int32, P, P, P, P, P, Physics, c_int, P, P, P, S],
    "gx_batch_create": [c_int32, P, Physics, c_int, PP],
    "gx_batch_destroy": [P],
    "gx_batch_set_stream": [P, S],
    "gx_batch_set_state": [P, P, P, P, P, P, P, P],
    "gx_batch_get_state": [P, P, P, P, P, P, P, P, P, P],
    "gx_batch_device_arrays": [P, PP],
    "gx_batch_compute_accelerations": [P, c_int],
    "gx_batch_step": [P, I64, D, c_int],
    "gx_batch_diagnostics": [P, POINTER(DiagnosticsStruct)],
    "gx_batch_synchronize": [P],
    "gx_batch_get_config": [P, c_int, POINTER(c_int)],
    "gx_batch_set_config": [P, c_int, c_int],
    "gx_batch_autotune": [P, c_int, POINTER(D)],
    "gx_batch_enable_timing": [P, c_int],
    "gx_batch_force_timing": [P, POINTER(D), POINTER(I64)],
    "gx_direct_vjp": [I64, P, P, P, P, P, P, P, Physics, c_int, P, P, P, P, S],
    "gx_direct_accel_noalloc": [I64, P, P, P, P, Physics, c_int, P, P, P, S],
    "gx_variant_count": [c_int, POINTER(c_int)],
    "gx_variant_describe": [c_int, c_int, c_char_p, c_int],
    "gx_debug_fail_allocations": [c_int],
    "gx_debug_stall_barrier": [I64],
    "gx_debug_p2p_targets_per_thread": [c_int],
    "gx_debug_small_targets_per_warp": [c_int],
    "gx_debug_small_warps_per_target": [c_int],
    "gx_debug_fmm_tight_pools": [c_int],
}
_RESTYPES = {"gx_last_error": c_char_p, "gx_galaxies_body_count": c_int64}

_lib = None


def load() -> ctypes.CDLL:
    """Loads libgx.so once and declares every entry point's argument types."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise ImportError(
            f"engine library {LIB_PATH} is missing; build it with __graft_entry__.build() "
            "(nvcc for sm_100a) -- there is no CPU fallback"
        )
    lib = ctypes.CDLL(str(LIB_PATH))
    for name, args in _SIGNATURES.items():
        fn = getattr(lib, name)
        fn.argtypes = args
        fn.restype = _RESTYPES.get(name, c_int)
    _lib = lib
    return lib


def exported_names() -> list[str]:
    return list(_SIGNATURES)


def last_error() -> str:
    msg = load().gx_last_error()
    return msg.decode() if msg else ""


def check(status: int) -> None:
    """Raises GxError for a non-zero gx_status."""
    if status != GX_OK:
        raise GxError(status, last_error())


def call(name: str, *args) -> None:
    check(getattr(load(), name)(*args))


def physics(G: float, softening: float) -> Physics:
    return Physics(float(G), float(softening))


def precision_code(p) -> int:
    if isinstance(p, str):
        return PRECISIONS[p]
    return int(p)


def device_available() -> bool:
    flag = c_int(0)
    call("gx_device_available", ctypes.byref(flag))
    return bool(flag.value)


def ptr(a):
    """Raw address of a float64/int array (numpy or torch), or None."""
    if a is None:
        return None
    if hasattr(a, "data_ptr"):  # torch.Tensor
        if not a.is_contiguous():
            raise ValueError("tensor must be contiguous")
        return a.data_ptr()
    if not a.flags["C_CONTIGUOUS"]:
        raise ValueError("array must be C-contiguous")
    return a.ctypes.data


def stream_ptr(stream) -> int | None:
    """cudaStream_t of a torch.cuda.Stream (or an int handle); None = legacy default."""
    if stream is None:
        return None
    if isinstance(stream, int):
        return stream
    return stream.cuda_stream


def diagnostics_dict(d: DiagnosticsStruct) -> dict:
    return {
        "total_mass": d.total_mass,
        "kinetic_energy": d.kinetic_energy,
        "potential_energy": d.potential_energy,
        "total_energy": d.total_energy,
        "momentum": tuple(d.momentum),
        "center_of_mass": tuple(d.center_of_mass),
        "angular_momentum": tuple(d.angular_momentum),
    }

"""Resident device sessions: one system (``Session``) or an ensemble (``Batch``).

A session keeps the FP64 state on the device and runs kick-drift-kick steps as CUDA-graph
launches with no host synchronisation; host copies happen only in ``set_state`` /
``get_state`` (the reference copies the whole state in and out on every step,
cpp/cuda/cuda_solver.cu:224-245).  Arrays may be numpy (host) or torch CUDA tensors.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _ffi
from ._ffi import PRECISION_F64, ptr
from .engine import Diagnostics, PhysicsParams

_STATE = ("x", "y", "z", "vx", "vy", "vz", "ax", "ay", "az", "m")


class Session:
    """gx_session: n bodies resident on `device`."""

    def __init__(self, n: int, params: PhysicsParams | None = None, device: int = 0):
        self.params = params or PhysicsParams()
        self.n = int(n)
        h = ctypes.c_void_p()
        _ffi.call("gx_session_create", self.n, self.params.ffi(), int(device), ctypes.byref(h))
        self._h = h

    # -- lifetime ---------------------------------------------------------------------
    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            _ffi.call("gx_session_destroy", self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- state ------------------------------------------------------------------------
    def set_stream(self, stream):
        _ffi.call("gx_session_set_stream", self._h, _ffi.stream_ptr(stream))

    @property
    def stream(self) -> int:
        s = ctypes.c_void_p()
        _ffi.call("gx_session_get_stream", self._h, ctypes.byref(s))
        return s.value or 0

    def set_state(self, x, y, z, vx, vy, vz, m, ax=None, ay=None, az=None):
        _ffi.call("gx_session_set_state", self._h, ptr(x), ptr(y), ptr(z), ptr(vx), ptr(vy), ptr(vz), ptr(m),
                  ptr(ax), ptr(ay), ptr(az))

    def set_particles(self, p):
        """From an engine.ParticleSet (accelerations included)."""
        self.set_state(p.x, p.y, p.z, p.vx, p.vy, p.vz, p.m, p.ax, p.ay, p.az)

    def get_state(self) -> dict:
        out = {k: np.empty(self.n) for k in _STATE[:9]}
        _ffi.call("gx_session_get_state", self._h, *(ptr(out[k]) for k in _STATE[:9]))
        return out

    def device_arrays(self) -> dict:
        """Device addresses of the resident arrays (x, y, z, vx, vy, vz, ax, ay, az, m)."""
        arr = (ctypes.c_void_p * 10)()
        _ffi.call("gx_session_device_arrays", self._h, arr)
        return {k: arr[i] for i, k in enumerate(_STATE)}

    # -- compute ----------------------------------------------------------------------
    def compute_accelerations(self, precision=PRECISION_F64):
        _ffi.call("gx_session_compute_accelerations", self._h, _ffi.precision_code(precision))

    def step(self, n_steps: int, dt: float, precision=PRECISION_F64):
        _ffi.call("gx_session_step", self._h, int(n_steps), float(dt), _ffi.precision_code(precision))

    def set_persistent(self, enable: bool) -> None:
        """Small FP64 / exact-form systems step in one cooperative launch (default True)."""
        _ffi.call("gx_session_set_persistent", self._h, 1 if enable else 0)

    def set_fmm(self, options=None) -> None:
        """The force of later steps: the reference FMM with ``options`` (an FmmOptions), or the
        direct sum again with None.  FMM steps run in graph-replayed chunks of up to 32."""
        if options is None:
            _ffi.call("gx_session_set_fmm", self._h, None)
        else:
            self._fmm_opt = options.ffi()
            _ffi.call("gx_session_set_fmm", self._h, ctypes.addressof(self._fmm_opt))

    def set_targets(self, begin: int, count: int) -> None:
        """Owned bodies [begin, begin + count): the only ones kicked, drifted and given forces."""
        _ffi.call("gx_session_set_targets", self._h, int(begin), int(count))

    def kick_drift(self, kick_dt: float, drift_dt: float) -> None:
        """Opening half of a KDK step of the owned bodies (stream-ordered)."""
        _ffi.call("gx_session_kick_drift", self._h, float(kick_dt), float(drift_dt))

    def force_kick(self, kick_dt: float, precision=PRECISION_F64) -> None:
        """Closing half: forces on the owned bodies from all bodies, then the kick."""
        _ffi.call("gx_session_force_kick", self._h, float(kick_dt), _ffi.precision_code(precision))

    def diagnostics(self) -> Diagnostics:
        d = _ffi.DiagnosticsStruct()
        _ffi.call("gx_session_diagnostics", self._h, ctypes.byref(d))
        return Diagnostics.from_struct(d)

    def snapshot(self, writer, step: int, time: float) -> None:
        """Hands the current state to a SnapshotWriter without stalling the session's stream."""
        _ffi.call("gx_session_snapshot", self._h, writer.handle, int(step), float(time))

    def synchronize(self, timeout_ms: float | None = None):
        if timeout_ms is None:
            _ffi.call("gx_session_synchronize", self._h)
        else:
            _ffi.call("gx_session_synchronize_timeout", self._h, float(timeout_ms))

    # -- timing and tuning ----------------------------------------------------------------
    def enable_timing(self, enable: bool = True):
        _ffi.call("gx_session_enable_timing", self._h, 1 if enable else 0)

    def force_timing(self) -> tuple[float, int]:
        ms, n = ctypes.c_double(), ctypes.c_int64()
        _ffi.call("gx_session_force_timing", self._h, ctypes.byref(ms), ctypes.byref(n))
        return ms.value, n.value

    def get_config(self, precision) -> tuple[int, int]:
        v, s = ctypes.c_int(), ctypes.c_int()
        _ffi.call("gx_session_get_config", self._h, _ffi.precision_code(precision), ctypes.byref(v), ctypes.byref(s))
        return v.value, s.value

    def set_config(self, precision, variant: int, jsplit: int):
        _ffi.call("gx_session_set_config", self._h, _ffi.precision_code(precision), int(variant), int(jsplit))

    def autotune(self, precision) -> float:
        ms = ctypes.c_double()
        _ffi.call("gx_session_autotune", self._h, _ffi.precision_code(precision), ctypes.byref(ms))
        return ms.value


def describe_variant(precision, variant: int) -> str:
    buf = ctypes.create_string_buffer(128)
    _ffi.call("gx_variant_describe", _ffi.precision_code(precision), int(variant), buf, 128)
    return buf.value.decode()


class Batch:
    """gx_batch: independent systems concatenated; instance b owns offsets[b]:offsets[b+1]."""

    def __init__(self, offsets, params: PhysicsParams | None = None, device: int = 0):
        self.params = params or PhysicsParams(1.0, 0.05)
        self.offsets = np.ascontiguousarray(offsets, dtype=np.int64)
        self.n_instances = len(self.offsets) - 1
        self.n = int(self.offsets[-1])
        h = ctypes.c_void_p()
        _ffi.call("gx_batch_create", self.n_instances, ptr(self.offsets), self.params.ffi(), int(device),
                  ctypes.byref(h))
        self._h = h

    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            _ffi.call("gx_batch_destroy", self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_stream(self, stream):
        _ffi.call("gx_batch_set_stream", self._h, _ffi.stream_ptr(stream))

    def set_state(self, x, y, z, vx, vy, vz, m):
        _ffi.call("gx_batch_set_state", self._h, ptr(x), ptr(y), ptr(z), ptr(vx), ptr(vy), ptr(vz), ptr(m))

    def get_state(self) -> dict:
        out = {k: np.empty(self.n) for k in _STATE[:9]}
        _ffi.call("gx_batch_get_state", self._h, *(ptr(out[k]) for k in _STATE[:9]))
        return out

    def device_arrays(self) -> dict:
        arr = (ctypes.c_void_p * 10)()
        _ffi.call("gx_batch_device_arrays", self._h, arr)
        return {k: arr[i] for i, k in enumerate(_STATE)}

    def compute_accelerations(self, precision=PRECISION_F64):
        _ffi.call("gx_batch_compute_accelerations", self._h, _ffi.precision_code(precision))

    def step(self, n_steps: int, dt: float, precision=PRECISION_F64):
        _ffi.call("gx_batch_step", self._h, int(n_steps), float(dt), _ffi.precision_code(precision))

    def diagnostics(self) -> list[Diagnostics]:
        arr = (_ffi.DiagnosticsStruct * self.n_instances)()
        _ffi.call("gx_batch_diagnostics", self._h, arr)
        return [Diagnostics.from_struct(arr[i]) for i in range(self.n_instances)]

    def synchronize(self):
        _ffi.call("gx_batch_synchronize", self._h)

    def get_config(self, precision) -> int:
        v = ctypes.c_int()
        _ffi.call("gx_batch_get_config", self._h, _ffi.precision_code(precision), ctypes.byref(v))
        return v.value

    def set_config(self, precision, variant: int):
        _ffi.call("gx_batch_set_config", self._h, _ffi.precision_code(precision), int(variant))

    def autotune(self, precision) -> float:
        ms = ctypes.c_double()
        _ffi.call("gx_batch_autotune", self._h, _ffi.precision_code(precision), ctypes.byref(ms))
        return ms.value

    def enable_timing(self, enable: bool = True):
        _ffi.call("gx_batch_enable_timing", self._h, 1 if enable else 0)

    def force_timing(self) -> tuple[float, int]:
        ms, n = ctypes.c_double(), ctypes.c_int64()
        _ffi.call("gx_batch_force_timing", self._h, ctypes.byref(ms), ctypes.byref(n))
        return ms.value, n.value


def batch_accelerations(offsets, x, y, z, m, params: PhysicsParams, precision=PRECISION_F64):
    """Stateless batched direct sum: returns (ax, ay, az) for host inputs."""
    offsets = np.ascontiguousarray(offsets, dtype=np.int64)
    n = int(offsets[-1])
    out = [np.zeros(n) for _ in range(3)]
    xs = [np.ascontiguousarray(a, np.float64) for a in (x, y, z, m)]
    _ffi.call("gx_batch_accel", len(offsets) - 1, ptr(offsets), *(ptr(a) for a in xs), params.ffi(),
              _ffi.precision_code(precision), *(ptr(o) for o in out), None)
    return tuple(out)

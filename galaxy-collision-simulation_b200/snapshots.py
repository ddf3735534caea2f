"""Snapshot and diagnostics output of the reference's SnapshotWriter
(cpp/io/snapshot_writer.cpp:38-128), taken asynchronously from device-resident state.

``SnapshotWriter(directory, n, group_id)`` writes snapshot_%06d.csv files byte-identical to the
reference's, diagnostics.csv rows, metadata.json, and optionally the binary SoA form snapshot_%06d.bin
(``read_binary`` loads one).  ``write`` accepts host numpy arrays, CUDA tensors or a
``ParticleSet``; ``Session.snapshot`` snapshots a session without stalling its stream.
"""
from __future__ import annotations

import ctypes
from pathlib import Path

import numpy as np

from . import _ffi
from ._ffi import ptr
from .engine import Diagnostics

FIELDS = ("x", "y", "z", "vx", "vy", "vz", "ax", "ay", "az", "m")


class SnapshotWriter:
    def __init__(self, directory, n: int, group_id=None, csv: bool = True, binary: bool = False, slots: int = 2):
        formats = (_ffi.SNAPSHOT_CSV if csv else 0) | (_ffi.SNAPSHOT_BINARY if binary else 0)
        g = None if group_id is None else np.ascontiguousarray(group_id, np.uint32)
        self._group = g
        self.n = int(n)
        self._h = ctypes.c_void_p()
        _ffi.call("gx_snapshot_writer_create", str(directory).encode(), self.n, None if g is None else ptr(g), formats,
                  int(slots), ctypes.byref(self._h))

    @property
    def handle(self):
        return self._h

    def write(self, step: int, time: float, particles=None, stream=None, **arrays) -> None:
        """Snapshot of a ParticleSet or of arrays x..az, m (host numpy or CUDA tensors)."""
        src = [getattr(particles, f) for f in FIELDS] if particles is not None else [arrays[f] for f in FIELDS]
        src = [np.ascontiguousarray(a, np.float64) if isinstance(a, np.ndarray) else a for a in src]
        _ffi.call("gx_snapshot_write", self._h, int(step), float(time), *(ptr(a) for a in src),
                  _ffi.stream_ptr(stream))

    def write_diagnostics(self, step: int, time: float, d: Diagnostics) -> None:
        st = _ffi.DiagnosticsStruct(d.total_mass, d.kinetic_energy, d.potential_energy, d.total_energy,
                                    (ctypes.c_double * 3)(*d.momentum), (ctypes.c_double * 3)(*d.center_of_mass),
                                    (ctypes.c_double * 3)(*d.angular_momentum))
        _ffi.call("gx_snapshot_write_diagnostics", self._h, int(step), float(time), ctypes.byref(st))

    def write_metadata(self, name: str, solver: str, particle_count: int, steps: int, dt: float,
                       snapshot_every: int, dim: int = 3, gravitational_constant: float = 1.0,
                       softening: float = 0.02, tree_theta: float = 0.6, tree_leaf_capacity: int = 16,
                       fmm_expansion_order: int = 4) -> None:
        """metadata.json of the run (SnapshotWriter::write_metadata, snapshot_writer.cpp:49-69);
        the defaults are SimulationConfig's (cpp/core/config.hpp:20-35)."""
        md = _ffi.RunMetadataStruct(str(name).encode(), str(solver).encode(), int(particle_count), int(steps),
                                    int(snapshot_every), int(dim), int(fmm_expansion_order), float(dt),
                                    float(gravitational_constant), float(softening), float(tree_theta),
                                    int(tree_leaf_capacity))
        _ffi.call("gx_snapshot_write_metadata", self._h, ctypes.byref(md))

    def flush(self) -> None:
        _ffi.call("gx_snapshot_writer_flush", self._h)

    def close(self) -> None:
        if self._h:
            h, self._h = self._h, ctypes.c_void_p()
            _ffi.call("gx_snapshot_writer_destroy", h)

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def read_binary(path) -> dict:
    """Loads snapshot_%06d.bin: {'step', 'time', 'group_id', and the FIELDS arrays}."""
    raw = Path(path).read_bytes()
    if raw[:8] != b"GXSNAP01":
        raise ValueError(f"{path}: not a snapshot file")
    n, step, fields = np.frombuffer(raw, np.int64, 1, 8)[0], *np.frombuffer(raw, np.int32, 2, 16)
    time = float(np.frombuffer(raw, np.float64, 1, 24)[0])
    data = np.frombuffer(raw, np.float64, int(fields) * int(n), 32).reshape(int(fields), int(n))
    out = {f: data[k].copy() for k, f in enumerate(FIELDS)}
    out.update(step=int(step), time=time,
               group_id=np.frombuffer(raw, np.uint32, int(n), 32 + 8 * int(fields) * int(n)).copy())
    return out

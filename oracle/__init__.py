"""TEST INFRASTRUCTURE ONLY: ctypes access to the parity checker.

* ``port``  -- _build/liboracle.so, the plain-C restatement of the reference path
               (gx_oracle.c; every function cites the reference file:line it follows);
* ``ref``   -- _ref/libgxref.so, the reference's own C++ sources compiled unmodified
               with ref_wrap.cpp (only where the reference tree was present at build time).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline / reference legs may
import this package.  The engine never calls it; it is the checker, not the product.
"""
from __future__ import annotations

import ctypes
import os
from ctypes import POINTER, c_double, c_int, c_int32, c_int64, c_void_p
from pathlib import Path

import numpy as np

ORACLE_DIR = Path(__file__).resolve().parent
PORT_PATH = ORACLE_DIR / "_build" / "liboracle.so"
REF_PATH = ORACLE_DIR / "_ref" / "libgxref.so"
REF_SIM_CPU = ORACLE_DIR / "_ref" / "fmm_galaxy_sim_cpu"
REF_SIM_B200 = ORACLE_DIR / "_ref" / "fmm_galaxy_sim_b200"
REF_SMOKE_B200 = ORACLE_DIR / "_ref" / "ref_smoke_tests_b200"
REF_SIM_RESIDENT = ORACLE_DIR / "_ref" / "fmm_galaxy_sim_resident"

_port = None
_ref = None
P = c_void_p


def _p(a):
    return None if a is None else a.ctypes.data


def port():
    global _port
    if _port is None:
        if not PORT_PATH.exists():
            raise FileNotFoundError(f"{PORT_PATH} missing: run __graft_entry__.build() (make -C oracle)")
        lib = ctypes.CDLL(str(PORT_PATH))
        lib.oracle_direct_targets.argtypes = [c_int64, P, P, P, P, c_double, c_double, c_int64, c_int64, P, P, P]
        lib.oracle_direct_indexed.argtypes = [c_int64, P, P, P, P, c_double, c_double, c_int64, P, P, P, P]
        lib.oracle_direct_indexed_mt.argtypes = [c_int64, P, P, P, P, c_double, c_double, c_int64, P, P, P, P, c_int]
        lib.oracle_direct_symmetric.argtypes = [c_int64, P, P, P, P, c_double, c_double, P, P, P]
        lib.oracle_leapfrog.argtypes = [c_int64, P, P, P, P, P, P, P, P, P, P, c_double, c_double, c_double, c_int, c_int]
        lib.oracle_diagnostics.argtypes = [c_int64, P, P, P, P, P, P, P, c_double, c_double, P]
        lib.oracle_leaf_lists.argtypes = [c_int64, P, P, P, P, c_double, c_double, c_int64, c_int,
                                          POINTER(c_int32), POINTER(c_void_p), POINTER(c_void_p), POINTER(c_void_p),
                                          POINTER(c_void_p), POINTER(c_int64), POINTER(c_int64)]
        lib.oracle_free.argtypes = [c_void_p]
        lib.oracle_p2p_near.argtypes = [c_int64, P, P, P, P, c_double, c_double, c_int32, P, P, P, P, P, P, P]
        lib.oracle_direct_vjp.argtypes = [c_int64, P, P, P, P, P, P, P, c_double, c_double, P, P, P, P]
        lib.oracle_ownership.argtypes = [c_int64, c_int, c_int, POINTER(c_int64), POINTER(c_int64)]
        lib.oracle_generate_disk.argtypes = [c_int64, c_double, c_double, c_double, ctypes.c_double, c_double, P, P,
                                             ctypes.c_uint32, c_double, c_double, ctypes.c_uint64, P, P, P, P, P, P, P]
        _port = lib
    return _port


def ref_available() -> bool:
    return REF_PATH.exists()


def ref():
    global _ref
    if _ref is None:
        if not REF_PATH.exists():
            raise FileNotFoundError(f"{REF_PATH} missing: the reference tree was absent at build time")
        lib = ctypes.CDLL(str(REF_PATH))
        lib.ref_direct.argtypes = [c_int64, P, P, P, P, c_double, c_double, P, P, P]
        lib.ref_direct_targets_mt.argtypes = [c_int64, P, P, P, P, c_double, c_double, c_int64, c_int64, P, P, P, c_int]
        lib.ref_leapfrog_direct.argtypes = [c_int64, P, P, P, P, P, P, P, P, P, P, c_double, c_double, c_double, c_int]
        lib.ref_diagnostics.argtypes = [c_int64, P, P, P, P, P, P, P, c_double, c_double, P]
        lib.ref_fmm.argtypes = [c_int64, P, P, P, P, c_double, c_double, c_double, c_int64, c_int, P, P, P]
        lib.ref_fmm_split.argtypes = [c_int64, P, P, P, P, c_double, c_double, c_double, c_int64, c_int,
                                      POINTER(c_int32), POINTER(c_int64), P, P, P, P, P, P, P]
        lib.ref_smoke80_inputs.argtypes = [P, P, P, P]
        lib.ref_generate_galaxies.argtypes = [c_int, P, c_double, c_double, ctypes.c_uint64, P, P, P, P, P, P, P, P]
        lib.ref_generate_galaxies.restype = c_int64
        lib.ref_write_metadata.argtypes = [ctypes.c_char_p, ctypes.c_char_p, ctypes.c_char_p, c_int64, c_int, c_double,
                                           c_int, c_int, c_double, c_double, c_double, c_int64, c_int]
        lib.ref_write_outputs.argtypes = [ctypes.c_char_p, c_int64, P, P, P, P, P, P, P, P, P, P, P, c_int, c_double,
                                          P]
        lib.ref_fmm_moments.argtypes = [c_int64, P, P, P, P, c_double, c_double, c_double, c_int64, c_int, c_int64, P,
                                        POINTER(c_int64), P]
        lib.ref_fmm_timed.argtypes = [c_int64, P, P, P, P, c_double, c_double, c_double, c_int64, c_int, c_int64, c_int,
                                      P, P, P, POINTER(c_double), POINTER(c_double), POINTER(c_int64)]
        lib.ref_leapfrog_fmm.argtypes = [c_int64, P, P, P, P, P, P, P, P, P, P, c_double, c_double, c_double, c_int,
                                         c_double, c_int64, c_int]
        _ref = lib
    return _ref


def _f(a):
    return np.ascontiguousarray(a, dtype=np.float64)


# ---- restatement (port) ------------------------------------------------------------
def direct_targets(x, y, z, m, G, eps, begin=0, end=None):
    x, y, z, m = map(_f, (x, y, z, m))
    n = len(x)
    end = n if end is None else end
    out = [np.zeros(n) for _ in range(3)]
    port().oracle_direct_targets(n, _p(x), _p(y), _p(z), _p(m), G, eps, begin, end, *map(_p, out))
    return np.stack([o[begin:end] for o in out], 1)


def direct_indexed(x, y, z, m, G, eps, targets, threads=1):
    x, y, z, m = map(_f, (x, y, z, m))
    t = np.ascontiguousarray(targets, np.int64)
    out = [np.zeros(len(t)) for _ in range(3)]
    if threads > 1:
        port().oracle_direct_indexed_mt(len(x), _p(x), _p(y), _p(z), _p(m), G, eps, len(t), _p(t), *map(_p, out), threads)
    else:
        port().oracle_direct_indexed(len(x), _p(x), _p(y), _p(z), _p(m), G, eps, len(t), _p(t), *map(_p, out))
    return np.stack(out, 1)


def direct_symmetric(x, y, z, m, G, eps):
    x, y, z, m = map(_f, (x, y, z, m))
    out = [np.zeros(len(x)) for _ in range(3)]
    port().oracle_direct_symmetric(len(x), _p(x), _p(y), _p(z), _p(m), G, eps, *map(_p, out))
    return np.stack(out, 1)


def leapfrog(state: dict, m, G, eps, dt, steps, solver=0) -> dict:
    """state: x,y,z,vx,vy,vz,ax,ay,az arrays (copied); solver 0 = symmetric, 1 = per-target."""
    s = {k: _f(state[k]).copy() for k in ("x", "y", "z", "vx", "vy", "vz", "ax", "ay", "az")}
    m = _f(m)
    port().oracle_leapfrog(len(m), *(_p(s[k]) for k in ("x", "y", "z", "vx", "vy", "vz", "ax", "ay", "az")),
                           _p(m), G, eps, dt, steps, solver)
    return s


def diagnostics(x, y, z, vx, vy, vz, m, G, eps) -> np.ndarray:
    arrs = list(map(_f, (x, y, z, vx, vy, vz, m)))
    out = np.zeros(13)
    port().oracle_diagnostics(len(arrs[0]), *map(_p, arrs), G, eps, _p(out))
    return out


def leaf_lists(x, y, z, m, eps, theta, leaf_capacity, max_depth=32):
    x, y, z, m = map(_f, (x, y, z, m))
    nl = c_int32()
    ptrs = [c_void_p() for _ in range(4)]
    nn, nf = c_int64(), c_int64()
    rc = port().oracle_leaf_lists(len(x), _p(x), _p(y), _p(z), _p(m), eps, theta, leaf_capacity, max_depth,
                                  ctypes.byref(nl), *(ctypes.byref(p) for p in ptrs), ctypes.byref(nn), ctypes.byref(nf))
    if rc != 0:
        raise RuntimeError("oracle_leaf_lists failed")
    lo = np.ctypeslib.as_array(ctypes.cast(ptrs[0], POINTER(c_int32)), shape=(nl.value + 1,))
    sizes = [nl.value + 1, int(lo[-1]), nl.value + 1, nn.value]
    out = []
    for p, s in zip(ptrs, sizes):
        a = np.ctypeslib.as_array(ctypes.cast(p, POINTER(c_int32)), shape=(max(s, 1),))[:s].copy() if p.value else np.zeros(0, np.int32)
        port().oracle_free(p)
        out.append(a)
    return dict(leaf_offsets=out[0], leaf_particles=out[1], near_offsets=out[2], near_leaves=out[3], n_far=nf.value)


def p2p_near(x, y, z, m, G, eps, lists, acc=None):
    x, y, z, m = map(_f, (x, y, z, m))
    n = len(x)
    a = [np.zeros(n) for _ in range(3)] if acc is None else [_f(acc[:, c]).copy() for c in range(3)]
    L = {k: np.ascontiguousarray(lists[k], np.int32) for k in ("leaf_offsets", "leaf_particles", "near_offsets", "near_leaves")}
    port().oracle_p2p_near(n, _p(x), _p(y), _p(z), _p(m), G, eps, len(L["leaf_offsets"]) - 1, _p(L["leaf_offsets"]),
                           _p(L["leaf_particles"]), _p(L["near_offsets"]), _p(L["near_leaves"]), *map(_p, a))
    return np.stack(a, 1)


def direct_vjp(x, y, z, m, lx, ly, lz, G, eps):
    arrs = list(map(_f, (x, y, z, m, lx, ly, lz)))
    out = [np.zeros(len(x)) for _ in range(4)]
    port().oracle_direct_vjp(len(x), *map(_p, arrs), G, eps, *map(_p, out))
    return np.stack(out[:3], 1), out[3]


def ownership(count, rank, size):
    b, e = c_int64(), c_int64()
    port().oracle_ownership(count, rank, size, ctypes.byref(b), ctypes.byref(e))
    return b.value, e.value


# ---- the reference itself (ref) ----------------------------------------------------
def ref_direct(x, y, z, m, G, eps):
    x, y, z, m = map(_f, (x, y, z, m))
    out = [np.zeros(len(x)) for _ in range(3)]
    ref().ref_direct(len(x), _p(x), _p(y), _p(z), _p(m), G, eps, *map(_p, out))
    return np.stack(out, 1)


def ref_direct_targets(x, y, z, m, G, eps, begin, end, threads=1):
    x, y, z, m = map(_f, (x, y, z, m))
    out = [np.zeros(end - begin) for _ in range(3)]
    ref().ref_direct_targets_mt(len(x), _p(x), _p(y), _p(z), _p(m), G, eps, begin, end, *map(_p, out), threads)
    return np.stack(out, 1)


def ref_leapfrog(state: dict, m, G, eps, dt, steps) -> dict:
    s = {k: _f(state[k]).copy() for k in ("x", "y", "z", "vx", "vy", "vz", "ax", "ay", "az")}
    m = _f(m)
    ref().ref_leapfrog_direct(len(m), *(_p(s[k]) for k in ("x", "y", "z", "vx", "vy", "vz", "ax", "ay", "az")), _p(m),
                              G, eps, dt, steps)
    return s


def ref_leapfrog_fmm(state: dict, m, G, eps, dt, steps, theta, leaf_capacity, order=4) -> dict:
    s = {k: _f(state[k]).copy() for k in ("x", "y", "z", "vx", "vy", "vz", "ax", "ay", "az")}
    m = _f(m)
    ref().ref_leapfrog_fmm(len(m), *(_p(s[k]) for k in ("x", "y", "z", "vx", "vy", "vz", "ax", "ay", "az")), _p(m),
                           G, eps, dt, steps, theta, leaf_capacity, order)
    return s


def ref_diagnostics(x, y, z, vx, vy, vz, m, G, eps) -> np.ndarray:
    arrs = list(map(_f, (x, y, z, vx, vy, vz, m)))
    out = np.zeros(13)
    ref().ref_diagnostics(len(arrs[0]), *map(_p, arrs), G, eps, _p(out))
    return out


def ref_fmm(x, y, z, m, G, eps, theta, leaf_capacity, order=4):
    x, y, z, m = map(_f, (x, y, z, m))
    out = [np.zeros(len(x)) for _ in range(3)]
    ref().ref_fmm(len(x), _p(x), _p(y), _p(z), _p(m), G, eps, theta, leaf_capacity, order, *map(_p, out))
    return np.stack(out, 1)


def ref_fmm_split(x, y, z, m, G, eps, theta, leaf_capacity, order=4):
    x, y, z, m = map(_f, (x, y, z, m))
    n = len(x)
    nl, nn = c_int32(), c_int64()
    ref().ref_fmm_split(n, _p(x), _p(y), _p(z), _p(m), G, eps, theta, leaf_capacity, order, ctypes.byref(nl),
                        ctypes.byref(nn), None, None, None, None, None, None, None)
    lo = np.zeros(nl.value + 1, np.int32)
    lp = np.zeros(n, np.int32)
    no = np.zeros(nl.value + 1, np.int32)
    nlv = np.zeros(max(nn.value, 1), np.int32)
    far = [np.zeros(n) for _ in range(3)]
    ref().ref_fmm_split(n, _p(x), _p(y), _p(z), _p(m), G, eps, theta, leaf_capacity, order, ctypes.byref(nl),
                        ctypes.byref(nn), _p(lo), _p(lp), _p(no), _p(nlv), *map(_p, far))
    return dict(leaf_offsets=lo, leaf_particles=lp, near_offsets=no, near_leaves=nlv[: nn.value]), np.stack(far, 1)


def ref_fmm_moments(x, y, z, m, G, eps, theta, leaf_capacity, order=4):
    """(records (n_nodes, 35), stats (4,)) of the reference tree's massive nodes, breadth-first."""
    x, y, z, m = map(_f, (x, y, z, m))
    nn = c_int64()
    stats = np.zeros(4, np.int64)
    ref().ref_fmm_moments(len(x), _p(x), _p(y), _p(z), _p(m), G, eps, theta, leaf_capacity, order, 0, None,
                          ctypes.byref(nn), _p(stats))
    rec = np.zeros((max(nn.value, 1), 35))
    ref().ref_fmm_moments(len(x), _p(x), _p(y), _p(z), _p(m), G, eps, theta, leaf_capacity, order, nn.value, _p(rec),
                          ctypes.byref(nn), _p(stats))
    return rec[: nn.value], stats


def ref_fmm_timed(x, y, z, m, G, eps, theta, leaf_capacity, order, stride, threads):
    """Reference build + evaluate_particle on every stride-th body (leaf order) over threads.
    Returns (accelerations (n, 3) with NaN where not evaluated, build_s, eval_s, n_evaluated)."""
    x, y, z, m = map(_f, (x, y, z, m))
    n = len(x)
    out = [np.full(n, np.nan) for _ in range(3)]
    b, e, k = c_double(), c_double(), c_int64()
    ref().ref_fmm_timed(n, _p(x), _p(y), _p(z), _p(m), G, eps, theta, leaf_capacity, order, stride, threads,
                        *map(_p, out), ctypes.byref(b), ctypes.byref(e), ctypes.byref(k))
    return np.stack(out, 1), b.value, e.value, k.value


def ref_write_outputs(directory, state: dict, m, group, step, time, diag13):
    """The reference SnapshotWriter writes diagnostics.csv (header + one row) and one snapshot."""
    arrs = [_f(state[k]) for k in ("x", "y", "z", "vx", "vy", "vz", "ax", "ay", "az")] + [_f(m)]
    g = None if group is None else np.ascontiguousarray(group, np.uint32)
    d = _f(diag13)
    ref().ref_write_outputs(str(directory).encode(), len(arrs[0]), *map(_p, arrs), None if g is None else _p(g),
                            int(step), float(time), _p(d))


def ref_write_metadata(directory, name, solver, particle_count, steps, dt, snapshot_every, dim, G, eps, theta,
                       leaf_capacity, order):
    """The reference SnapshotWriter writes metadata.json (and an empty diagnostics.csv)."""
    ref().ref_write_metadata(str(directory).encode(), str(name).encode(), str(solver).encode(), int(particle_count),
                             int(steps), float(dt), int(snapshot_every), int(dim), float(G), float(eps), float(theta),
                             int(leaf_capacity), int(order))


GALAXY_FIELDS = ("n_particles", "mass", "radius", "position", "velocity", "orientation", "group_id", "thickness",
                 "inclination")


def _galaxy_row(g: dict):
    return [g["n_particles"], g["mass"], g["radius"], *g.get("position", (0, 0, 0)), *g.get("velocity", (0, 0, 0)),
            g.get("orientation", 0.0), g.get("group_id", 0), g.get("thickness", 0.0), g.get("inclination", 0.0)]


def ref_generate_galaxies(galaxies, G, eps, seed):
    """The reference's generate_galaxies (mt19937_64): dict of x..vz, m, group_id."""
    cfg = np.array([_galaxy_row(g) for g in galaxies], dtype=np.float64).ravel()
    n = ref().ref_generate_galaxies(len(galaxies), _p(cfg), G, eps, seed, *([None] * 8))
    out = {k: np.zeros(n) for k in ("x", "y", "z", "vx", "vy", "vz", "m")}
    grp = np.zeros(n, np.uint32)
    ref().ref_generate_galaxies(len(galaxies), _p(cfg), G, eps, seed, *(_p(out[k]) for k in ("x", "y", "z", "vx", "vy",
                                                                                              "vz", "m")), _p(grp))
    out["group_id"] = grp
    return out


def generate_galaxies(galaxies, G, eps, seed):
    """The oracle's restatement with the engine's counter-based draws (oracle_generate_disk)."""
    lib = port()
    parts = []
    for k, g in enumerate(galaxies):
        n = int(g["n_particles"])
        if n <= 0 or not g["mass"] > 0 or not g["radius"] > 0:
            continue
        arr = {f: np.zeros(n) for f in ("x", "y", "z", "vx", "vy", "vz", "m")}
        pos = _f(np.array(g.get("position", (0, 0, 0)), np.float64))
        vel = _f(np.array(g.get("velocity", (0, 0, 0)), np.float64))
        lib.oracle_generate_disk(n, float(g["mass"]), float(g["radius"]), float(g.get("thickness", 0.0)),
                                 float(g.get("orientation", 0.0)), float(g.get("inclination", 0.0)), _p(pos), _p(vel),
                                 k, G, eps, seed, *(_p(arr[f]) for f in ("x", "y", "z", "vx", "vy", "vz", "m")))
        arr["group_id"] = np.full(n, int(g.get("group_id", 0)), np.uint32)
        parts.append(arr)
    if not parts:
        return {f: np.zeros(0) for f in ("x", "y", "z", "vx", "vy", "vz", "m", "group_id")}
    return {f: np.concatenate([q[f] for q in parts]) for f in parts[0]}


def ref_smoke80_inputs():
    a = [np.zeros(80) for _ in range(4)]
    ref().ref_smoke80_inputs(*map(_p, a))
    return a


def default_threads() -> int:
    return len(os.sched_getaffinity(0))

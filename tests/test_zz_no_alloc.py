"""The allocation-free direct-sum entry point (gx_direct_accel_noalloc) on B200.

Who needs it: callers that cannot allocate device memory when they call in -- a process
whose GPU memory is reserved up front by another allocator, a real-time step loop that must
stay out of the allocator, code running under a stream capture that forbids allocation.
The entry point keeps its scratch in a fixed device array inside the library instead.

Checked here through the C ABI: two calls in a row (different systems, so the second call
finds the first call's leftovers in the shared array) give the same accelerations as the
allocating entry point gx_direct_accel within the engine's tolerances, and the same as the
oracle's per-target direct sum (the reference's compute_direct_accelerations_for_targets
restated in C): bit for bit in the exact form, within 1e-12 relative in FP64, at a size that
needs no source split and at the limit, where the partial sums of a split fill the array;
sizes above the fixed limit and host arrays are refused with a clear error.  This file is
collected last and depends on no other test, so it also passes alone in a fresh process.
"""
import numpy as np
import pytest
import torch

import gx
import oracle
from gx import _ffi

pytestmark = pytest.mark.gpu

LIMIT = 65536


def _device_system(n, seed, eps):
    p = gx.ics.two_disk_encounter(n // 2, n - n // 2, seed, eps)
    return {k: torch.from_numpy(getattr(p, k)).cuda() for k in ("x", "y", "z", "m")}


def _accel(entry, d, eps, precision):
    lib = _ffi.load()
    n = d["x"].numel()
    out = [torch.full_like(d["x"], float("nan")) for _ in range(3)]
    stream = torch.cuda.current_stream().cuda_stream
    status = getattr(lib, entry)(n, *(d[k].data_ptr() for k in ("x", "y", "z", "m")), _ffi.physics(1.0, eps),
                                 precision, *(o.data_ptr() for o in out), stream)
    assert status == gx.GX_OK, _ffi.last_error()
    torch.cuda.synchronize()
    return torch.stack(out, 1).cpu().numpy()


def _rel(a, b):
    return np.linalg.norm(a - b, axis=1) / np.maximum(np.linalg.norm(b, axis=1), 1e-300)


@pytest.mark.parametrize("precision,median_tol,max_tol", [(gx.PRECISION_F64, 1e-14, 1e-12),
                                                          (gx.PRECISION_MIXED, 1e-7, 1e-6)])
def test_two_calls_in_a_row_match_the_allocating_entry_point(precision, median_tol, max_tol):
    systems = [(_device_system(LIMIT, 101, 0.02), 0.02), (_device_system(3001, 202, 0.05), 0.05)]
    for d, eps in systems:  # the second call reuses the array the first call filled
        got = _accel("gx_direct_accel_noalloc", d, eps, precision)
        want = _accel("gx_direct_accel", d, eps, precision)
        assert np.all(np.isfinite(got))
        e = _rel(got, want)
        assert np.median(e) <= median_tol and e.max() <= max_tol, (np.median(e), e.max())


@pytest.mark.parametrize("n,seed,eps", [(3001, 303, 0.05), (LIMIT, 404, 0.02)])
def test_two_calls_in_a_row_match_the_oracle(n, seed, eps):
    d = _device_system(n, seed, eps)
    h = {k: d[k].cpu().numpy() for k in ("x", "y", "z", "m")}
    rng = np.random.default_rng(seed)
    idx = np.arange(n) if n <= 4096 else np.sort(rng.choice(n, 2048, replace=False))
    want = oracle.direct_indexed(h["x"], h["y"], h["z"], h["m"], 1.0, eps, idx, threads=oracle.default_threads())
    for _ in range(2):  # the second call finds the first call's contents in the array
        exact = _accel("gx_direct_accel_noalloc", d, eps, gx.PRECISION_F64_EXACT)[idx]
        assert np.array_equal(exact, want)
        f64 = _accel("gx_direct_accel_noalloc", d, eps, gx.PRECISION_F64)[idx]
        assert _rel(f64, want).max() <= 1e-12


def test_limits_are_refused_clearly():
    lib = _ffi.load()
    big = torch.zeros(LIMIT + 1, dtype=torch.float64, device="cuda")
    status = lib.gx_direct_accel_noalloc(LIMIT + 1, *(big.data_ptr() for _ in range(4)), _ffi.physics(1.0, 0.1),
                                         gx.PRECISION_F64, *(big.data_ptr() for _ in range(3)), None)
    assert status == gx.GX_ERR_INVALID_ARGUMENT
    assert "65536" in _ffi.last_error()
    host = np.zeros(8)
    status = lib.gx_direct_accel_noalloc(8, *(host.ctypes.data for _ in range(4)), _ffi.physics(1.0, 0.1),
                                         gx.PRECISION_F64, *(host.ctypes.data for _ in range(3)), None)
    assert status == gx.GX_ERR_INVALID_ARGUMENT
    assert "device arrays only" in _ffi.last_error()

"""Benchmark: direct softened gravity at N = 2^20 on B200 (mixed precision vs FP64).

A "step" is one kick-drift-kick step of the whole system (one force evaluation of
N(N-1) ordered interactions).  Default workload: two exponential disks of 524,288 bodies
(mass ratio 3:1), softening 0.01, dt 0.001; one initial force evaluation, W untimed warm-up
steps and K timed steps (K = 10: "1 eval + 10 KDK steps").  The 80 MiB FP64 state fits in
L2, so L2 is flushed (a 256 MiB device write) before every timed step, outside the timed
interval.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

One JSON line from rank 0.  `value` is device-resident throughput (CUDA events on the
stream the session launches on, max over ranks); `e2e` is the same metric through the C ABI
with host buffers (gx_leapfrog_step: H2D of the state, the step, D2H of the result, every
step).  Multi-GPU (torchrun): target ranges per rank, one NCCL all-gather of positions per
step, strong scaling at fixed N.
"""
from __future__ import annotations

import argparse
import importlib.util
import json
import math
import os
import re
import subprocess
import sys
import tempfile
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
PKG_DIR = ROOT / "galaxy-collision-simulation_b200"
METRIC = "Ginteractions/s at N=1M: mixed-prec vs FP64 GPU @ rel-err≤1e-6; adjoint/fwd"
UNIT = "Ginteractions/s"
FMA_PIPE_OPS_PER_INTERACTION = 12  # 3 FADD, 3 FFMA (r^2), 2 FMUL (inv^3), 1 FMUL (m), 3 FFMA (acc)
FP32_LANES_PER_SM = 128


def load_gx():
    if "gx" in sys.modules:
        return sys.modules["gx"]
    spec = importlib.util.spec_from_file_location("gx", PKG_DIR / "__init__.py",
                                                  submodule_search_locations=[str(PKG_DIR)])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["gx"] = mod
    spec.loader.exec_module(mod)
    return mod


def measured_peaks() -> dict:
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        try:
            return json.loads(p.read_text())
        except Exception:
            return {}
    return {}


# ---------------------------------------------------------------------------------------
# clocks during the timed region
# ---------------------------------------------------------------------------------------
class ClockSampler:
    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(prefix="gx_clocks_", suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.QUERY}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except FileNotFoundError:
            self.proc = None

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"], "samples": 0}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        rows = []
        for line in Path(self.path).read_text().splitlines():
            f = [c.strip() for c in line.split(",")]
            if len(f) < 9:
                continue
            try:
                rows.append(dict(sm=float(f[1]), max=float(f[2]), power=float(f[3]) if f[3] not in ("[N/A]", "") else 0.0,
                                 hw=f[5], hwt=f[6], swt=f[7], swp=f[8]))
            except ValueError:
                continue
        os.unlink(self.path)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        loaded = [r for r in rows if r["power"] > 300.0] or rows
        reasons = set()
        for r in loaded:
            for key, name in (("hw", "hw_slowdown"), ("hwt", "hw_thermal_slowdown"), ("swt", "sw_thermal_slowdown"),
                              ("swp", "sw_power_cap")):
                if r[key].lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": float(np.median([r["sm"] for r in loaded])), "sm_max_mhz": max(r["max"] for r in rows),
                "reasons": sorted(reasons), "samples": len(rows), "samples_under_load": len(loaded),
                "power_w_max": max(r["power"] for r in rows)}


def other_gpu_processes():
    """Compute processes on the visible GPUs other than this one (another tenant would skew timing)."""
    try:
        out = subprocess.run(["nvidia-smi", "--query-compute-apps=pid", "--format=csv,noheader"],
                             capture_output=True, text=True, timeout=10).stdout
    except Exception:
        return None
    pids = [int(x) for x in out.split() if x.strip().isdigit()]
    return len([p for p in pids if p != os.getpid()])


# ---------------------------------------------------------------------------------------
# CPU baseline: the reference's own per-target direct sum on the host cores
# ---------------------------------------------------------------------------------------
def cpu_threads() -> int:
    return len(os.sched_getaffinity(0))


def cpu_reference_rate(p, eps, seconds: float = 10.0, threads: int | None = None) -> dict:
    """G interactions/s of compute_direct_accelerations_for_targets split over all host
    threads by ownership ranges (oracle/_ref), or of the C restatement when the reference
    library is absent, on a contiguous target sample sized to about `seconds` of wall time."""
    sys.path.insert(0, str(ROOT))
    import oracle

    threads = threads or cpu_threads()
    n = len(p)
    kind = "reference" if oracle.ref_available() else "port"

    def run(count):
        t0 = time.perf_counter()
        if kind == "reference":
            oracle.ref_direct_targets(p.x, p.y, p.z, p.m, 1.0, eps, 0, count, threads=threads)
        else:
            oracle.direct_indexed(p.x, p.y, p.z, p.m, 1.0, eps, np.arange(count), threads=threads)
        return time.perf_counter() - t0

    cal = min(n, threads * 2)
    t = run(cal)
    count = int(min(n, max(threads, cal * seconds / max(t, 1e-3))))
    t = run(count)
    rate = count * (n - 1) / t / 1e9
    return {"value": rate, "unit": UNIT, "cores": threads, "kind": kind,
            "sample": f"targets 0..{count} of N={n} against all N sources "
                      f"({'compute_direct_accelerations_for_targets' if kind == 'reference' else 'oracle restatement'}"
                      f", {threads} threads by ownership ranges), {t:.1f} s wall",
            "seconds": t, "targets": count}


# ---------------------------------------------------------------------------------------
# DRAM traffic of the timed force launch (ncu dram__bytes_read.sum + dram__bytes_write.sum)
# ---------------------------------------------------------------------------------------
# Measured per body on two launches of each candidate headline variant at source split 8 with
# the closing kick fused (ncu flushes L2 before each launch), captured at N = 262,144:
#   ncu --metrics dram__bytes_read.sum,dram__bytes_write.sum,gpu__time_duration.sum
#       --clock-control none -k regex:force_mixed_tp -s 1 -c 2
#       python bench.py --quick --n 262144 --variant V --jsplit 8 --steps 2 --warmup 2 --no-configs
#   V = 0, force_mixed_tp_kernel<256,6,512>: read 15.22 / 15.46 MB, written 9.97 / 7.94 MB
#   V = 2, force_mixed_tp_kernel<128,6,512>: read 15.27 / 15.46 MB, written 9.76 / 7.06 MB
# per launch: 92.7 and 90.7 B/body on average, scaled to N by the bodies per launch (the
# launch's traffic is per-body work: positions and masses read once, accelerations written,
# velocities read and written).  The split's partial sums (8 x 24 B/body) do not reach DRAM:
# the tile's last CTA consumes them from L2.  Keyed by the kernel the bench ran (the autotuner
# picks either; they are within 0.1% of each other at N = 2^20).
TRAFFIC_BYTES_PER_BODY = {"mixed block=256 ipt=6 jt=512 f32x2-targets": 92.7,
                          "mixed block=128 ipt=6 jt=512 f32x2-targets": 90.7}


def traffic_capture(kernel: str):
    return None if kernel not in TRAFFIC_BYTES_PER_BODY else (
        f"ncu dram__bytes_read.sum + dram__bytes_write.sum of {kernel} at split 8 with the closing kick, "
        f"2 launches at N=262144: {TRAFFIC_BYTES_PER_BODY[kernel]} B/body, scaled to N")


# Algorithmic bytes per body of one force launch with the closing kick: x, y, z, m read
# (32 B), a written (24 B), v read and written (48 B).
ALGORITHMIC_BYTES_PER_BODY = 104


def ncu_traffic(n: int, kernel: str, jsplit: int):
    if kernel not in TRAFFIC_BYTES_PER_BODY or jsplit != 8:
        return None
    return TRAFFIC_BYTES_PER_BODY[kernel] * n


# ---------------------------------------------------------------------------------------
def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--n", type=int, default=1 << 20, help="bodies (default 2^20; two disks, mass ratio 3:1)")
    ap.add_argument("--precision", choices=["mixed", "f64"], default="mixed")
    ap.add_argument("--quick", action="store_true", help="kernel timing only (profiling runs)")
    ap.add_argument("--no-autotune", action="store_true")
    ap.add_argument("--variant", type=int, default=None, help="force a kernel variant id (skips autotuning)")
    ap.add_argument("--jsplit", type=int, default=None, help="source split used with --variant")
    ap.add_argument("--cpu-seconds", type=float, default=10.0)
    ap.add_argument("--fit-iters", type=int, default=30, help="Adam iterations of the fit workload")
    ap.add_argument("--sharded", action="store_true",
                    help="use the multi-GPU (target-range + NCCL all-gather) step even on one rank")
    ap.add_argument("--leaf-capacity", type=int, default=64, help="leaf capacity of the fmm-evals workload")
    ap.add_argument("--p2p-n", type=int, default=65536, help="bodies of the p2p and fmm-evals workloads")
    ap.add_argument("--p2p-tpt", type=int, default=0, choices=[0, 2, 4],
                    help="targets per thread of the P2P kernel (0: chosen by mean leaf size)")
    ap.add_argument("--no-configs", action="store_true",
                    help="skip the N=1000, N=65536 and ensemble configurations of the default line")
    ap.add_argument("--workload", default="mixed-n1048576",
                    choices=["mixed-n1048576", "ensemble", "fmm-n65536", "fmm-session-n65536", "fmm-evals",
                             "snapshots-n1048576",
                             "ics-ensemble512", "p2p", "p2p-n65536", "direct-n65536", "direct-n1000", "fit-n16384"],
                    help="headline (default) or one of the other configurations")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 1)

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    eps, dt = 0.01, 0.001
    n = args.n

    if args.impl == "reference":
        return reference_arm(args, rank, n, eps, dt)
    if args.workload != "mixed-n1048576":
        import torch
        torch.cuda.set_device(local)
        if world > 1 and args.workload != "ensemble":
            # the other workloads run on one GPU: rank 0 alone
            if rank != 0:
                return
        elif world > 1:
            import datetime
            import torch.distributed as dist
            dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                    device_id=torch.device("cuda", local))
        res = OTHER_WORKLOADS[args.workload](load_gx(), torch, args)
        if rank == 0:
            print(json.dumps(res), flush=True)
        if world > 1 and args.workload == "ensemble":
            import torch.distributed as dist
            dist.barrier()
            dist.destroy_process_group()
        return

    import torch
    import torch.distributed as dist

    gx = load_gx()
    torch.cuda.set_device(local)
    sharded = world > 1 or args.sharded
    if sharded:
        import datetime
        os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
        os.environ.setdefault("MASTER_PORT", "29533")
        os.environ.setdefault("RANK", "0")
        os.environ.setdefault("WORLD_SIZE", "1")
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=torch.device("cuda", local))
    p = gx.ics.two_disk_encounter(n // 2, n - n // 2, 20260502, eps, mass1=1.0, mass2=1.0 / 3.0)
    prec = gx.PRECISION_MIXED if args.precision == "mixed" else gx.PRECISION_F64
    if sharded:
        res = run_sharded(gx, torch, dist, p, args, rank, world, eps, dt, prec)
    else:
        res = run_single(gx, torch, p, args, eps, dt, prec)
    if rank == 0:
        print(json.dumps(res), flush=True)
    if sharded:
        dist.barrier()
        dist.destroy_process_group()


def l2_flusher(torch):
    buf = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    return lambda: buf.fill_(1)


def run_single(gx, torch, p, args, eps, dt, prec) -> dict:
    n = len(p)
    params = gx.PhysicsParams(1.0, eps)
    pairs = n * (n - 1)
    stream = torch.cuda.current_stream()
    flush = l2_flusher(torch)
    peaks = measured_peaks()
    sms = torch.cuda.get_device_properties(0).multi_processor_count
    sm_max_mhz = float(peaks.get("sm_max_mhz", 1965.0))
    out = {"metric": METRIC, "unit": UNIT, "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
           "higher_is_better": True, "scaling": "strong", "vs_baseline": None, "data": "synthetic",
           "dtype": "f32" if prec == gx.PRECISION_MIXED else "f64",
           "precision_note": ("FP32 pair arithmetic on offsets from per-tile FP64 origins; FP64 state, "
                              "per-tile compensated accumulation, FP64 diagnostics")
           if prec == gx.PRECISION_MIXED else "FP64 throughout"}

    sess = gx.Session(n, params)
    sess.set_stream(stream)
    sess.set_particles(p)
    tune_ms = None
    if args.variant is not None:
        sess.set_config(prec, args.variant, args.jsplit or 1)
    elif not args.no_autotune and not args.quick:
        tune_ms = sess.autotune(prec)
    variant, jsplit = sess.get_config(prec)
    sess.compute_accelerations(prec)  # the initial force evaluation
    torch.cuda.synchronize()
    e0 = None if args.quick else sess.diagnostics().total_energy
    for _ in range(args.warmup):
        sess.step(1, dt, prec)
    torch.cuda.synchronize()

    clocks = ClockSampler(torch.cuda.current_device())
    clocks.start()
    time.sleep(0.3)
    sess.enable_timing(True)
    evs = []
    for _ in range(args.steps):
        flush()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        sess.step(1, dt, prec)
        b.record(stream)
        evs.append((a, b))
    torch.cuda.synchronize()
    step_ms = [a.elapsed_time(b) for a, b in evs]
    force_ms, force_launches = sess.force_timing()
    sess.enable_timing(False)
    clk = clocks.stop()
    total_s = sum(step_ms) / 1e3
    value = args.steps * pairs / total_s / 1e9
    force_avg_s = force_ms / 1e3 / max(force_launches, 1)
    launches_per_step = 2  # kick-drift, force (the split's reduction runs inside the force kernel)
    out.update({"value": value, "ms_per_step": sum(step_ms) / args.steps, "steps_per_s": args.steps / total_s,
                "gpu_launches": args.steps * launches_per_step, "step_ms": [round(t, 3) for t in step_ms],
                "other_gpu_processes": other_gpu_processes()})
    fp32_peak = sms * FP32_LANES_PER_SM * sm_max_mhz * 1e6 / 1e12
    achieved = pairs * FMA_PIPE_OPS_PER_INTERACTION / force_avg_s / 1e12
    roof = {"bound": "fp32_fma_pipe", "achieved": achieved,
            "peak": fp32_peak, "unit": "T FP32-pipe lane-ops/s",
            "frac": achieved / fp32_peak,
            "peak_basis": f"{sms} SMs x {FP32_LANES_PER_SM} FP32 lanes x {sm_max_mhz:.0f} MHz (sm_max_mhz of "
                          "MEASURED_PEAKS.json); the FP32 FMA pipe bounds this kernel, not HBM or tensor cores",
            "ops_per_interaction": FMA_PIPE_OPS_PER_INTERACTION,
            "kernel_ms_per_launch": force_avg_s * 1e3,
            "traffic": ncu_traffic(n, gx.describe_variant(prec, variant), jsplit),
            "algorithmic_bytes": ALGORITHMIC_BYTES_PER_BODY * n,
            "traffic_capture": traffic_capture(gx.describe_variant(prec, variant)) if jsplit == 8 else None}
    if clk.get("sm_mhz"):
        roof["frac_at_observed_clock"] = achieved / (sms * FP32_LANES_PER_SM * clk["sm_mhz"] * 1e6 / 1e12)
    if prec == gx.PRECISION_F64:
        roof["note"] = "FP64 form: 17 FP64 pipe ops per interaction; frac is against the FP32 pipe"
    out["roofline"] = roof
    out["clocks"] = clk
    out["config"] = {"workload": f"direct-mixed-n{n}" if prec == gx.PRECISION_MIXED else f"direct-f64-n{n}",
                     "n": n, "disks": "2 exponential disks, mass ratio 3:1", "softening": eps, "dt": dt,
                     "initial_eval": 1, "kernel": gx.describe_variant(prec, variant), "jsplit": jsplit,
                     "autotune_ms_per_eval": tune_ms,
                     "l2": "flushed (256 MiB device write) before every timed step, outside the timed interval"}
    if args.quick:
        sess.close()
        return out

    state = sess.get_state()
    e1 = sess.diagnostics().total_energy
    out["energy_drift"] = {"relative": abs(e1 - e0) / abs(e0), "steps": args.warmup + args.steps,
                           "precision": "fp64 diagnostics"}

    # -- accuracy of the production accelerations on 4096 sampled targets (FP64 exact form
    #    = compute_direct_accelerations_for_targets bit for bit) --------------------------
    rng = np.random.default_rng(4096)
    idx = np.sort(rng.choice(n, 4096, replace=False))
    q = gx.ParticleSet(state["x"], state["y"], state["z"], state["vx"], state["vy"], state["vz"], p.m)
    a_prod = np.stack([state["ax"], state["ay"], state["az"]], 1)[idx]
    a_ref = gx.indexed_accelerations(q, params, idx, gx.PRECISION_F64_EXACT)
    err = np.linalg.norm(a_prod - a_ref, axis=1) / np.maximum(np.linalg.norm(a_ref, axis=1), 1e-300)
    out["rel_err"] = {"median": float(np.median(err)), "max": float(err.max()), "targets": 4096,
                      "vs": "FP64 (exact per-target form) at the final positions"}

    # -- FP64 direct path on the same system ---------------------------------------------
    if prec == gx.PRECISION_MIXED:
        fclk = ClockSampler(torch.cuda.current_device())
        fclk.start()
        time.sleep(0.3)
        out["fp64"] = fp64_rate(gx, torch, sess, p, dt, flush)
        out["fp64"]["clocks"] = fclk.stop()
        out["mixed_over_fp64"] = value / out["fp64"]["value"]
    sess.close()

    # -- end to end through the C ABI with host buffers ------------------------------------
    out["e2e"] = e2e_rate(gx, torch, p, params, dt, prec)

    # -- adjoint vs forward at the differentiable-fit size --------------------------------
    out["adjoint"] = adjoint_ratio(gx, torch)

    # -- CPU baseline on the host cores -----------------------------------------------------
    q0 = gx.ParticleSet(p.x, p.y, p.z, p.vx, p.vy, p.vz, p.m)
    out["cpu_baseline"] = cpu_reference_rate(q0, eps, args.cpu_seconds)

    # -- the other configurations, each with its own clock record and parity figures --------
    if not args.no_configs:
        out["configs"] = other_configs(gx, torch, args)
    return out


def fp64_rate(gx, torch, sess, p, dt, flush, steps: int = 10) -> dict:
    n = len(p)
    stream = torch.cuda.current_stream()
    sess.set_particles(p)
    sess.compute_accelerations(gx.PRECISION_F64)
    sess.step(1, dt, gx.PRECISION_F64)
    torch.cuda.synchronize()
    ms = []
    for _ in range(steps):
        flush()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        sess.step(1, dt, gx.PRECISION_F64)
        b.record(stream)
        torch.cuda.synchronize()
        ms.append(a.elapsed_time(b))
    v, js = sess.get_config(gx.PRECISION_F64)
    return {"value": steps * n * (n - 1) / (sum(ms) / 1e3) / 1e9, "unit": UNIT, "ms_per_step": sum(ms) / steps,
            "steps": steps, "kernel": gx.describe_variant(gx.PRECISION_F64, v), "jsplit": js}


def e2e_rate(gx, torch, p, params, dt, prec, steps: int = 3) -> dict:
    """gx_leapfrog_step on pinned host arrays: copies in, step, copies out, every step."""
    n = len(p)
    host = {}
    for k in ("x", "y", "z", "vx", "vy", "vz", "ax", "ay", "az", "m"):
        t = torch.empty(n, dtype=torch.float64, pin_memory=True)
        t.numpy()[:] = getattr(p, k)
        host[k] = t.numpy()
    q = gx.ParticleSet(*(host[k] for k in ("x", "y", "z", "vx", "vy", "vz", "m", "ax", "ay", "az")))
    # the ParticleSet keeps the pinned buffers (already contiguous float64)
    for k in host:
        setattr(q, k, host[k])
    gx.compute_cuda_direct_accelerations(q, params, prec)
    gx.cuda_direct_leapfrog_step(q, dt, params, prec)  # warm-up
    times = []
    for _ in range(steps):
        t0 = time.perf_counter()
        gx.cuda_direct_leapfrog_step(q, dt, params, prec)
        times.append(time.perf_counter() - t0)
    return {"value": steps * n * (n - 1) / sum(times) / 1e9, "unit": UNIT, "h2d_bytes_per_step": 10 * 8 * n,
            "d2h_bytes_per_step": 9 * 8 * n, "steps": steps, "step_ms": [round(t * 1e3, 3) for t in times],
            "api": "gx_leapfrog_step (cuda_direct_leapfrog_step) on pinned host arrays, wall clock"}


def adjoint_ratio(gx, torch, n: int = 16384) -> dict:
    """Adjoint step (VJP kernel + reverse kick-drift-kick vector work) vs forward KDK step."""
    from gx import adjoint

    p = gx.ics.two_disk_encounter(n // 2, n // 2, 16384, 0.05)
    params = gx.PhysicsParams(1.0, 0.05)
    X = torch.tensor(np.stack([p.x, p.y, p.z]), device="cuda")
    V = torch.tensor(np.stack([p.vx, p.vy, p.vz]), device="cuda")
    m = torch.tensor(p.m, device="cuda")
    A = adjoint.accelerations(X, m, params, gx.PRECISION_MIXED)
    xb = torch.randn_like(X)
    vb = torch.randn_like(X)
    dt = 0.005

    def fwd():
        adjoint._step(X, V, A, m, dt, params, gx.PRECISION_MIXED)

    def adj():
        nonlocal xb, vb
        vb2 = vb + dt * xb
        g, gm = adjoint.direct_vjp(X, m, dt * vb2, params, gx.PRECISION_MIXED)
        xb = xb + g

    res = {}
    for name, fn in (("fwd_step_ms", fwd), ("adj_step_ms", adj)):
        for _ in range(3):
            fn()
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        for _ in range(20):
            fn()
        b.record()
        torch.cuda.synchronize()
        res[name] = a.elapsed_time(b) / 20
    res["ratio"] = res["adj_step_ms"] / res["fwd_step_ms"]
    res["n"] = n
    res["precision"] = "mixed"
    res["note"] = "checkpoint recompute costs one forward step per adjoint step, reported separately"
    return res


def run_sharded(gx, torch, dist, p, args, rank, world, eps, dt, prec) -> dict:
    """Strong scaling: rank r owns the targets of ownership_range(n, r, world).  Each rank's
    state is resident in an engine session (padded rank-major slots, gx.sharded.ShardedSession);
    a step is the session's kick-drift of the owned bodies, three in-place NCCL all-gathers
    of x, y, z, and the session's force on the owned targets with the closing kick."""
    from gx.sharded import ShardedSession

    n = len(p)
    params = gx.PhysicsParams(1.0, eps)
    pairs = n * (n - 1)
    sh = ShardedSession(n, params)
    sh.set_state(p.x, p.y, p.z, p.vx, p.vy, p.vz, p.m)
    if args.variant is not None:
        sh.backend.session.set_config(prec, args.variant, args.jsplit or 1)
    elif not args.no_autotune and world == 1:
        sh.backend.session.autotune(prec)
    sh.compute_accelerations(prec)
    sh.step(args.warmup, dt, prec)
    flush = l2_flusher(torch)
    torch.cuda.synchronize()
    dist.barrier()
    clocks = ClockSampler(torch.cuda.current_device())
    clocks.start()
    time.sleep(0.3)
    evs = []
    for _ in range(args.steps):
        flush()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        sh.step(1, dt, prec)
        b.record()
        evs.append((a, b))
    torch.cuda.synchronize()
    dist.barrier()
    ms = torch.tensor([sum(a.elapsed_time(b) for a, b in evs)], device="cuda")
    dist.all_reduce(ms, op=dist.ReduceOp.MAX)
    clk = clocks.stop()
    total_s = float(ms) / 1e3
    v, js = sh.backend.session.get_config(prec)
    sh.backend.close()
    # engine kernels per step: the owned range's kick-drift and its force (split reduction fused)
    return {"metric": METRIC, "value": args.steps * pairs / total_s / 1e9, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": float(ms) / args.steps,
            "higher_is_better": True, "scaling": "strong", "vs_baseline": None, "dtype": "f32" if prec == 1 else "f64",
            "data": "synthetic", "gpu_launches": args.steps * 2, "clocks": clk,
            "config": {"workload": f"direct-mixed-n{n}", "n": n, "parallelism": f"targets{world}",
                       "kernel": gx.describe_variant(prec, v), "jsplit": js,
                       "exchange": "three in-place NCCL all-gathers of FP64 positions (24 B/body/step) into the "
                                   "session's padded rank-major arrays",
                       "softening": eps, "dt": dt,
                       "l2": "flushed (256 MiB device write) before every timed step, outside the timed interval"}}


# ---------------------------------------------------------------------------------------
# the other configurations (one JSON line each; not the headline)
# ---------------------------------------------------------------------------------------
def _events(torch):
    return torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)


def wl_ensemble(gx, torch, args) -> dict:
    """512 independent encounters, N_b ~ U[1024, 16384], 200 KDK steps in one graph-captured
    run of the persistent batched kernel, mixed precision, autotuned.  Under torchrun the
    instances are split over the ranks by cost (sharded.partition_instances) and each rank
    steps its own with no exchange; the time is the max over ranks (strong scaling: the 512
    instances are the whole job at every N)."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    off, p, meta = gx.ics.ensemble(512, seed=7)
    steps = args.steps if args.steps != 10 else 200
    pairs = float(np.sum(np.diff(off).astype(np.float64) * (np.diff(off) - 1)))
    from gx.sharded import ensemble_shard

    ids, sub, body = ensemble_shard(off, rank, world)
    b = gx.Batch(sub, gx.PhysicsParams(1.0, 0.05))
    b.set_state(*(np.ascontiguousarray(getattr(p, k)[body]) for k in ("x", "y", "z", "vx", "vy", "vz", "m")))
    tune = b.autotune(gx.PRECISION_MIXED)
    b.compute_accelerations(gx.PRECISION_MIXED)
    d0 = b.diagnostics()
    b.step(args.warmup, 0.005, gx.PRECISION_MIXED)
    b.synchronize()
    st = torch.cuda.Stream()
    b.set_stream(st)
    a, e = _events(torch)
    a.record(st)
    b.step(steps, 0.005, gx.PRECISION_MIXED)
    e.record(st)
    e.synchronize()
    ms = a.elapsed_time(e)
    d1 = b.diagnostics()
    drift = [abs(x.total_energy - y.total_energy) / abs(y.total_energy) for x, y in zip(d1, d0)]
    v = b.get_config(gx.PRECISION_MIXED)
    b.close()
    if world > 1:  # timing only: the max over ranks and the gathered drifts
        import torch.distributed as dist
        t = torch.tensor([ms], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
        got = [None] * world
        dist.all_gather_object(got, drift)
        drift = [x for q in got for x in q]
    return {"metric": "Ginteractions/s (batched ensemble)", "value": steps * pairs / (ms / 1e3) / 1e9,
            "unit": UNIT, "n_gpus": world, "ms_per_step": ms / steps, "steps": steps, "instances": 512,
            "bodies": int(off[-1]), "interactions_per_step": pairs, "autotune_ms_per_eval": tune, "kernel_variant": v,
            "energy_drift": {"median": float(np.median(drift)), "max": float(np.max(drift))},
            "scaling": "strong",
            "config": {"workload": "ensemble-512", "dt": 0.005, "softening": 0.05, "precision": "mixed",
                       "parallelism": f"instances{world}" if world > 1 else "one GPU",
                       "launch": "one CUDA graph of all steps (kick_drift + persistent force per step)"}}


def wl_p2p(gx, torch, args) -> dict:
    """FMM near field of the two-disk workload (N = 65,536 by default, --p2p-n), reference
    octree leaf lists (--leaf-capacity, default 64; theta 0.6) built on the device, P2P on the
    device; --p2p-tpt forces the kernel's targets per thread.  Each form is timed over 20
    launches and checked against the oracle's near loop (the reference's, restated in C)."""
    n = int(getattr(args, "p2p_n", 65536))
    cap = int(getattr(args, "leaf_capacity", 64))
    p = gx.ics.two_disk_encounter(n // 2, n - n // 2, 20260502, 0.02)
    t0 = time.perf_counter()
    lists = gx.build_leaf_lists(p.x, p.y, p.z, p.m, 0.02, 0.6, cap, on_device=True)
    build_s = time.perf_counter() - t0
    tpt = int(getattr(args, "p2p_tpt", 0))
    gx._ffi.call("gx_debug_p2p_targets_per_thread", tpt)
    T = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
    dl = gx.LeafLists(T(lists.leaf_offsets), T(lists.leaf_particles), T(lists.near_offsets), T(lists.near_leaves))
    X = {k: T(getattr(p, k)) for k in ("x", "y", "z", "m")}
    acc = [torch.zeros(n, dtype=torch.float64, device="cuda") for _ in range(3)]
    params = gx.PhysicsParams(1.0, 0.02)
    # ordered source-target pairs minus self pairs
    pairs = lists.n_pairs - n
    out = {"metric": "Ginteractions/s (FMM P2P leaves)", "unit": UNIT, "n": n, "leaves": lists.n_leaves,
           "near_pairs_of_leaves": int(len(lists.near_leaves)), "interactions": int(pairs),
           "leaf_list_build_s": build_s, "targets_per_thread": tpt or "auto",
           "config": {"workload": f"p2p-n{n}", "leaf_capacity": cap, "theta": 0.6}}
    import oracle
    L = dict(leaf_offsets=lists.leaf_offsets, leaf_particles=lists.leaf_particles,
             near_offsets=lists.near_offsets, near_leaves=lists.near_leaves)
    want = oracle.p2p_near(p.x, p.y, p.z, p.m, 1.0, 0.02, L)  # the reference's near loop, restated in C
    wn = np.maximum(np.linalg.norm(want, axis=1), 1e-300)
    for name, prec in (("f64", gx.PRECISION_F64), ("mixed", gx.PRECISION_MIXED), ("f64_exact", gx.PRECISION_F64_EXACT)):
        for a_ in acc:
            a_.zero_()
        gx.p2p_leaves(X["x"], X["y"], X["z"], X["m"], dl, params, *acc, prec)
        got = torch.stack(acc, 1).cpu().numpy()
        err = np.linalg.norm(got - want, axis=1) / wn
        for _ in range(3):
            gx.p2p_leaves(X["x"], X["y"], X["z"], X["m"], dl, params, *acc, prec)
        a, e = _events(torch)
        a.record()
        reps = 20
        for _ in range(reps):
            gx.p2p_leaves(X["x"], X["y"], X["z"], X["m"], dl, params, *acc, prec)
        e.record()
        e.synchronize()
        ms = a.elapsed_time(e) / reps
        rate = pairs / (ms / 1e3) / 1e9
        out[name] = {"ms": ms, "value": rate,
                     "rel_err_vs_oracle_near_field": {"median": float(np.median(err)), "max": float(err.max()),
                                                      "bit_identical": bool(np.array_equal(got, want))}}
        if name == "f64":
            out[name]["fp64_pipe_frac"] = rate * 1e9 * FP64_OPS_PER_P2P_PAIR / fp64_peak_ops(torch)
        elif name == "mixed":
            out[name]["fp32_pipe_frac"] = rate * 1e9 * FMA_PIPE_OPS_PER_INTERACTION / fp32_peak_ops(torch)
    gx._ffi.call("gx_debug_p2p_targets_per_thread", 0)
    out["value"] = out["f64"]["value"]
    return out


def fp32_peak_ops(torch) -> float:
    """FP32 pipe lane-ops/s: SMs x 128 lanes x the maximum SM clock (MEASURED_PEAKS.json)."""
    sms = torch.cuda.get_device_properties(0).multi_processor_count
    return sms * FP32_LANES_PER_SM * float(measured_peaks().get("sm_max_mhz", 1965.0)) * 1e6


def fp64_peak_ops(torch) -> float:
    """FP64 pipe lane-ops/s: SMs x 64 lanes x the maximum SM clock."""
    return fp32_peak_ops(torch) / 2.0


def wl_direct(gx, torch, args, n, eps, dt, steps, ref_targets: int = 0) -> dict:
    """Resident direct-sum sessions (FP64, mixed, exact form) on the two-disk system: `steps`
    KDK steps in CUDA graphs.  With ref_targets > 0, the accelerations of the initial
    positions are checked against the reference's compute_direct_accelerations_for_targets
    (oracle/_ref, or its C restatement) on ref_targets targets of each disk."""
    import oracle
    p = gx.ics.two_disk_encounter(n // 2, n - n // 2, 20260502, eps)
    params = gx.PhysicsParams(1.0, eps)
    out = {"metric": f"Ginteractions/s (direct, N={n})", "unit": UNIT, "n": n, "steps": steps,
           "config": {"workload": f"direct-n{n}", "softening": eps, "dt": dt}}
    ref = None
    if ref_targets:
        ranges = [(0, ref_targets), (n // 2, n // 2 + ref_targets)]
        threads = oracle.default_threads()
        if oracle.ref_available():
            ref = np.concatenate([oracle.ref_direct_targets(p.x, p.y, p.z, p.m, 1.0, eps, b, e, threads=threads)
                                  for b, e in ranges])
            kind = "reference (compute_direct_accelerations_for_targets, oracle/_ref)"
        else:
            idx = np.concatenate([np.arange(b, e) for b, e in ranges])
            ref = oracle.direct_indexed(p.x, p.y, p.z, p.m, 1.0, eps, idx, threads=threads)
            kind = "oracle restatement of compute_direct_accelerations_for_targets"
        sel = np.concatenate([np.arange(b, e) for b, e in ranges])
        out["parity"] = {"vs": kind, "targets": int(len(sel)), "at": "initial positions"}
    for name, prec in (("f64", gx.PRECISION_F64), ("mixed", gx.PRECISION_MIXED), ("f64_exact", gx.PRECISION_F64_EXACT)):
        s = gx.Session(n, params)
        s.set_particles(p)
        if name != "f64_exact":
            s.autotune(prec)
        s.compute_accelerations(prec)
        res = {}
        if ref is not None:
            st0 = s.get_state()
            a0 = np.stack([st0["ax"], st0["ay"], st0["az"]], 1)[sel]
            e = np.linalg.norm(a0 - ref, axis=1) / np.maximum(np.linalg.norm(ref, axis=1), 1e-300)
            res["rel_err"] = {"median": float(np.median(e)), "max": float(e.max()),
                              "bit_identical": bool(np.array_equal(a0, ref))}
        e0 = s.diagnostics().total_energy
        s.step(3, dt, prec)
        s.synchronize()
        st = torch.cuda.Stream()
        s.set_stream(st)
        a, e = _events(torch)
        a.record(st)
        s.step(steps, dt, prec)
        e.record(st)
        e.synchronize()
        ms = a.elapsed_time(e)
        e1 = s.diagnostics().total_energy
        res.update({"ms_per_step": ms / steps, "value": steps * n * (n - 1) / (ms / 1e3) / 1e9,
                    "steps_per_s": steps / (ms / 1e3), "energy_drift": abs(e1 - e0) / abs(e0),
                    "kernel": gx.describe_variant(prec, s.get_config(prec)[0])})
        out[name] = res
        s.close()
    out["value"] = out["mixed"]["value"]
    return out


def cfg0_n1000(gx, torch, args) -> dict:
    """The reference CLI's own workload size: N = 1000 (two disks of 500), softening 0.05,
    dt 0.005, 20 KDK steps in FP64.  The exact form's 20-step trajectory is compared with the
    oracle's (the reference's per-target sum and leapfrog restated in C, pinned bit for bit
    to the reference); the rate repeats the 20-step run for ~0.5 s.  Both step loops are
    timed: one cooperative launch per call (the default for small systems) and CUDA graphs of
    separate kick-drift and force launches."""
    import oracle
    n, eps, dt, steps = 1000, 0.05, 0.005, 20
    p = gx.ics.two_disk_encounter(n // 2, n // 2, 20260502, eps)
    params = gx.PhysicsParams(1.0, eps)
    ref0 = oracle.direct_targets(p.x, p.y, p.z, p.m, 1.0, eps)
    st0 = dict(x=p.x, y=p.y, z=p.z, vx=p.vx, vy=p.vy, vz=p.vz, ax=ref0[:, 0], ay=ref0[:, 1], az=ref0[:, 2])
    want = oracle.leapfrog(st0, p.m, 1.0, eps, dt, steps, solver=1)
    out = {"n": n, "steps": steps, "softening": eps, "dt": dt, "unit": "steps/s",
           "parity_vs": "oracle leapfrog over compute_direct_accelerations_for_targets (20 steps)"}
    forms = (("f64", gx.PRECISION_F64, True), ("f64_exact", gx.PRECISION_F64_EXACT, True),
             ("f64_graphs", gx.PRECISION_F64, False), ("f64_exact_graphs", gx.PRECISION_F64_EXACT, False))
    for name, prec, persistent in forms:
        with gx.Session(n, params) as s:
            s.set_persistent(persistent)
            s.set_particles(p)
            s.compute_accelerations(prec)
            s.step(steps, dt, prec)
            got = s.get_state()
            dx = max(float(np.max(np.abs(got[k] - want[k]))) for k in ("x", "y", "z"))
            same = all(np.array_equal(got[k], want[k]) for k in ("x", "y", "z", "vx", "vy", "vz"))
            st = torch.cuda.Stream()
            s.set_stream(st)
            s.step(steps, dt, prec)
            s.synchronize()
            a, e = _events(torch)
            reps = 0
            t0 = time.perf_counter()
            a.record(st)
            while True:
                s.step(steps, dt, prec)
                reps += 1
                if reps % 25 == 0:
                    s.synchronize()
                    if time.perf_counter() - t0 > 0.5:
                        break
            e.record(st)
            e.synchronize()
            ms = a.elapsed_time(e)
        total = reps * steps
        out[name] = {"steps_per_s": total / (ms / 1e3), "us_per_step": ms * 1e3 / total,
                     "value_gint_s": total * n * (n - 1) / (ms / 1e3) / 1e9, "timed_steps": total,
                     "max_abs_dx_20_steps": dx, "trajectory_bit_identical": same,
                     "launch": "one cooperative launch per 20 steps (small.cu)" if persistent else
                               "CUDA graph of 20 steps (kick-drift + force launches per step)"}
    out["value"] = out["f64"]["steps_per_s"]
    return out


def _clocked(torch, fn):
    c = ClockSampler(torch.cuda.current_device())
    c.start()
    time.sleep(0.25)
    try:
        r = fn()
    finally:
        clk = c.stop()
    r["clocks"] = clk
    return r


def other_configs(gx, torch, args) -> dict:
    """The reference's other configurations, measured in the default run so that their
    figures come with the headline's: N = 1000 (the reference CLI workload), N = 65,536
    (direct FP64 and mixed, the FMM's P2P leaves at capacity 64, the whole FMM on the
    device, each with its error against the reference) and the 512-encounter ensemble."""
    import copy
    sub = copy.copy(args)
    sub.steps, sub.warmup, sub.cpu_seconds = 10, 3, 3.0
    res = {"cfg0_n1000": _clocked(torch, lambda: cfg0_n1000(gx, torch, sub))}
    c1 = {}
    c1["direct"] = _clocked(torch, lambda: wl_direct(gx, torch, sub, 65536, 0.02, 0.002, 100, ref_targets=512))
    c1["p2p_leaf64"] = _clocked(torch, lambda: wl_p2p(gx, torch, sub))
    c1["fmm_leaf64"] = _clocked(torch, lambda: wl_fmm(gx, torch, sub, e2e=False))
    res["cfg1_n65536"] = c1
    ens = copy.copy(sub)
    ens.steps = 200
    res["cfg3_ensemble512"] = _clocked(torch, lambda: wl_ensemble(gx, torch, ens))
    return res


def wl_fit(gx, torch, args) -> dict:
    """Differentiable encounter: N = 16,384, 500 KDK steps, checkpoint every 50; forward and
    backward (adjoint) of the loss over the 6 orbit parameters and all initial positions."""
    from gx import adjoint

    n, steps, dt, K = 16384, 500, 0.005, 50
    p = gx.ics.two_disk_encounter(n // 2, n // 2, 16384, 0.05)
    params = gx.PhysicsParams(1.0, 0.05)
    pos = torch.tensor(p.positions, device="cuda")
    vel = torch.tensor(p.velocities, device="cuda")
    m = torch.tensor(p.m, device="cuda")
    disk2 = torch.tensor(p.group_id == 1, device="cuda")
    truth = torch.tensor([0.04, -0.02, 0.03, 0.02, -0.01, 0.01], dtype=torch.float64, device="cuda")
    res = {"metric": "adjoint/forward cost (differentiable fit)", "unit": "ratio", "n": n, "steps": steps,
           "checkpoint_every": K, "config": {"workload": "fit-n16384", "dt": dt, "softening": 0.05}}
    for name, prec in (("mixed", gx.PRECISION_MIXED), ("f64", gx.PRECISION_F64)):
        with torch.no_grad():
            x0t, v0t = adjoint.encounter_initial_state(pos, vel, disk2, truth)
            target, _ = adjoint.leapfrog(x0t, v0t, m, steps, dt, params, K, prec)
        orbit = torch.zeros(6, dtype=torch.float64, device="cuda", requires_grad=True)
        x0 = pos.clone().requires_grad_(True)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        xs, vs = adjoint.encounter_initial_state(x0, vel, disk2, orbit)
        xT, _ = adjoint.leapfrog(xs, vs, m, steps, dt, params, K, prec)
        loss = ((xT - target) ** 2).sum(1).mean()
        torch.cuda.synchronize()
        t1 = time.perf_counter()
        loss.backward()
        torch.cuda.synchronize()
        t2 = time.perf_counter()
        fwd, bwd = t1 - t0, t2 - t1
        res[name] = {"forward_s": fwd, "backward_s": bwd, "backward_over_forward": bwd / fwd,
                     "adjoint_over_forward_excl_recompute": (bwd - fwd) / fwd, "loss": float(loss)}
    res["adjoint_step"] = adjoint_ratio(gx, torch)
    res["value"] = res["adjoint_step"]["ratio"]
    # the fit itself: recover the 6 orbit parameters from the target snapshot (mixed precision)
    with torch.no_grad():
        x0t, v0t = adjoint.encounter_initial_state(pos, vel, disk2, truth)
        target, _ = adjoint.leapfrog(x0t, v0t, m, steps, dt, params, K, gx.PRECISION_MIXED)
    t0 = time.perf_counter()
    orbit, hist = adjoint.fit_orbit(pos, vel, m, disk2, target, steps, dt, params, iters=args.fit_iters,
                                    lr=0.005, checkpoint_every=K, precision=gx.PRECISION_MIXED)
    torch.cuda.synchronize()
    res["fit"] = {"iterations": args.fit_iters, "seconds": time.perf_counter() - t0, "loss_first": float(hist[0]),
                  "loss_last": float(hist[-1]), "truth": truth.tolist(), "recovered": orbit.tolist(),
                  "position_plus_T_velocity_error": float(torch.linalg.norm(
                      (orbit[:3] + steps * dt * orbit[3:]) - (truth[:3] + steps * dt * truth[3:])))}
    return res


FP64_LANES_PER_SM = 64
# FP64 pipe instructions of one far-field (target, node) evaluation at expansion order 4
# (m2p_one<4> in csrc/fmm.cu: offsets, softened r^-1 with one refinement step, g1..g5,
# the quadrupole, octupole and hexadecapole contractions and the accumulation; 171.3
# measured as DADD + DMUL + DFMA thread instructions per pair), and of one FP64 near-field
# interaction (offsets, r^2 + eps^2, r^-3 with one refinement step, m r^-3, three
# accumulations), the count of the direct FP64 kernel.
FP64_OPS_PER_M2P_PAIR = 171
FP64_OPS_PER_P2P_PAIR = 17


def wl_fmm_session(gx, torch, args) -> dict:
    """The FMM KDK step of the N = 65,536 workload (leaf 64, theta 0.6, order 4, FP64) in a
    resident session only: gx_session_set_fmm, --warmup calls of min(--steps, 32) steps (the
    first sizes the pools and captures the chunk's graph), then --steps steps timed on the
    session's stream.  Small enough to run under a profiler."""
    n, cap, theta, eps, dt = 65536, 64, 0.6, 0.02, 0.002
    p = gx.ics.two_disk_encounter(n // 2, n // 2, 20260502, eps)
    params, opt = gx.PhysicsParams(1.0, eps), gx.FmmOptions(theta, cap, 32, 4)
    st = torch.cuda.Stream()
    with gx.Session(n, params) as s:
        s.set_stream(st)
        s.set_fmm(opt)
        s.set_particles(p)
        s.compute_accelerations(gx.PRECISION_F64)
        for _ in range(max(1, args.warmup)):
            s.step(min(args.steps, 32), dt, gx.PRECISION_F64)
        s.synchronize()
        a, e = _events(torch)
        a.record(st)
        s.step(args.steps, dt, gx.PRECISION_F64)
        e.record(st)
        e.synchronize()
        ms = a.elapsed_time(e) / args.steps
    return {"metric": "FMM KDK steps/s (N=65536, leaf 64, theta 0.6, p=4, FP64, resident session)",
            "value": 1e3 / ms, "unit": "steps/s", "ms_per_step": ms, "steps": args.steps, "warmup": args.warmup,
            "higher_is_better": True, "dtype": "f64", "data": "synthetic",
            "config": {"workload": "fmm-session-n65536", "leaf_capacity": cap, "theta": theta, "order": 4}}


def wl_fmm(gx, torch, args, e2e: bool = True) -> dict:
    """The reference FMM solver on the N = 65,536 two-disk workload (leaf_capacity 64,
    theta 0.6, expansion order 4, softening 0.02, dt 0.002): one KDK step = kick-drift,
    a full FMM force evaluation (octree, lists, moments, far and near field, all on the
    device), kick.  Device-resident state; the e2e line runs the public API on host
    arrays.  CPU baseline: the reference's own FastMultipoleSolver (build + evaluate_particle
    over all host threads), timed on a target sample and extrapolated to one evaluation."""
    import oracle
    n, cap, theta, eps, dt = 65536, 64, 0.6, 0.02, 0.002
    steps = args.steps if args.steps != 10 else 20
    p = gx.ics.two_disk_encounter(n // 2, n // 2, 20260502, eps)
    params, opt = gx.PhysicsParams(1.0, eps), gx.FmmOptions(theta, cap, 32, 4)
    D = {k: torch.tensor(getattr(p, k), device="cuda") for k in ("x", "y", "z", "vx", "vy", "vz", "m")}
    A = [torch.zeros(n, dtype=torch.float64, device="cuda") for _ in range(3)]
    st = torch.cuda.Stream()
    sp = st.cuda_stream
    P3 = lambda *ts: [t.data_ptr() for t in ts]

    def step():
        gx._ffi.call("gx_kick_drift", n, *P3(D["x"], D["y"], D["z"], D["vx"], D["vy"], D["vz"], *A), 0.5 * dt, dt, sp)
        gx.fmm.fmm_accelerations(D["x"], D["y"], D["z"], D["m"], *A, params, opt, gx.PRECISION_F64, stream=sp)
        gx._ffi.call("gx_kick", n, *P3(D["vx"], D["vy"], D["vz"], *A), 0.5 * dt, sp)

    with torch.cuda.stream(st):
        stats = gx.fmm.fmm_accelerations(D["x"], D["y"], D["z"], D["m"], *A, params, opt, gx.PRECISION_F64, stream=sp)
        a0 = torch.stack(A, 1).cpu().numpy()
        for _ in range(max(3, args.warmup)):
            step()
        st.synchronize()
        clocks = ClockSampler(torch.cuda.current_device())
        clocks.start()
        time.sleep(0.3)
        e0, e1 = _events(torch)
        e0.record(st)
        for _ in range(steps):
            step()
        e1.record(st)
        e1.synchronize()
        clk = clocks.stop()
        ms = e0.elapsed_time(e1) / steps
        # phase times of a few evaluations (same state, same stream)
        phases = []
        for _ in range(5):
            _, ph = gx.fmm.fmm_accelerations_timed(D["x"], D["y"], D["z"], D["m"], *A, params, opt, gx.PRECISION_F64,
                                                   stream=sp)
            phases.append(ph)
    ph = {k: float(np.median([q[k] for q in phases])) for k in gx.fmm.PHASES}
    sms = torch.cuda.get_device_properties(0).multi_processor_count
    peaks = json.loads(Path(__file__).with_name("MEASURED_PEAKS.json").read_text()) \
        if Path(__file__).with_name("MEASURED_PEAKS.json").exists() else {}
    mhz = float(peaks.get("sm_max_mhz", 1965.0))
    fp64_peak = sms * FP64_LANES_PER_SM * mhz * 1e6 / 1e12
    near_int = stats.near_pairs - n  # ordered pairs, self pairs excluded
    p2p_ach = near_int * FP64_OPS_PER_P2P_PAIR / (ph["near_field"] / 1e3) / 1e12
    m2p_ach = stats.far_pairs * FP64_OPS_PER_M2P_PAIR / (ph["far_field"] / 1e3) / 1e12
    dominant = "near_field" if ph["near_field"] >= ph["far_field"] else "far_field"
    roof = {"bound": "fp64_pipe", "kernel": "p2p_kernel<F64> (near field)" if dominant == "near_field"
            else "fmm_m2p_kernel<4> (far field)",
            "achieved": p2p_ach if dominant == "near_field" else m2p_ach, "peak": fp64_peak,
            "unit": "T FP64-pipe lane-ops/s",
            "frac": (p2p_ach if dominant == "near_field" else m2p_ach) / fp64_peak,
            "peak_basis": f"{sms} SMs x {FP64_LANES_PER_SM} FP64 lanes x {mhz:.0f} MHz (sm_max_mhz of "
                          "MEASURED_PEAKS.json); FP64 arithmetic bounds both kernels, not HBM",
            "near_field": {"interactions": near_int, "ops_per_interaction": FP64_OPS_PER_P2P_PAIR,
                           "phase_ms": ph["near_field"], "achieved": p2p_ach, "frac": p2p_ach / fp64_peak,
                           "note": "phase = plan (count, scan) + kernel"},
            "far_field": {"pairs": stats.far_pairs, "ops_per_pair": FP64_OPS_PER_M2P_PAIR,
                          "phase_ms": ph["far_field"], "achieved": m2p_ach, "frac": m2p_ach / fp64_peak},
            "traffic": None,
            "traffic_note": "node records, bodies and lists stay in L2: ncu DRAM reads 7.7 MB (far field) and "
                            "5.1 MB (near field) per evaluation at this size"}

    # the resident session with the FMM force: chunks of 32 KDK steps replayed as CUDA graphs
    # (no host synchronisation inside a chunk; one read of the pool-overflow word after it)
    sess_steps = 64
    with gx.Session(n, params) as sess:
        sess.set_fmm(opt)
        sess.set_particles(p)
        sess.compute_accelerations(gx.PRECISION_F64)
        sst = torch.cuda.Stream()
        sess.set_stream(sst)
        sess.step(32, dt, gx.PRECISION_F64)  # sizes the pools, captures the graph
        sess.synchronize()
        s0, s1 = _events(torch)
        s0.record(sst)
        sess.step(sess_steps, dt, gx.PRECISION_F64)
        s1.record(sst)
        s1.synchronize()
        sess_ms = s0.elapsed_time(s1) / sess_steps
    session = {"value": 1e3 / sess_ms, "unit": "steps/s", "ms_per_step": sess_ms, "steps": sess_steps,
               "launch": "gx_session_step with the FMM force: CUDA graphs of 32 KDK steps, device pools sized by "
                         "capacity, one read of the overflow word per chunk"}

    # e2e: the public API on host arrays (H2D of x, y, z, m and D2H of a inside the call)
    e2e_rate_ = None
    if e2e:
        q = p.copy()
        gx.fmm.compute_fmm_accelerations(q, params, opt)
        t0 = time.perf_counter()
        e2e_steps = max(3, steps // 2)
        for _ in range(e2e_steps):
            q.vx += q.ax * (0.5 * dt); q.vy += q.ay * (0.5 * dt); q.vz += q.az * (0.5 * dt)
            q.x += q.vx * dt; q.y += q.vy * dt; q.z += q.vz * dt
            gx.fmm.compute_fmm_accelerations(q, params, opt)
            q.vx += q.ax * (0.5 * dt); q.vy += q.ay * (0.5 * dt); q.vz += q.az * (0.5 * dt)
        e2e_rate_ = e2e_steps / (time.perf_counter() - t0)

    # the mixed form (both fields in FP32 arithmetic on FP64 offsets) on the same system
    Dm = {k: torch.tensor(getattr(p, k), device="cuda") for k in ("x", "y", "z", "vx", "vy", "vz", "m")}
    Am = [torch.zeros(n, dtype=torch.float64, device="cuda") for _ in range(3)]

    def step_mixed():
        gx._ffi.call("gx_kick_drift", n, *P3(Dm["x"], Dm["y"], Dm["z"], Dm["vx"], Dm["vy"], Dm["vz"], *Am), 0.5 * dt, dt,
                     sp)
        gx.fmm.fmm_accelerations(Dm["x"], Dm["y"], Dm["z"], Dm["m"], *Am, params, opt, gx.PRECISION_MIXED, stream=sp)
        gx._ffi.call("gx_kick", n, *P3(Dm["vx"], Dm["vy"], Dm["vz"], *Am), 0.5 * dt, sp)

    with torch.cuda.stream(st):
        gx.fmm.fmm_accelerations(Dm["x"], Dm["y"], Dm["z"], Dm["m"], *Am, params, opt, gx.PRECISION_MIXED, stream=sp)
        am0 = torch.stack(Am, 1).cpu().numpy()
        for _ in range(max(3, args.warmup)):
            step_mixed()
        st.synchronize()
        m0, m1 = _events(torch)
        m0.record(st)
        for _ in range(steps):
            step_mixed()
        m1.record(st)
        m1.synchronize()
        ms_mixed = m0.elapsed_time(m1) / steps
    em = np.linalg.norm(am0 - a0, axis=1) / np.linalg.norm(a0, axis=1)
    mixed = {"value": 1e3 / ms_mixed, "unit": "steps/s", "ms_per_step": ms_mixed,
             "rel_err_vs_f64": {"median": float(np.median(em)), "max": float(em.max()), "bodies": n}}

    out = {"metric": "FMM KDK steps/s (N=65536, leaf 64, theta 0.6, p=4, FP64)", "value": session["value"],
           "session": session, "evaluation_loop": {"value": 1e3 / ms, "unit": "steps/s", "ms_per_step": ms,
                                                   "launch": "kick-drift, gx_fmm_accel (two host reads), kick"},
           "unit": "steps/s", "n_gpus": 1, "steps": steps, "warmup": max(3, args.warmup), "ms_per_step": sess_ms,
           "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
           "phases_ms_per_eval": ph, "stats": stats.__dict__,
           "gpu_launches": steps * (19 + stats.tree_levels + 2),
           "e2e": None if e2e_rate_ is None else
           {"value": e2e_rate_, "unit": "steps/s", "h2d_bytes_per_step": 4 * n * 8, "d2h_bytes_per_step": 3 * n * 8},
           "roofline": roof, "clocks": clk, "mixed": mixed,
           "config": {"workload": "fmm-n65536", "n": n, "leaf_capacity": cap, "theta": theta, "expansion_order": 4,
                      "softening": eps, "dt": dt, "near_field_precision": "f64",
                      "l2": "inputs (5 MiB) stay L2-resident; not flushed between steps"}}
    if oracle.ref_available():
        threads = os.cpu_count() or 1
        _, b_s, e_s, k = oracle.ref_fmm_timed(p.x, p.y, p.z, p.m, 1.0, eps, theta, cap, 4, 256, threads)
        per_target = e_s / max(k, 1)
        stride = max(1, int(np.ceil(n * per_target / max(args.cpu_seconds, 1.0))))
        acc, b_s, e_s, k = oracle.ref_fmm_timed(p.x, p.y, p.z, p.m, 1.0, eps, theta, cap, 4, stride, threads)
        eval_s = b_s + e_s * n / k
        ok = ~np.isnan(acc[:, 0])
        err = np.linalg.norm(a0[ok] - acc[ok], axis=1) / np.linalg.norm(acc[ok], axis=1)
        out["cpu_baseline"] = {"value": 1.0 / eval_s, "unit": "steps/s", "cores": threads, "kind": "reference",
                               "sample": f"FastMultipoleSolver::build once ({b_s:.3f} s) + evaluate_particle on every "
                                         f"{stride}-th body ({k} bodies, {e_s:.2f} s on {threads} threads), "
                                         "extrapolated to all bodies; one evaluation per step"}
        out["parity_vs_reference"] = {"bodies": int(ok.sum()), "rel_err_max": float(err.max()),
                                      "rel_err_median": float(np.median(err))}
    return out


def wl_fmm_evals(gx, torch, args) -> dict:
    """FMM force evaluations alone (no KDK step) of the two-disk system (N = 65,536 by default,
    --p2p-n; eps 0.02, theta 0.6, order 4) on device arrays, with --leaf-capacity and
    --precision (f64 or mixed): --warmup untimed evaluations, then --steps timed ones, and the
    device time per phase (tree, moments, lists, far field, near field) of a few more.  The
    case the FMM kernel profiles capture (the P2P and M2P launches of one evaluation)."""
    n, eps = int(getattr(args, "p2p_n", 65536)), 0.02
    p = gx.ics.two_disk_encounter(n // 2, n - n // 2, 20260502, eps)
    prec = gx.PRECISION_MIXED if args.precision == "mixed" else gx.PRECISION_F64
    params, opt = gx.PhysicsParams(1.0, eps), gx.FmmOptions(0.6, args.leaf_capacity, 32, 4)
    D = {k: torch.tensor(getattr(p, k), device="cuda") for k in ("x", "y", "z", "m")}
    A = [torch.zeros(n, dtype=torch.float64, device="cuda") for _ in range(3)]

    def evaluate():
        return gx.fmm.fmm_accelerations(D["x"], D["y"], D["z"], D["m"], *A, params, opt, prec)

    for _ in range(args.warmup):
        evaluate()
    torch.cuda.synchronize()
    e0, e1 = _events(torch)
    e0.record()
    for _ in range(args.steps):
        st = evaluate()
    e1.record()
    e1.synchronize()
    ms = e0.elapsed_time(e1) / args.steps
    phases = []
    for _ in range(3):
        _, ph = gx.fmm.fmm_accelerations_timed(D["x"], D["y"], D["z"], D["m"], *A, params, opt, prec)
        phases.append(ph)
    ph = {k: float(np.median([q[k] for q in phases])) for k in gx.fmm.PHASES}
    return {"metric": f"FMM evaluations/s (N={n})", "value": 1e3 / ms, "unit": "evaluations/s", "ms_per_eval": ms,
            "steps": args.steps, "warmup": args.warmup, "stats": st.__dict__, "dtype": args.precision,
            "phases_ms": ph,
            "note": "includes the two host synchronisations of each evaluation (node and list sizes)",
            "config": {"workload": "fmm-evals", "n": n, "leaf_capacity": args.leaf_capacity, "theta": 0.6,
                       "expansion_order": 4, "softening": eps, "precision": args.precision}}


def wl_snapshots(gx, torch, args) -> dict:
    """Snapshot output from the resident N = 2^20 session (mixed precision): 20 KDK steps with
    a snapshot (reference CSV + binary) every 5 steps vs the same steps without; the stepping
    stream pays only the device-to-device copy, the writer thread does the rest."""
    import shutil
    import tempfile
    n, eps, dt, steps, every = 1 << 20, 0.01, 0.001, 20, 5
    p = gx.ics.two_disk_encounter(n // 2, n - n // 2, 20260502, eps, mass1=1.0, mass2=1.0 / 3.0)
    out = tempfile.mkdtemp(prefix="gx_snap_")
    try:
        with gx.Session(n, gx.PhysicsParams(1.0, eps)) as s, gx.SnapshotWriter(out, n, binary=True, slots=2) as w:
            s.set_particles(p)
            s.compute_accelerations(gx.PRECISION_MIXED)
            st = torch.cuda.Stream()
            s.set_stream(st)
            s.step(3, dt, gx.PRECISION_MIXED)
            s.synchronize()
            res = {}
            for label, snap in (("without", False), ("with", True)):
                a, e = _events(torch)
                t0 = time.perf_counter()
                a.record(st)
                for k in range(steps // every):
                    s.step(every, dt, gx.PRECISION_MIXED)
                    if snap:
                        s.snapshot(w, k, k * every * dt)
                e.record(st)
                e.synchronize()
                res[label] = {"device_ms": a.elapsed_time(e), "wall_ms_to_last_step": (time.perf_counter() - t0) * 1e3}
            t1 = time.perf_counter()
            w.flush()
            drain = time.perf_counter() - t1
            # the stream's own cost of one snapshot: events around the call on an idle stream
            copies = []
            for k in range(3):
                a, e = _events(torch)
                a.record(st)
                s.snapshot(w, 100 + k, 0.0)
                e.record(st)
                e.synchronize()
                copies.append(a.elapsed_time(e))
                w.flush()
        snaps = steps // every
        csv_bytes = sum(os.path.getsize(os.path.join(out, f)) for f in os.listdir(out)
                        if f.endswith(".csv") and f.startswith("snapshot_0000")) / snaps * snaps
    finally:
        shutil.rmtree(out, ignore_errors=True)
    over = (res["with"]["device_ms"] - res["without"]["device_ms"]) / snaps
    cpu = None
    import oracle
    if oracle.ref_available():
        # the reference's SnapshotWriter on the same state (one snapshot, single thread)
        ref_dir = tempfile.mkdtemp(prefix="gx_refsnap_")
        try:
            st0 = {k: getattr(p, k) for k in ("x", "y", "z", "vx", "vy", "vz")}
            st0.update(ax=np.zeros(n), ay=np.zeros(n), az=np.zeros(n))
            t0 = time.perf_counter()
            oracle.ref_write_outputs(ref_dir, st0, p.m, None, 0, 0.0, np.zeros(13))
            cs = time.perf_counter() - t0
        finally:
            shutil.rmtree(ref_dir, ignore_errors=True)
        cpu = {"value": cs * 1e3, "unit": "ms", "cores": 1, "kind": "reference",
               "sample": "SnapshotWriter::write_snapshot of the same N=2^20 state (the reference writes on the "
                         "step loop's own thread, after a full device-to-host copy)"}
    return {"metric": "stream time per snapshot (N=2^20, device copy)", "value": float(np.median(copies)),
            "cpu_baseline": cpu,
            "unit": "ms", "step_overhead_ms_per_snapshot": over,
            "higher_is_better": False, "steps": steps, "snapshot_every": every, "snapshots": snaps,
            "step_ms_without": res["without"]["device_ms"] / steps, "step_ms_with": res["with"]["device_ms"] / steps,
            "writer_drain_s_after_last_step": drain, "csv_bytes_per_snapshot": csv_bytes / snaps,
            "config": {"workload": "snapshots-n1048576", "n": n, "formats": "reference CSV + binary SoA",
                       "precision": "mixed"}}


def wl_ics(gx, torch, args) -> dict:
    """Initial conditions of the 512-encounter ensemble generated on the device: 1024 disks
    (N_b ~ U[1024, 16384] per encounter, two disks each, mass ratio ~ U[1, 10], impact
    parameter ~ U[0.5, 4], inclination ~ U[0, 90] deg) with the reference's disk model.
    CPU baseline: the reference's generate_galaxies (one mt19937_64 stream) on a sample."""
    import oracle
    rng = np.random.Generator(np.random.PCG64(7))
    sizes = 2 * rng.integers(512, 8193, 512)
    ratio, impact, incl = rng.uniform(1, 10, 512), rng.uniform(0.5, 4.0, 512), rng.uniform(0, np.pi / 2, 512)
    gals = []
    for b in range(512):
        h = int(sizes[b]) // 2
        gals.append(dict(n_particles=h, mass=1.0, radius=1.0, thickness=0.05, group_id=2 * b))
        gals.append(dict(n_particles=h, mass=1.0 / ratio[b], radius=1.0, thickness=0.05, group_id=2 * b + 1,
                         position=(10.0, impact[b], 0.0), velocity=(-0.5, 0.0, 0.0), inclination=incl[b]))
    params = gx.PhysicsParams(1.0, 0.05)
    n = int(sum(g["n_particles"] for g in gals))
    st = torch.cuda.Stream()
    with torch.cuda.stream(st):
        for _ in range(3):
            out = gx.ics.generate_galaxies(gals, params, 11, device="cuda", stream=st.cuda_stream)
        a, e = _events(torch)
        a.record(st)
        reps = 10
        for _ in range(reps):
            out = gx.ics.generate_galaxies(gals, params, 11, device="cuda", stream=st.cuda_stream)
        e.record(st)
        e.synchronize()
    ms = a.elapsed_time(e) / reps
    t0 = time.perf_counter()
    host = gx.ics.generate_galaxies(gals, params, 11)
    e2e_s = time.perf_counter() - t0
    res = {"metric": "bodies generated per second (512-encounter ensemble ICs)", "value": n / (ms / 1e3),
           "unit": "bodies/s", "bodies": n, "galaxies": len(gals), "ms_per_generation": ms,
           "e2e": {"value": n / e2e_s, "unit": "bodies/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 7 * 8 * n + 4 * n},
           "config": {"workload": "ics-ensemble512", "model": "reference disk (initial_conditions.cpp:37-89)",
                      "random_numbers": "Philox4x32-10, counter (galaxy, body, block)"}}
    if oracle.ref_available():
        sample = gals[: max(2, len(gals) // 16)]
        ns = int(sum(g["n_particles"] for g in sample))
        t0 = time.perf_counter()
        oracle.ref_generate_galaxies(sample, 1.0, 0.05, 11)
        cs = time.perf_counter() - t0
        res["cpu_baseline"] = {"value": ns / cs, "unit": "bodies/s", "cores": 1, "kind": "reference",
                               "sample": f"generate_galaxies on the first {len(sample)} disks ({ns} bodies, {cs:.2f} s)"}
    del host, out
    return res


OTHER_WORKLOADS = {
    "ensemble": wl_ensemble,
    "fmm-n65536": wl_fmm,
    "fmm-session-n65536": wl_fmm_session,
    "fmm-evals": wl_fmm_evals,
    "snapshots-n1048576": wl_snapshots,
    "ics-ensemble512": wl_ics,
    "p2p-n65536": wl_p2p,
    "p2p": wl_p2p,
    "direct-n65536": lambda gx, torch, args: wl_direct(gx, torch, args, 65536, 0.02, 0.002, 100),
    "direct-n1000": lambda gx, torch, args: wl_direct(gx, torch, args, 1000, 0.05, 0.005, 20),
    "fit-n16384": wl_fit,
}


def reference_arm(args, rank, n, eps, dt):
    """The reference's own CPU direct sum (compute_direct_accelerations_for_targets, its
    unmodified sources in oracle/_ref) on all host threads; each step a bounded sample of
    targets of the same N=2^20 system."""
    if rank != 0:
        return
    gx = load_gx()
    p = gx.ics.two_disk_encounter(n // 2, n - n // 2, 20260502, eps, mass1=1.0, mass2=1.0 / 3.0)
    per_step_s = max(2.0, min(12.0, 150.0 / max(1, args.steps + args.warmup)))
    first = cpu_reference_rate(p, eps, per_step_s)
    rates = []
    for k in range(args.steps):
        rates.append(cpu_reference_rate(p, eps, per_step_s)["value"])
    value = float(np.median(rates))
    print(json.dumps({
        "metric": METRIC, "value": value, "unit": UNIT, "impl": "reference", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": n * (n - 1) / (value * 1e9) * 1e3,
        "higher_is_better": True, "scaling": "strong", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": f"direct-mixed-n{n}", "n": n, "softening": eps, "dt": dt,
                   "note": "CPU timing extrapolated from a bounded target sample per step"},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": first["cores"], "kind": first["kind"],
                         "sample": first["sample"]},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }), flush=True)


if __name__ == "__main__":
    main()

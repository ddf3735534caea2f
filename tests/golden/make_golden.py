"""Regenerates the golden fixtures of tests/golden/ (run where a reference checkout is
present: python tests/golden/make_golden.py REFERENCE_ROOT).

Sources, all produced by the reference itself:
* experiments/benchmarks/local_cpu/outputs/direct_{250,1000}_r1/ and fmm_1000_r1/ -- the
  reference's own committed snapshots and diagnostics (17 significant digits);
* oracle/_ref/libgxref.so -- the reference's unmodified sources compiled here (ref_wrap.cpp):
  the smoke-test known-answer case (cpp/tests/smoke_tests.cpp:54-123), the FMM leaf lists and
  far field of fmm_1000_r1's step 0, and a 20-step direct run of the N=1000 two-disk workload.
"""
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))
import oracle  # noqa: E402

if len(sys.argv) < 2:
    sys.exit("usage: python tests/golden/make_golden.py REFERENCE_ROOT (the reference checkout)")
REF = Path(sys.argv[1])
OUT = Path(__file__).resolve().parent
BENCH = REF / "experiments/benchmarks/local_cpu/outputs"


def load_csv(path):
    a = np.loadtxt(path, delimiter=",", comments="#", skiprows=2)
    return dict(group=a[:, 1].astype(np.uint32), m=a[:, 2], x=a[:, 3], y=a[:, 4], z=a[:, 5], vx=a[:, 6],
                vy=a[:, 7], vz=a[:, 8], ax=a[:, 9], ay=a[:, 10], az=a[:, 11])


def load_diag(path):
    return np.loadtxt(path, delimiter=",", skiprows=1)


def snapshots():
    out = {}
    for name in ("direct_250_r1", "direct_1000_r1"):
        d = BENCH / name
        for step in (0, 20):
            s = load_csv(d / f"snapshot_{step:06d}.csv")
            for k, v in s.items():
                out[f"{name}/s{step}/{k}"] = v
        out[f"{name}/diagnostics"] = load_diag(d / "diagnostics.csv")
    # softening 0.025, dt 0.01, 20 steps, G 1 (experiments/benchmarks/local_cpu/configs/direct_*_r1.toml)
    np.savez_compressed(OUT / "direct_snapshots.npz", **out)


def smoke80():
    x, y, z, m = oracle.ref_smoke80_inputs()
    a2 = oracle.ref_direct(x, y, z, m, 1.0, 0.03)
    a3 = oracle.ref_direct_targets(x, y, z, m, 1.0, 0.03, 0, 80)
    tb = dict(x=np.array([-0.5, 0.5]), y=np.zeros(2), z=np.array([0.2, -0.2]), m=np.array([2.0, 3.0]))
    tb_a = oracle.ref_direct(tb["x"], tb["y"], tb["z"], tb["m"], 1.0, 0.0)
    np.savez_compressed(OUT / "smoke80.npz", x=x, y=y, z=z, m=m, a_direct=a2, a_targets=a3, two_body_x=tb["x"],
                        two_body_y=tb["y"], two_body_z=tb["z"], two_body_m=tb["m"], two_body_a=tb_a)


def fmm1000():
    s = load_csv(BENCH / "fmm_1000_r1" / "snapshot_000000.csv")
    s20 = load_csv(BENCH / "fmm_1000_r1" / "snapshot_000020.csv")
    lists, far = oracle.ref_fmm_split(s["x"], s["y"], s["z"], s["m"], 1.0, 0.025, 0.58, 16, 4)
    np.savez_compressed(OUT / "fmm1000.npz", x=s["x"], y=s["y"], z=s["z"], m=s["m"], ax=s["ax"], ay=s["ay"],
                        az=s["az"], vx=s["vx"], vy=s["vy"], vz=s["vz"], far=far, theta=0.58, leaf_capacity=16,
                        softening=0.025, dt=0.01, steps=20,
                        **{f"{k}20": s20[k] for k in ("x", "y", "z", "vx", "vy", "vz", "ax", "ay", "az")}, **lists)


def readme1000():
    """experiments/validation/readme_1000_body_collision: the reference's 299-step FMM run
    (dt 0.012, theta 0.58, leaf 16, softening 0.025, order 4) -- its step-0 state, the
    accelerations at step 10, positions and velocities at steps 10, 40, 100 and 299, and every
    diagnostics row."""
    d = REF / "experiments/validation/readme_1000_body_collision"
    s0 = load_csv(d / "snapshot_000000.csv")
    out = {f"{k}0": s0[k] for k in ("x", "y", "z", "vx", "vy", "vz", "ax", "ay", "az")}
    for step in (10, 40, 100, 299):
        s = load_csv(d / f"snapshot_{step:06d}.csv")
        keys = ("x", "y", "z", "vx", "vy", "vz") + (("ax", "ay", "az") if step == 10 else ())
        out.update({f"{k}{step}": s[k] for k in keys})
    np.savez_compressed(OUT / "readme1000.npz", m=s0["m"], group=s0["group"], diagnostics=load_diag(d / "diagnostics.csv"),
                        dt=0.012, theta=0.58, leaf_capacity=16, softening=0.025, steps=299,
                        checkpoints=np.array([10, 40, 100, 299]), **out)


def cfg0():
    sys.path.insert(0, str(ROOT))
    import importlib.util
    spec = importlib.util.spec_from_file_location(
        "gx_pkg", ROOT / "galaxy-collision-simulation_b200" / "__init__.py",
        submodule_search_locations=[str(ROOT / "galaxy-collision-simulation_b200")])
    pkg = importlib.util.module_from_spec(spec)
    sys.modules["gx_pkg"] = pkg
    spec.loader.exec_module(pkg)
    p = pkg.ics.two_disk_encounter(500, 500, 20260502, 0.05)
    eps, dt = 0.05, 0.005
    a0 = oracle.ref_direct(p.x, p.y, p.z, p.m, 1.0, eps)
    st = dict(x=p.x, y=p.y, z=p.z, vx=p.vx, vy=p.vy, vz=p.vz, ax=a0[:, 0], ay=a0[:, 1], az=a0[:, 2])
    d0 = oracle.ref_diagnostics(p.x, p.y, p.z, p.vx, p.vy, p.vz, p.m, 1.0, eps)
    s20 = oracle.ref_leapfrog(st, p.m, 1.0, eps, dt, 20)
    d20 = oracle.ref_diagnostics(s20["x"], s20["y"], s20["z"], s20["vx"], s20["vy"], s20["vz"], p.m, 1.0, eps)
    np.savez_compressed(OUT / "cfg0_n1000.npz", x0=p.x, y0=p.y, z0=p.z, vx0=p.vx, vy0=p.vy, vz0=p.vz, m=p.m,
                        a0=a0, diag0=d0, diag20=d20, **{f"{k}20": v for k, v in s20.items()}, softening=eps, dt=dt)


if __name__ == "__main__":
    snapshots()
    smoke80()
    fmm1000()
    cfg0()
    readme1000()
    for f in sorted(OUT.glob("*.npz")):
        print(f.name, f.stat().st_size)

"""Adjoint kernel and the differentiable leapfrog (B200).

No reference counterpart exists (the reference has no gradients), so parity is pinned to
(1) the oracle's VJP restatement, (2) plain FP64 PyTorch O(N^2) autograd through the same
leapfrog, (3) FP64 central finite differences -- gradients within 1e-5 relative.
"""
import numpy as np
import pytest
import torch

import gx
import oracle
from gx import adjoint
from conftest import rel_err

pytestmark = pytest.mark.gpu

F64, MIX = gx.PRECISION_F64, gx.PRECISION_MIXED
DEV = "cuda"
# Mixed-precision bounds, about 4x the figures measured on B200 for these inputs:
MIXED_VJP_MAX = 2e-4         # position VJP, max relative error per body vs the oracle (measured 4.9e-5)
MIXED_VJP_MASS_MAX = 1e-3    # mass VJP, max relative error per body vs the oracle (measured 1.7e-4)
MIXED_ORBIT_GRAD_TOL = 2e-9  # mixed orbit gradient vs FP64 central differences, relative to
                             # max |g| (measured 4.0e-10, the level of the differences' own error)


def torch_accel(x, m, eps):
    d = x[None, :, :] - x[:, None, :]  # d[i, j] = x_j - x_i
    s = (d * d).sum(-1) + eps * eps
    eye = torch.eye(len(m), dtype=torch.bool, device=x.device)
    inv3 = torch.where(eye, torch.zeros_like(s), s.clamp_min(1e-300) ** -1.5)
    return (d * (m[None, :] * inv3)[..., None]).sum(1)


def torch_leapfrog(x0, v0, m, steps, dt, eps):
    h = 0.5 * dt
    a = torch_accel(x0, m, eps)
    x, v = x0, v0
    for _ in range(steps):
        v = v + a * h
        x = x + v * dt
        a = torch_accel(x, m, eps)
        v = v + a * h
    return x, v


@pytest.mark.parametrize("prec", [F64, MIX])
def test_vjp_kernel_vs_oracle(prec):
    rng = np.random.default_rng(2)
    p = gx.ics.two_disk_encounter(400, 377, 6, 0.05)
    lam = rng.normal(size=(len(p), 3))
    gpos, gm = oracle.direct_vjp(p.x, p.y, p.z, p.m, lam[:, 0], lam[:, 1], lam[:, 2], 1.0, 0.05)
    X = torch.tensor(np.stack([p.x, p.y, p.z]), device=DEV)
    L = torch.tensor(lam.T.copy(), device=DEV)
    m = torch.tensor(p.m, device=DEV)
    GX, GM = adjoint.direct_vjp(X, m, L, gx.PhysicsParams(1.0, 0.05), prec)
    got = GX.t().cpu().numpy()
    e = rel_err(got, gpos)
    em = np.abs(GM.cpu().numpy() - gm) / np.maximum(np.abs(gm), 1e-12)
    if prec == F64:
        assert np.median(e) <= 1e-13 and e.max() <= 1e-10
        assert np.median(em) <= 1e-13
    else:
        print(f"mixed VJP vs oracle: median {np.median(e):.3e} max {e.max():.3e}; "
              f"mass median {np.median(em):.3e} max {em.max():.3e}")
        assert np.median(e) <= 1e-5 and np.median(em) <= 1e-5
        assert e.max() <= MIXED_VJP_MAX and em.max() <= MIXED_VJP_MASS_MAX


def _setup(n=512, seed=5):
    p = gx.ics.two_disk_encounter(n // 2, n // 2, seed, 0.05)
    pos = torch.tensor(p.positions, device=DEV)
    vel = torch.tensor(p.velocities, device=DEV)
    m = torch.tensor(p.m, device=DEV)
    disk2 = torch.tensor(p.group_id == 1, device=DEV)
    return pos, vel, m, disk2


def test_gradient_vs_torch_fp64_autograd():
    pos, vel, m, disk2 = _setup()
    steps, dt, eps = 50, 0.005, 0.05
    params = gx.PhysicsParams(1.0, eps)
    truth = torch.tensor([0.05, -0.03, 0.02, 0.01, 0.005, -0.01], dtype=torch.float64, device=DEV)
    with torch.no_grad():
        x0t, v0t = adjoint.encounter_initial_state(pos, vel, disk2, truth)
        target, _ = torch_leapfrog(x0t, v0t, m, steps, dt, eps)
    # engine: adjoint kernel + checkpointed leapfrog
    orbit = torch.zeros(6, dtype=torch.float64, device=DEV, requires_grad=True)
    x0 = pos.clone().requires_grad_(True)
    xs, vs = adjoint.encounter_initial_state(x0, vel, disk2, orbit)
    xT, _ = adjoint.leapfrog(xs, vs, m, steps, dt, params, checkpoint_every=10)
    loss = ((xT - target) ** 2).sum(1).mean()
    g_orbit, g_x0 = torch.autograd.grad(loss, [orbit, x0])
    # reference: plain FP64 torch autograd
    orbit_r = torch.zeros(6, dtype=torch.float64, device=DEV, requires_grad=True)
    x0_r = pos.clone().requires_grad_(True)
    xs_r, vs_r = adjoint.encounter_initial_state(x0_r, vel, disk2, orbit_r)
    xT_r, _ = torch_leapfrog(xs_r, vs_r, m, steps, dt, eps)
    loss_r = ((xT_r - target) ** 2).sum(1).mean()
    go_r, gx_r = torch.autograd.grad(loss_r, [orbit_r, x0_r])
    assert abs(float(loss) - float(loss_r)) <= 1e-12 * abs(float(loss_r))
    assert torch.max(torch.abs(g_orbit - go_r) / torch.abs(go_r).max()) <= 1e-9
    assert torch.max(torch.abs(g_x0 - gx_r)) / torch.abs(gx_r).max() <= 1e-9


def test_gradient_vs_finite_differences():
    pos, vel, m, disk2 = _setup()
    steps, dt, eps = 50, 0.005, 0.05
    params = gx.PhysicsParams(1.0, eps)
    truth = torch.tensor([0.05, -0.03, 0.02, 0.01, 0.005, -0.01], dtype=torch.float64, device=DEV)
    with torch.no_grad():
        x0t, v0t = adjoint.encounter_initial_state(pos, vel, disk2, truth)
        target, _ = adjoint.leapfrog(x0t, v0t, m, steps, dt, params)
    orbit = torch.zeros(6, dtype=torch.float64, device=DEV, requires_grad=True)
    loss = adjoint.orbit_loss(orbit, pos, vel, m, disk2, target, steps, dt, params, checkpoint_every=10)
    (g,) = torch.autograd.grad(loss, [orbit])
    h = 1e-6
    for k in range(6):
        e = torch.zeros(6, dtype=torch.float64, device=DEV)
        e[k] = h
        with torch.no_grad():
            lp = adjoint.orbit_loss(orbit + e, pos, vel, m, disk2, target, steps, dt, params)
            lm = adjoint.orbit_loss(orbit - e, pos, vel, m, disk2, target, steps, dt, params)
        fd = float(lp - lm) / (2 * h)
        assert abs(fd - float(g[k])) <= 1e-5 * max(abs(fd), 1e-8), (k, fd, float(g[k]))


def test_mixed_gradient_vs_fp64_finite_differences():
    """How far the mixed-precision gradient (FP32 pair arithmetic in the forward steps and in
    the adjoint kernel) sits from the true gradient: FP64 central differences of the FP64
    loss, N=512, 50 steps.  (Differences of the mixed loss itself would only measure its
    FP32 rounding noise divided by h.)"""
    pos, vel, m, disk2 = _setup()
    steps, dt, eps = 50, 0.005, 0.05
    params = gx.PhysicsParams(1.0, eps)
    truth = torch.tensor([0.05, -0.03, 0.02, 0.01, 0.005, -0.01], dtype=torch.float64, device=DEV)
    with torch.no_grad():
        x0t, v0t = adjoint.encounter_initial_state(pos, vel, disk2, truth)
        target, _ = adjoint.leapfrog(x0t, v0t, m, steps, dt, params)
    orbit = torch.zeros(6, dtype=torch.float64, device=DEV, requires_grad=True)
    loss = adjoint.orbit_loss(orbit, pos, vel, m, disk2, target, steps, dt, params, checkpoint_every=10,
                              precision=MIX)
    (g,) = torch.autograd.grad(loss, [orbit])
    h = 1e-6
    fd = np.zeros(6)
    for k in range(6):
        e = torch.zeros(6, dtype=torch.float64, device=DEV)
        e[k] = h
        with torch.no_grad():
            lp = adjoint.orbit_loss(orbit + e, pos, vel, m, disk2, target, steps, dt, params)
            lm = adjoint.orbit_loss(orbit - e, pos, vel, m, disk2, target, steps, dt, params)
        fd[k] = float(lp - lm) / (2 * h)
    err = np.abs(g.cpu().numpy() - fd) / np.abs(fd).max()
    print(f"mixed orbit gradient vs FP64 central differences: max {err.max():.3e} (relative to max |g|)")
    assert err.max() <= MIXED_ORBIT_GRAD_TOL, (err, fd)


def test_mass_gradient_vs_torch():
    pos, vel, m, disk2 = _setup(256, 9)
    steps, dt, eps = 20, 0.005, 0.05
    mm = m.clone().requires_grad_(True)
    xT, vT = adjoint.leapfrog(pos, vel, mm, steps, dt, gx.PhysicsParams(1.0, eps))
    (gm,) = torch.autograd.grad((xT ** 2).sum() + (vT ** 3).sum(), [mm])
    mr = m.clone().requires_grad_(True)
    xr, vr = torch_leapfrog(pos, vel, mr, steps, dt, eps)
    (gmr,) = torch.autograd.grad((xr ** 2).sum() + (vr ** 3).sum(), [mr])
    assert torch.max(torch.abs(gm - gmr)) / torch.abs(gmr).max() <= 1e-9


def test_orbit_fit_reduces_loss():
    pos, vel, m, disk2 = _setup(1024, 11)
    steps, dt = 100, 0.005
    params = gx.PhysicsParams(1.0, 0.05)
    truth = torch.tensor([0.04, -0.02, 0.03, 0.02, -0.01, 0.01], dtype=torch.float64, device=DEV)
    with torch.no_grad():
        x0t, v0t = adjoint.encounter_initial_state(pos, vel, disk2, truth)
        target, _ = adjoint.leapfrog(x0t, v0t, m, steps, dt, params)
    orbit, hist = adjoint.fit_orbit(pos, vel, m, disk2, target, steps, dt, params, iters=60, lr=0.005,
                                    checkpoint_every=25, precision=MIX)
    assert hist[-1] < hist[0] / 20.0, hist

"""Differentiable leapfrog over the engine's kernels (PyTorch autograd entry).

No reference counterpart: the reference has no gradients.  ``LeapfrogFunction`` runs
n KDK steps (kick dt/2, drift dt, force, kick dt/2; the first kick reuses a(x0)) with the
engine's direct-force kernel on CUDA tensors, keeps (x, v, a) every ``checkpoint_every``
steps, and in backward recomputes each segment forward, then walks it in reverse with the
hand-written adjoint kernel (gx_direct_vjp):

    xb <- dL/dx_T;  vb <- dL/dv_T;  xb += J_T^T (h vb)                 (h = dt/2)
    for k = T-1 .. 0:
        vb <- vb + dt xb                        (cotangent of v_{k+1/2})
        lam <- (2h if k >= 1 else h) vb         (closing kick of step k-1 + opening kick of k)
        xb <- xb + J_k^T lam ;  mb <- mb + (dA/dm)^T lam
    returns xb = dL/dx_0, vb = dL/dv_0, mb = dL/dm

where J_k = dA/dx at x_k.  One VJP per state, T + 1 in all.
"""
from __future__ import annotations

import numpy as np
import torch

from . import _ffi
from ._ffi import PRECISION_F64, PRECISION_MIXED
from .engine import PhysicsParams


def _stream() -> int:
    return torch.cuda.current_stream().cuda_stream


def _soa(t: torch.Tensor) -> torch.Tensor:
    """(n, 3) -> contiguous (3, n) float64 on the same device."""
    return t.detach().to(torch.float64).t().contiguous()


def _rows(a: torch.Tensor):
    return a[0].data_ptr(), a[1].data_ptr(), a[2].data_ptr()


def accelerations(X: torch.Tensor, m: torch.Tensor, params: PhysicsParams, precision=PRECISION_F64) -> torch.Tensor:
    """Direct-sum accelerations of SoA positions X (3, n) -> (3, n)."""
    A = torch.empty_like(X)
    n = X.shape[1]
    _ffi.call("gx_direct_accel", n, *_rows(X), m.data_ptr(), params.ffi(), _ffi.precision_code(precision), *_rows(A),
              _stream())
    return A


def direct_vjp(X: torch.Tensor, m: torch.Tensor, lam: torch.Tensor, params: PhysicsParams,
               precision=PRECISION_F64):
    """(dL/dX, dL/dm) for L = sum lam . a(X, m); X, lam are SoA (3, n) CUDA float64."""
    GX = torch.empty_like(X)
    GM = torch.empty_like(m)
    n = X.shape[1]
    _ffi.call("gx_direct_vjp", n, *_rows(X), m.data_ptr(), *_rows(lam), params.ffi(), _ffi.precision_code(precision),
              *_rows(GX), GM.data_ptr(), _stream())
    return GX, GM


def _step(X, V, A, m, dt, params, precision):
    n = X.shape[1]
    _ffi.call("gx_leapfrog_step", n, *_rows(X), *_rows(V), *_rows(A), m.data_ptr(), float(dt), params.ffi(),
              _ffi.precision_code(precision), _stream())


class LeapfrogFunction(torch.autograd.Function):
    """(x0 (n,3), v0 (n,3), m (n,)) -> (x_T, v_T) after n_steps KDK steps."""

    @staticmethod
    def forward(ctx, x0, v0, m, n_steps: int, dt: float, G: float, softening: float, checkpoint_every: int,
                precision: int):
        params = PhysicsParams(G, softening)
        X, V = _soa(x0), _soa(v0)
        mm = m.detach().to(torch.float64).contiguous()
        A = accelerations(X, mm, params, precision)
        K = max(1, int(checkpoint_every))
        ckpts = [(X.clone(), V.clone(), A.clone())]
        for s in range(n_steps):
            _step(X, V, A, mm, dt, params, precision)
            if (s + 1) % K == 0 and s + 1 < n_steps:
                ckpts.append((X.clone(), V.clone(), A.clone()))
        ctx.save_for_backward(mm)
        ctx.ckpts = ckpts
        ctx.cfg = (n_steps, dt, params, K, precision)
        return X.t().contiguous(), V.t().contiguous()

    @staticmethod
    def backward(ctx, gx, gv):
        (mm,) = ctx.saved_tensors
        n_steps, dt, params, K, precision = ctx.cfg
        vjp_prec = PRECISION_MIXED if precision == PRECISION_MIXED else PRECISION_F64
        h = 0.5 * dt
        n = mm.shape[0]
        xb = _soa(gx) if gx is not None else torch.zeros(3, n, dtype=torch.float64, device=mm.device)
        vb = _soa(gv) if gv is not None else torch.zeros(3, n, dtype=torch.float64, device=mm.device)
        mb = torch.zeros_like(mm)
        n_seg = len(ctx.ckpts)
        for seg in reversed(range(n_seg)):
            s0 = seg * K
            s1 = min(s0 + K, n_steps)
            X, V, A = (t.clone() for t in ctx.ckpts[seg])
            states = [X.clone()]
            for _ in range(s0, s1):
                _step(X, V, A, mm, dt, params, precision)
                states.append(X.clone())
            if seg == n_seg - 1:
                g, gm = direct_vjp(states[-1], mm, h * vb, params, vjp_prec)
                xb += g
                mb += gm
            for k in range(s1 - 1, s0 - 1, -1):
                vb = vb + dt * xb
                lam = (2.0 * h if k >= 1 else h) * vb
                g, gm = direct_vjp(states[k - s0], mm, lam, params, vjp_prec)
                xb = xb + g
                mb = mb + gm
        ctx.ckpts = None
        return xb.t().contiguous(), vb.t().contiguous(), mb, None, None, None, None, None, None


def leapfrog(x0, v0, m, n_steps: int, dt: float, params: PhysicsParams, checkpoint_every: int = 50,
             precision=PRECISION_F64):
    return LeapfrogFunction.apply(x0, v0, m, int(n_steps), float(dt), params.gravitational_constant,
                                  params.softening, int(checkpoint_every), _ffi.precision_code(precision))


# ---- encounter orbit fit -----------------------------------------------------------------
def encounter_initial_state(base_pos: torch.Tensor, base_vel: torch.Tensor, disk2: torch.Tensor,
                            orbit: torch.Tensor):
    """Shifts disk 2 (boolean mask) by the 6 orbit parameters (dx, dy, dz, dvx, dvy, dvz)."""
    sel = disk2.to(base_pos.dtype).unsqueeze(1)
    return base_pos + sel * orbit[:3], base_vel + sel * orbit[3:]


def orbit_loss(orbit, base_pos, base_vel, m, disk2, target, n_steps, dt, params, checkpoint_every=50,
               precision=PRECISION_F64):
    x0, v0 = encounter_initial_state(base_pos, base_vel, disk2, orbit)
    xT, _ = leapfrog(x0, v0, m, n_steps, dt, params, checkpoint_every, precision)
    return ((xT - target) ** 2).sum(1).mean()


def fit_orbit(base_pos, base_vel, m, disk2, target, n_steps, dt, params, init=None, iters: int = 40,
              lr: float = 0.05, checkpoint_every: int = 50, precision=PRECISION_F64):
    """Recovers the 6 orbit parameters that produced `target` (Adam on the adjoint gradient).
    Returns (orbit, loss history)."""
    orbit = (torch.zeros(6, dtype=torch.float64, device=base_pos.device) if init is None
             else init.detach().clone().to(torch.float64)).requires_grad_(True)
    opt = torch.optim.Adam([orbit], lr=lr)
    hist = []
    for _ in range(iters):
        opt.zero_grad()
        loss = orbit_loss(orbit, base_pos, base_vel, m, disk2, target, n_steps, dt, params, checkpoint_every,
                          precision)
        loss.backward()
        opt.step()
        hist.append(float(loss))
    return orbit.detach(), np.array(hist)

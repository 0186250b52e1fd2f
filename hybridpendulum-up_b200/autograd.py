"""torch.autograd wrapper over forward-Euler propagation and its hand-written
reverse pass (``hp_pendulum_adjoint``).

Coefficient arrays are complex128 tensors whose memory is the reference's
column-major layout F(2lmax+1, 2lmax+1, lmax+1, 2Bx, ...): as torch tensors
they carry the reversed shape (..., 2Bx, lmax+1, 2lmax+1, 2lmax+1) and are
C-contiguous (``to_torch`` / ``from_torch`` convert numpy arrays).  Complex
gradients follow torch's convention dL = Re sum conj(grad) dF; for real
densities they are taken on the real-density subspace.

The model parameters are differentiable: damping b, the gyroscopic
coefficients gyro, the noise matrix G = H H^T / 2 and per-component gravity
scales gscale (MR_i -> gscale_i MR_i; a diagonal inertia J rescales MR_i by
J_ref_i / J_i).  ``pendulum_params`` maps (b, J, H) onto them with torch
operations, so gradients with respect to b, J and H follow by the chain rule.
"""
from __future__ import annotations

import numpy as np
import torch

from . import HP_REAL, Plan, State, fftSO3R_mex

__all__ = ['to_torch', 'from_torch', 'propagate', 'pendulum_params', 'measurement_weights']


def to_torch(F, device=None) -> torch.Tensor:
    """numpy array in the reference layout -> C-contiguous tensor of reversed shape."""
    t = torch.from_numpy(np.ascontiguousarray(np.asarray(F).T))
    return t.to(device) if device is not None else t


def from_torch(t: torch.Tensor) -> np.ndarray:
    return t.detach().cpu().numpy().T


def _set_model(plan: Plan, L, MR, b, gyro, G, gscale):
    nd = plan.ndim
    MRs = np.array(MR, dtype=np.complex128, copy=True)
    gs = gscale.detach().cpu().numpy()
    for i in range(nd):
        MRs[..., i] *= gs[i]
    gy = np.zeros(3)
    if nd == 3:
        gy[:] = gyro.detach().cpu().numpy()
    plan.set_model(L, b.detach().cpu().numpy(), G.detach().cpu().numpy(), MRs, tuple(gy))


class _Trajectory(torch.autograd.Function):
    @staticmethod
    def forward(ctx, F0, b, gyro, G, gscale, plan, MR, L, dt, nsteps, ckpt):
        _set_model(plan, L, MR, b, gyro, G, gscale)
        F0c = F0.detach().contiguous()
        st = State(plan)
        st.load(F0c)
        st.step(dt, 'euler', nsteps)
        out = torch.empty_like(F0c)
        st.store(out)
        ctx.save_for_backward(F0c, b, gyro, G, gscale)
        ctx.cfg = (plan, MR, L, dt, nsteps, ckpt)
        return out

    @staticmethod
    def backward(ctx, gF):
        F0, b, gyro, G, gscale = ctx.saved_tensors
        plan, MR, L, dt, nsteps, ckpt = ctx.cfg
        _set_model(plan, L, MR, b, gyro, G, gscale)
        lamT = gF.detach().to(dtype=torch.complex128, device=F0.device).contiguous()
        lam0, g = plan.adjoint(F0, lamT, nsteps, dt, ckpt)
        lam0 = lam0.reshape(F0.shape)
        nd = plan.ndim
        kw = dict(dtype=torch.float64, device=b.device)
        return (lam0,
                torch.tensor(g['b'][:nd], **kw),
                torch.tensor(g['gyro'][:gyro.numel()], **kw),
                torch.tensor(g['G'][:nd, :nd], **kw),
                torch.tensor(g['gscale'][:nd], **kw),
                None, None, None, None, None, None)


def propagate(F0: torch.Tensor, b: torch.Tensor, gyro: torch.Tensor, G: torch.Tensor, gscale: torch.Tensor, *,
              plan: Plan, MR, L: float, dt: float, nsteps: int, checkpoint_every: int = 10) -> torch.Tensor:
    """F_T after ``nsteps`` forward-Euler steps of the pendulum derivative
    (pendulum.m:346-527) from F0, differentiable in F0, b, gyro, G and gscale.
    MR is the gravity transform at gscale = 1 (numpy, reference layout)."""
    if F0.dtype != torch.complex128:
        raise TypeError('F0 must be complex128')
    return _Trajectory.apply(F0, b, gyro, G, gscale, plan, MR, float(L), float(dt), int(nsteps),
                             int(checkpoint_every))


def pendulum_params(b: torch.Tensor, J: torch.Tensor, H: torch.Tensor, J_ref) -> tuple:
    """(b, gyro, G, gscale) of a pendulum with diagonal inertia J (3,), noise
    H and the gravity transform MR computed at inertia J_ref:
    gyro = ((J2-J3)/J1, (J3-J1)/J2, (J1-J2)/J3) (pendulum.m:145-158),
    G = H H^T / 2 (pendulum.m:202-208), gscale_i = J_ref_i / J_i
    (MR = fftSO3(J^-1 (-m g rho x R^T e3)), pendulum.m:166-193)."""
    J_ref = torch.as_tensor(np.asarray(J_ref, float), dtype=torch.float64, device=J.device)
    gyro = torch.stack([(J[1] - J[2]) / J[0], (J[2] - J[0]) / J[1], (J[0] - J[1]) / J[2]])
    G = 0.5 * H @ H.T
    nd = H.shape[0]
    gscale = J_ref[:nd] / J[:nd]
    return b, gyro, G, gscale


def measurement_weights(plan: Plan, p_meas: np.ndarray, L: float) -> torch.Tensor:
    """Pw with Re sum conj(Pw) F = sum_grid w_beta (L/2Bx)^n p_meas f, f the
    real density of F on the grid (the quadrature of fftSO3R.m:62-66 times the
    omega cell volume).  By the backward transform's definition this is
    (2l+1) / nx * (L/2Bx)^n * fftSO3R(p_meas)."""
    P = fftSO3R_mex('forward', np.asarray(p_meas, float))
    lmax = plan.lmax
    nx = plan.N ** plan.ndim
    w = (2 * np.arange(lmax + 1) + 1).reshape(1, 1, lmax + 1, *([1] * plan.ndim)) / nx
    w = w * (L / plan.N) ** plan.ndim
    return to_torch(P * w)

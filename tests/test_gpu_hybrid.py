"""Hybrid step of pendulum_reduced_hybrid.m:224-234 on the resident state
(density-gravity propagation, backward transform, in-place collision update,
forward transform) against the oracle composition of the same four steps.

The oracle uses the collision tables the library built (their own parity is in
test_gpu_collision), so this test checks the composition and the in-place
update.  Tolerances: FP64 <= 1e-10 relative L2 on the increment F - F0;
mixed <= 1e-6 relative L2 on F and f themselves, because in mixed plans every
hybrid step re-projects the whole density through FP32 transforms (the
transform bar of test_gpu_parity), not only the increment.
"""
import math

import numpy as np
import pytest

from oracle import collision as co
from oracle import pendulum as pd
from oracle import so3

pytestmark = pytest.mark.gpu

PRM = dict(d=0.12, h=0.2, r=0.025, theta_t=5 * math.pi / 180, lambda_max=100.0, epsilon=0.8)


def rel(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return float(np.linalg.norm((a - b).ravel()) / np.linalg.norm(b.ravel()))


def to_ixiR(f):
    return np.transpose(f, (4, 3, 2, 1, 0)).reshape(f.shape[3] * f.shape[4], -1)


def from_ixiR(fl, shape):
    n = shape[0]
    return np.transpose(fl.reshape(shape[4], shape[3], n, n, n), (4, 3, 2, 1, 0))


def oracle_hybrid(F, f, P, t, dt, method, nsteps):
    for _ in range(nsteps):
        calls = []

        def deriv(Fx):
            fx = f if not calls else None
            calls.append(1)
            return pd.derivative_den(Fx, fx, P)
        F = pd.integrate(F, deriv, dt, method)
        fg = np.real(so3.ifftSO3R_backward(F, real=True))
        fl = to_ixiR(fg)
        fl = fl + dt * co.propagate_noise(fl, t['lambda_'], t['indR'], t['fcL'], t['fcL_indx'])
        f = from_ixiR(fl, fg.shape)
        F = so3.fftSO3R_forward(f)
    return F, f


@pytest.mark.parametrize('B,Bx', [(4, 3), (6, 4)])
@pytest.mark.parametrize('precision', [0, 1])
@pytest.mark.parametrize('method', ['euler', 'RK4'])
def test_hybrid_steps_vs_oracle(hp, B, Bx, precision, method):
    import torch
    P = pd.pendulum_reduced(B, Bx, L=3.4)
    f0, _ = pd.seeded_density(B, Bx, 2, P.L, seed=B + Bx, sigma=0.5)
    F0 = so3.fftSO3R_forward(f0)
    Gd = 0.0025 * np.eye(2)
    dt = 0.01
    plan = hp.Plan(B, Bx, 2, precision, hp.HP_REAL)
    plan.set_den_model(P.L, P.b, P.G, P.mR)
    coll = hp.Collision(plan, L=P.L, Gd=Gd, nD=10, **PRM)
    assert coll.numR > 0
    t = coll.tables()
    Fref, fref = oracle_hybrid(F0, so3.ifftSO3R_backward(F0, real=True), P, t, dt, method, 2)

    st = hp.State(plan)
    st.load(F0)
    st.hybrid_step(coll, dt, method, 2)
    F = st.store()
    if precision == 0:
        tol = 1e-10
        assert rel(F - F0, Fref - F0) < tol
    else:
        tol = 1e-6
        assert rel(F, Fref) < tol
    dtype = torch.float64 if precision == 0 else torch.float32
    fd = torch.zeros(tuple(reversed(f0.shape)), dtype=dtype, device='cuda')
    st.density_into(fd.data_ptr())
    torch.cuda.synchronize()
    fg = np.transpose(fd.cpu().double().numpy(), (4, 3, 2, 1, 0))
    assert rel(fg, fref) < tol


def test_hybrid_needs_a_model(hp):
    B, Bx = 3, 2
    P = pd.pendulum_reduced(B, Bx, L=3.4)
    plan = hp.Plan(B, Bx, 2, 0, hp.HP_REAL)
    coll = hp.Collision(plan, L=P.L, Gd=0.0025 * np.eye(2), nD=4, **PRM)
    st = hp.State(plan)
    with pytest.raises(hp.HPError):
        st.hybrid_step(coll, 0.01, 'euler', 1)


def oracle_hybrid_cg(F, P, t, dt, method, nsteps):
    """Hybrid loop with the coefficient-gravity derivative (any ndim)."""
    for _ in range(nsteps):
        F = pd.integrate(F, lambda Fx: pd.derivative_fast(Fx, P), dt, method)
        fg = np.real(so3.ifftSO3R_backward(F, real=True))
        nR = fg.shape[0] * fg.shape[1] * fg.shape[2]
        fl = fg.T.reshape(-1, nR)
        fl = fl + dt * co.propagate_noise(fl, t['lambda_'], t['indR'], t['fcL'], t['fcL_indx'])
        F = so3.fftSO3R_forward(fl.reshape(fg.T.shape).T)
    return F


@pytest.mark.parametrize('ndim,B,Bx', [(2, 4, 3), (3, 4, 3)])
@pytest.mark.parametrize('precision', [0, 1])
def test_hybrid_coefficient_model(hp, ndim, B, Bx, precision):
    """Hybrid steps with a coefficient-gravity model: the reduced pendulum with
    Clebsch-Gordan gravity, and the 3-D pendulum with the 3-D collision operator."""
    P = pd.pendulum_3d(B, Bx, L=4.0) if ndim == 3 else pd.pendulum_reduced(B, Bx, L=3.4)
    f0, _ = pd.seeded_density(B, Bx, ndim, P.L, seed=B + ndim, sigma=0.5)
    F0 = so3.fftSO3R_forward(f0)
    Gd = (0.0025 if ndim == 2 else 0.04) * np.eye(ndim)
    dt = 0.005
    plan = hp.Plan(B, Bx, ndim, precision, hp.HP_REAL)
    gyro = (0.0, 0.0, 0.0)
    if ndim == 3:
        J = np.diag(P.params['J'])
        gyro = ((J[1] - J[2]) / J[0], (J[2] - J[0]) / J[1], (J[0] - J[1]) / J[2])
    plan.set_model(P.L, P.b, P.G, P.MR, gyro)
    coll = hp.Collision(plan, L=P.L, Gd=Gd, nD=8, **PRM)
    assert coll.numR > 0
    Fref = oracle_hybrid_cg(F0, P, coll.tables(), dt, 'RK2', 2)
    st = hp.State(plan)
    st.load(F0)
    st.hybrid_step(coll, dt, 'RK2', 2)
    F = st.store()
    if precision == 0:
        assert rel(F - F0, Fref - F0) < 1e-10
    else:
        assert rel(F, Fref) < 1e-6

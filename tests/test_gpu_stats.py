"""Moments of get_stat from the GPU coefficients (hp_moments, hp_state_moments)
against the oracle's grid sums over f; FP64 agreement 1e-11 relative."""
import importlib
import math

import numpy as np
import pytest

from oracle import collision as co
from oracle import pendulum as pd
from oracle import so3
from oracle import stats as ost

pytestmark = [pytest.mark.gpu, pytest.mark.filterwarnings('ignore::scipy.integrate.IntegrationWarning')]


def close(a, b, tol=1e-11):
    a, b = np.asarray(a), np.asarray(b)
    return np.abs(a - b).max() <= tol * max(1.0, np.abs(b).max())


def model_plan(hp, B, Bx, nd, precision=0):
    P = pd.pendulum_3d(B, Bx, L=4.0) if nd == 3 else pd.pendulum_reduced(B, Bx, L=4.0)
    plan = hp.Plan(B, Bx, nd, precision, hp.HP_REAL)
    plan.set_model(P.L, P.b, P.G, P.MR)
    return P, plan


@pytest.mark.parametrize('B,Bx,nd', [(3, 2, 3), (5, 3, 2), (6, 4, 3), (15, 4, 3)])
def test_moments_vs_grid(hp, B, Bx, nd):
    P, plan = model_plan(hp, B, Bx, nd)
    f, _ = pd.seeded_density(B, Bx, nd, P.L, seed=B + Bx)
    F = so3.fftSO3R_forward(f)
    ref = ost.raw_moments_grid(f, P.L)
    out = plan.moments(F, want_fx=True)
    for k in ref:
        assert close(out[k], ref[k]), k
    fx = np.einsum('b,abc...->...', so3.quad_weights(B), f)
    assert close(out['fx'], fx)


def test_get_stat_vs_oracle(hp):
    pst = importlib.import_module('hybridpendulum-up_b200.stats')
    B, Bx, nd = 6, 4, 3
    P, plan = model_plan(hp, B, Bx, nd)
    f, _ = pd.seeded_density(B, Bx, nd, P.L, seed=7)
    ref = ost.get_stat_grid(f, P.L)
    out = pst.get_stat(plan.moments(so3.fftSO3R_forward(f), want_fx=True))
    for k in ('ER', 'Ex', 'Varx', 'EvR', 'ExvR', 'EvRvR', 'U', 'S', 'V', 'P', 'Miu', 'Sigma', 'fx'):
        assert close(out[k], ref[k], 1e-8), k


def test_state_moments_after_hybrid_steps(hp):
    """After hybrid steps the statistics are those of the post-collision grid
    density (pendulum_reduced_hybrid.m:232-238)."""
    B, Bx, dt = 4, 3, 0.01
    prm = dict(d=0.12, h=0.2, r=0.025, theta_t=5 * math.pi / 180, lambda_max=100.0, epsilon=0.8)
    Pm = pd.pendulum_reduced(B, Bx, L=3.4)
    plan = hp.Plan(B, Bx, 2, 0, hp.HP_REAL)
    plan.set_den_model(Pm.L, Pm.b, Pm.G, Pm.mR)
    coll = hp.Collision(plan, L=Pm.L, Gd=0.0025 * np.eye(2), nD=10, **prm)
    t = coll.tables()
    f0, _ = pd.seeded_density(B, Bx, 2, Pm.L, seed=5)
    F0 = so3.fftSO3R_forward(f0)
    st = hp.State(plan)
    st.load(F0)
    st.hybrid_step(coll, dt, 'euler', 1)
    # oracle: one step of the same composition
    F1 = pd.integrate(F0, lambda Fx: pd.derivative_den(Fx, so3.ifftSO3R_backward(F0, real=True)
                                                       if Fx is F0 else None, Pm), dt, 'euler')
    fg = np.real(so3.ifftSO3R_backward(F1, real=True))
    fl = np.transpose(fg, (4, 3, 2, 1, 0)).reshape(fg.shape[3] * fg.shape[4], -1)
    fl = fl + dt * co.propagate_noise(fl, t['lambda_'], t['indR'], t['fcL'], t['fcL_indx'])
    n = fg.shape[0]
    f1 = np.transpose(fl.reshape(fg.shape[4], fg.shape[3], n, n, n), (4, 3, 2, 1, 0))
    ref = ost.raw_moments_grid(f1, Pm.L)
    out = st.moments()
    for k in ref:
        assert close(out[k], ref[k], 1e-9), k

"""Gyro-bias attitude model (gyro_bias.m:226-300, MEX gyrobias_propagate) on the
GPU against the FP64 oracle.  Tolerances as in test_gpu_parity: FP64 <= 1e-10,
mixed <= 1e-6 relative L2 on the step increment."""
import numpy as np
import pytest

from oracle import gyro_bias as gb
from oracle import pendulum as pd
from oracle import so3

pytestmark = pytest.mark.gpu

TOL64 = 1e-10
TOLMIX = 1e-6


def rel(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return float(np.linalg.norm((a - b).ravel()) / np.linalg.norm(b.ravel()))


def setup(B, Bx, L, seed):
    rng = np.random.default_rng(seed)
    f, _ = pd.seeded_density(B, Bx, 3, L, seed=seed, sigma=0.3 * L / 2)
    F = so3.fftSO3R_forward(f)
    A = rng.standard_normal((3, 3))
    G1 = 0.05 * (A @ A.T)              # correlated attitude noise
    A = rng.standard_normal((3, 3))
    G2 = 0.01 * (A @ A.T)
    return F, G1, G2


@pytest.mark.parametrize('B,Bx', [(3, 2), (5, 4), (8, 6), (6, 15)])
@pytest.mark.parametrize('precision', [0, 1])
def test_gyrobias_step_vs_oracle(hp, B, Bx, precision):
    L = 2.0
    F, G1, G2 = setup(B, Bx, L, seed=B * 7 + Bx)
    dt = 0.01
    ref = F + dt * gb.derivative_fast(F, L, G1, G2)
    plan = hp.Plan(B, Bx, 3, precision, hp.HP_REAL)
    plan.set_gyro_bias_model(L, G1, G2)
    out = plan.gyrobias_propagate(F, dt)
    assert rel(out - F, ref - F) < (TOL64 if precision == 0 else TOLMIX)


@pytest.mark.parametrize('method', ['midpoint', 'RK2', 'RK4'])
def test_gyrobias_higher_order_and_period(hp, method):
    B, Bx, L = 4, 3, 3.0
    F, G1, G2 = setup(B, Bx, L, seed=11)
    ref = pd.integrate(F, lambda Fx: gb.derivative_fast(Fx, L, G1, G2), 0.02, method)
    plan = hp.Plan(B, Bx, 3, 0, hp.HP_REAL)
    plan.set_gyro_bias_model(L, G1, G2)
    out = plan.propagate(F, 0.02, method)
    assert rel(out - F, ref - F) < TOL64


def test_reference_named_entry_vs_literal(hp):
    """gyrobias_propagate(F,X,dt,u,G1,G2) against the literal restatement."""
    B, Bx = 3, 2
    F, G1, G2 = setup(B, Bx, 2.0, seed=4)
    X = pd.make_X(gb.bias_grid(Bx, 2.0))
    ref = gb.propagate(F, X, 0.01, G1, G2)
    out = hp.gyrobias_propagate(F, X, 0.01, hp.getu(B - 1), G1, G2)
    assert rel(out - F, ref - F) < TOL64
    out32 = hp.gyrobias_propagate32(F, X, 0.01, None, G1, G2)
    assert rel(out32 - F, ref - F) < TOLMIX


def test_state_steps_and_allocation_free_derivative(hp):
    B, Bx, L = 5, 4, 2.0
    F, G1, G2 = setup(B, Bx, L, seed=8)
    plan = hp.Plan(B, Bx, 3, 0, hp.HP_REAL)
    plan.set_gyro_bias_model(L, G1, G2)
    ref = F
    for _ in range(3):
        ref = ref + 0.01 * gb.derivative_fast(ref, L, G1, G2)
    st = hp.State(plan)
    st.load(F)
    st.step(0.01, 'euler', 3)
    assert rel(st.store() - F, ref - F) < TOL64
    d = plan.derivative(F)
    assert rel(d, gb.derivative_fast(F, L, G1, G2)) < TOL64


def test_gyro_bias_model_errors(hp):
    B, Bx = 3, 2
    F, G1, G2 = setup(B, Bx, 2.0, seed=1)
    plan2 = hp.Plan(B, Bx, 2, 0, hp.HP_REAL)
    with pytest.raises(hp.HPError):
        plan2.set_gyro_bias_model(2.0, G1, G2)
    plan = hp.Plan(B, Bx, 3, 0, hp.HP_REAL)
    with pytest.raises(hp.HPError):              # no model yet
        plan.gyrobias_propagate(F, 0.01)
    bad = G1.copy()
    bad[0, 1] = np.inf
    with pytest.raises(hp.HPError):
        plan.set_gyro_bias_model(2.0, bad, G2)
    plan.set_gyro_bias_model(2.0, G1, G2)
    with pytest.raises(hp.HPError):              # the adjoint covers the pendulum models
        plan.derivative_adjoint(F)
    P = pd.pendulum_3d(B, Bx)
    plan.set_model(P.L, P.b, P.G, P.MR)          # a pendulum model replaces it
    with pytest.raises(hp.HPError):
        plan.gyrobias_propagate(F, 0.01)

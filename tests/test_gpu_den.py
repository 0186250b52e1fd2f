"""Density-gravity model of the reduced pendulum (pendulum_reduced_den.m,
propagation/mex/sources/pendulum_propagate_reduced_den) on the GPU against the
FP64 oracle ``derivative_den``.

Tolerances as in test_gpu_parity: FP64 <= 1e-10, mixed <= 1e-6 relative L2 on
the step increment.
"""
import numpy as np
import pytest

from oracle import pendulum as pd
from oracle import so3

pytestmark = pytest.mark.gpu

TOL64 = 1e-10
TOLMIX = 1e-6


def rel(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return float(np.linalg.norm((a - b).ravel()) / np.linalg.norm(b.ravel()))


def setup(B, Bx, seed):
    P = pd.pendulum_reduced(B, Bx)
    f, _ = pd.seeded_density(B, Bx, 2, P.L, seed=seed, sigma=0.4)
    F = so3.fftSO3R_forward(f)
    return P, f, F


def oracle_step(F, f, P, dt, method):
    calls = []

    def deriv(Fx):
        fx = f if not calls else None          # the first stage uses the given f
        calls.append(1)
        return pd.derivative_den(Fx, fx, P)
    return pd.integrate(F, deriv, dt, method)


@pytest.mark.parametrize('B,Bx', [(3, 2), (5, 4), (8, 6)])
@pytest.mark.parametrize('precision', [0, 1])
@pytest.mark.parametrize('method', ['euler', 'midpoint', 'RK2', 'RK4'])
def test_propagate_den_vs_oracle(hp, B, Bx, precision, method):
    P, f, F = setup(B, Bx, seed=3 * B + Bx)
    # a grid density that differs from backward(F): the first stage must use it
    f_given = f * (1.0 + 0.05 * np.cos(np.arange(f.size).reshape(f.shape, order='F') * 0.37))
    dt = 0.01
    ref = oracle_step(F, f_given, P, dt, method)
    plan = hp.Plan(B, Bx, 2, precision, hp.HP_REAL)
    plan.set_den_model(P.L, P.b, P.G, P.mR)
    out = plan.propagate_den(F, f_given, dt, method)
    tol = TOL64 if precision == 0 else TOLMIX
    assert rel(out - F, ref - F) < tol


@pytest.mark.parametrize('precision', [0, 1])
def test_propagate_den_without_f(hp, precision):
    B, Bx = 6, 4
    P, f, F = setup(B, Bx, seed=11)
    ref = pd.integrate(F, lambda Fx: pd.derivative_den(Fx, None, P), 0.02, 'rk4')
    plan = hp.Plan(B, Bx, 2, precision, hp.HP_REAL)
    plan.set_den_model(P.L, P.b, P.G, P.mR)
    out = plan.propagate_den(F, None, 0.02, 'rk4')
    assert rel(out - F, ref - F) < (TOL64 if precision == 0 else TOLMIX)


def test_den_matches_coefficient_gravity(hp):
    """For f = backward(F) the grid gravity equals the Clebsch-Gordan gravity of
    the coefficient model (mR is of degree 1 and the quadrature is exact)."""
    B, Bx = 5, 4
    P, f, F = setup(B, Bx, seed=5)
    a = hp.Plan(B, Bx, 2, 0, hp.HP_REAL)
    a.set_den_model(P.L, P.b, P.G, P.mR)
    out_den = a.propagate_den(F, None, 0.01, 'euler')
    b = hp.Plan(B, Bx, 2, 0, hp.HP_REAL)
    b.set_model(P.L, P.b, P.G, P.MR)
    out_cg = b.propagate(F, 0.01, 'euler')
    assert rel(out_den - F, out_cg - F) < 1e-10


def test_reference_named_den_entry(hp):
    B, Bx = 4, 3
    P, f, F = setup(B, Bx, seed=2)
    ref = oracle_step(F, f, P, 0.01, 'euler')
    out = hp.pendulum_propagate_reduced_den(F, f, P.X, P.mR, P.b, P.G, 0.01, P.L, None, None, None, 'euler')
    assert rel(out - F, ref - F) < TOL64
    out32 = hp.pendulum_propagate_reduced_den32(F, f, P.X, P.mR, P.b, P.G, 0.01, P.L, None, None, None,
                                                'euler')
    assert rel(out32 - F, ref - F) < TOLMIX


def test_den_model_errors(hp):
    B, Bx = 3, 2
    P, f, F = setup(B, Bx, seed=1)
    plan3 = hp.Plan(B, Bx, 3, 0, hp.HP_REAL)
    with pytest.raises(hp.HPError):
        plan3.set_den_model(P.L, P.b, P.G, P.mR)
    plan = hp.Plan(B, Bx, 2, 0, hp.HP_REAL)
    with pytest.raises(hp.HPError):            # no density model yet
        plan.propagate_den(F, f, 0.01)
    bad = P.mR.copy()
    bad[0, 0, 0, 0] = np.nan
    with pytest.raises(hp.HPError):
        plan.set_den_model(P.L, P.b, P.G, bad)
    plan.set_den_model(P.L, P.b, P.G, P.mR)
    with pytest.raises(hp.HPError):
        plan.propagate_den(F, f[..., :2], 0.01)

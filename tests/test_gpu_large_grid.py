"""The reference's density-gravity and hybrid drivers run BR = 30, Bx = 30
(pendulum_reduced_den.m:64-65, pendulum_reduced_hybrid.m:58-59): bandlimit 30
and a 60 x 60 omega grid.  Parity with the oracle on those grids at small B
(FP64 <= 1e-10, mixed <= 1e-6 relative L2), and the B=24, B=30 transforms."""
import numpy as np
import pytest

from oracle import pendulum as pd
from oracle import so3

pytestmark = pytest.mark.gpu


def rel(a, b):
    return float(np.linalg.norm((np.asarray(a) - np.asarray(b)).ravel()) / np.linalg.norm(np.asarray(b).ravel()))


@pytest.mark.parametrize('Bx', [20, 24, 30])
@pytest.mark.parametrize('precision', [0, 1])
def test_reduced_step_large_omega_grid(hp, Bx, precision):
    B = 4
    P = pd.pendulum_reduced(B, Bx, L=3.4)
    f, _ = pd.seeded_density(B, Bx, 2, P.L, seed=Bx)
    F = so3.fftSO3R_forward(f)
    plan = hp.Plan(B, Bx, 2, precision, hp.HP_REAL)
    plan.set_model(P.L, P.b, P.G, P.MR)
    ref = pd.integrate(F, lambda x: pd.derivative_fast(x, P), 1e-3, 'rk4')
    out = plan.propagate(F, 1e-3, 'RK4')
    tol = 1e-10 if precision == 0 else 1e-6
    assert rel(out - F, ref - F) < tol
    assert rel(plan.backward(F), so3.ifftSO3R_backward(F, real=True)) < tol


@pytest.mark.parametrize('precision', [0, 1])
def test_den_large_omega_grid(hp, precision):
    B, Bx = 4, 30
    P = pd.pendulum_reduced(B, Bx, L=3.4)
    f, _ = pd.seeded_density(B, Bx, 2, P.L, seed=3)
    F = so3.fftSO3R_forward(f)
    ref = F + 1e-3 * pd.derivative_den(F, f, P)
    plan = hp.Plan(B, Bx, 2, precision, hp.HP_REAL)
    plan.set_den_model(P.L, P.b, P.G, P.mR)
    out = plan.propagate_den(F, f, 1e-3, 'euler')
    assert rel(out - F, ref - F) < (1e-10 if precision == 0 else 1e-6)


@pytest.mark.parametrize('B', [24, 30])
@pytest.mark.parametrize('precision', [0, 1])
def test_transforms_b24_b30(hp, B, precision):
    Bx = 2
    f, _ = pd.seeded_density(B, Bx, 2, 4.0, seed=B)
    plan = hp.Plan(B, Bx, 2, precision, hp.HP_REAL)
    F = plan.forward(f)
    tol = 1e-10 if precision == 0 else 1e-6
    Fref = so3.fftSO3R_forward(f)
    assert rel(F, Fref) < tol
    assert rel(plan.backward(F), so3.ifftSO3R_backward(Fref, real=True)) < tol

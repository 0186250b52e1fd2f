"""CUDA path vs the committed golden fixtures (tests/golden/make_golden.py:
outputs of the oracle's literal restatement of pendulum.m / fftSO3_prod.m)."""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

Z = os.path.join(os.path.dirname(__file__), 'golden', 'pendulum_small.npz')


def rel(a, b):
    return float(np.linalg.norm((np.asarray(a) - b).ravel()) / np.linalg.norm(b.ravel()))


@pytest.fixture(scope='module')
def z():
    return np.load(Z)


def test_golden_transforms(hp, z):
    plan = hp.Plan(3, 2, 3, hp.HP_FP64, hp.HP_REAL)
    assert rel(plan.forward(z['p3_f']), z['p3_F']) < 1e-12
    assert rel(plan.backward(z['p3_F']), z['p3_fback']) < 1e-12


@pytest.mark.parametrize('method', ['euler', 'midpoint', 'RK2', 'RK4'])
def test_golden_propagate_3d(hp, z, method):
    from oracle import pendulum as pd
    P = pd.pendulum_3d(3, 2)
    out = hp.pendulum_propagate(z['p3_F'], P.X, P.OJO, z['p3_MR'], P.b, P.G, 1e-3, P.L, None, None, method)
    assert rel(out, z[f'p3_Fnew_{method}']) < 1e-12


def test_golden_derivatives(hp, z):
    from oracle import pendulum as pd
    P = pd.pendulum_3d(3, 2)
    J = np.diag(P.params['J'])
    plan = hp.Plan(3, 2, 3, hp.HP_FP64, hp.HP_REAL)
    plan.set_model(P.L, P.b, P.G, z['p3_MR'], ((J[1] - J[2]) / J[0], (J[2] - J[0]) / J[1], (J[0] - J[1]) / J[2]))
    assert rel(plan.derivative(z['p3_F']), z['p3_dF']) < 1e-12
    Q = pd.pendulum_reduced(3, 3)
    plan2 = hp.Plan(3, 3, 2, hp.HP_FP64, hp.HP_REAL)
    plan2.set_model(Q.L, Q.b, Q.G, z['p2_MR'])
    assert rel(plan2.derivative(z['p2_F']), z['p2_dF']) < 1e-12


def test_golden_prod(hp, z):
    assert rel(hp.fftSO3_prod(z['prod_F'], z['prod_G']), z['prod_FG']) < 1e-12

"""CUDA hybrid collision operator vs the oracle restatement of
propagation/discrete/mex/sources/pendulum_reduced_collision (FP64)."""
import math

import numpy as np
import pytest

from oracle import collision as co
from oracle import pendulum as pd
from oracle import so3

pytestmark = pytest.mark.gpu

PRM = dict(d=0.12, h=0.2, r=0.025, theta_t=5 * math.pi / 180, lambda_max=100.0, epsilon=0.8)


@pytest.mark.parametrize('B,Bx', [(4, 3), (6, 8)])
def test_collision_tables_and_df(hp, B, Bx):
    L = 3.4
    Gd = (np.eye(2) * 0.05) @ (np.eye(2) * 0.05).T
    R = so3.rotation_grid(B)
    x = pd.omega_grid(Bx, L, 2)
    lam, indR, PC = co.get_lambda(R, x, PRM['d'], PRM['h'], PRM['r'], PRM['theta_t'], PRM['lambda_max'])
    Om = co.get_omega_new(R, x, indR, PRM['epsilon'])
    fcL, idx = co.get_fcL(x, Om, lam, Gd.ravel(order='F'), 10)

    plan = hp.Plan(B, Bx, 2, hp.HP_FP64, hp.HP_REAL)
    c = hp.Collision(plan, L=L, Gd=Gd, nD=10, **PRM)
    t = c.tables()
    assert c.numR == len(indR) and np.array_equal(t['indR'], indR)
    assert np.abs(t['PC'] - PC).max() < 1e-13
    assert np.abs(t['lambda_'] - lam).max() < 1e-10 * PRM['lambda_max']
    assert np.abs(t['omega'] - Om).max() < 1e-12
    # The kept taps agree up to the order of candidates whose Gaussian weights
    # tie in exact arithmetic (mirror-image source points; the last bit of exp
    # decides their order), which can move a tap across the nD boundary and
    # renormalise its source: most indices match and df agrees.
    assert np.mean(t['fcL_indx'] == idx) > 0.95
    # df on a seeded density
    f, _ = pd.seeded_density(B, Bx, 2, L, seed=3)
    fl = np.transpose(f, (4, 3, 2, 1, 0)).reshape(f.shape[3] * f.shape[4], -1)   # [ix][iR]
    ref = co.propagate_noise(fl, lam, indR, fcL, idx)
    out = c.df(f)
    outl = np.transpose(out, (4, 3, 2, 1, 0)).reshape(ref.shape)
    err = np.linalg.norm(outl - ref) / np.linalg.norm(ref)
    assert err < 1e-6, err

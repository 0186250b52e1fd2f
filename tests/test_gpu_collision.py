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


def to_ixiR(f):
    """f(a, b, c, i, j[, k]) -> [ix][iR] (ix = i + N j [+ N^2 k], iR = a + 2B b + 4B^2 c)."""
    nR = f.shape[0] * f.shape[1] * f.shape[2]
    return f.T.reshape(-1, nR)


@pytest.mark.parametrize('B,Bx', [(4, 3), (5, 4)])
def test_collision_3d_omega(hp, B, Bx):
    """The operator on a 3-D Omega grid (omega = R Omega with all three
    components, Omega+ in R^3, 3-D Gaussian landing kernel) against the
    oracle's 3-D restatement."""
    L = 3.4
    A = np.array([[0.06, 0.01, 0.0], [0.0, 0.05, 0.01], [0.0, 0.0, 0.07]])
    Gd = A @ A.T
    R = so3.rotation_grid(B)
    x = pd.omega_grid(Bx, L, 3)
    lam, indR, PC = co.get_lambda(R, x, PRM['d'], PRM['h'], PRM['r'], PRM['theta_t'], PRM['lambda_max'])
    Om = co.get_omega_new(R, x, indR, PRM['epsilon'])
    fcL, idx = co.get_fcL(x, Om, lam, Gd.ravel(order='F'), 10)

    plan = hp.Plan(B, Bx, 3, hp.HP_FP64, hp.HP_REAL)
    c = hp.Collision(plan, L=L, Gd=Gd, nD=10, **PRM)
    t = c.tables()
    assert c.numR == len(indR) > 0 and np.array_equal(t['indR'], indR)
    assert t['omega'].shape == Om.shape == ((2 * Bx) ** 3, len(indR), 3)
    assert np.abs(t['lambda_'] - lam).max() < 1e-10 * PRM['lambda_max']
    assert np.abs(t['omega'] - Om).max() < 1e-12
    assert np.mean(t['fcL_indx'] == idx) > 0.95
    f, _ = pd.seeded_density(B, Bx, 3, L, seed=5)
    ref = co.propagate_noise(to_ixiR(f), lam, indR, fcL, idx)
    out = c.df(f)
    err = np.linalg.norm(to_ixiR(out) - ref) / np.linalg.norm(ref)
    assert err < 1e-6, err


def test_collision_3d_tap_mass_balance(hp):
    """Every source point (ix2, k) that some landing point keeps as a tap loses
    exactly lambda(ix2, k) f through its taps (the per-source normalisation of
    getFcL.cu, with the dx^3 factors cancelling)."""
    B, Bx, L = 4, 3, 3.4
    Gd = np.diag([0.004, 0.004, 0.004])
    plan = hp.Plan(B, Bx, 3, hp.HP_FP64, hp.HP_REAL)
    c = hp.Collision(plan, L=L, Gd=Gd, nD=10, **PRM)
    t = c.tables()
    nx, k = t['lambda_'].shape
    out = np.zeros((nx, k))
    cnt = np.zeros((nx, k))
    for d in range(t['fcL'].shape[2]):
        sel = (t['fcL_indx'][:, :, d].astype(np.int64), np.arange(k)[None, :])
        np.add.at(out, sel, t['fcL'][:, :, d])
        np.add.at(cnt, sel, 1)
    kept = cnt > 0
    assert kept.mean() > 0.9
    assert np.allclose(out[kept], t['lambda_'][kept], rtol=1e-12, atol=1e-12 * PRM['lambda_max'])

"""Initial densities built on the GPU (matrix Fisher x Gaussian,
pendulum.m:210-220) against the oracle's seeded density and transform."""
import math

import numpy as np
import pytest

from oracle import pendulum as pd
from oracle import so3

pytestmark = pytest.mark.gpu


def rel(a, b):
    return float(np.linalg.norm((np.asarray(a) - np.asarray(b)).ravel()) / np.linalg.norm(np.asarray(b).ravel()))


def plan_for(hp, B, Bx, nd, precision=0, L=8.0):
    P = pd.pendulum_3d(B, Bx, L=L) if nd == 3 else pd.pendulum_reduced(B, Bx, L=L)
    plan = hp.Plan(B, Bx, nd, precision, hp.HP_REAL)
    plan.set_model(P.L, P.b, P.G, P.MR)
    return plan


@pytest.mark.parametrize('B,Bx,nd', [(4, 3, 3), (6, 4, 2), (10, 4, 3)])
def test_density_vs_oracle(hp, B, Bx, nd):
    f, prm = pd.seeded_density(B, Bx, nd, 8.0, seed=B * 7 + nd)
    plan = plan_for(hp, B, Bx, nd)
    out = plan.density_mf_gauss(prm['U'], prm['s'], prm['V'], prm['mu'], 0.25 * np.eye(nd))
    assert rel(out, f) < 1e-12


def test_correlated_gaussian(hp):
    B, Bx, nd, L = 4, 3, 3, 8.0
    rng = np.random.default_rng(1)
    U, V = pd.haar_rotation(rng), pd.haar_rotation(rng)
    s = np.array([9.0, 4.0, -1.5])
    A = rng.standard_normal((3, 3))
    Sigma = A @ A.T + 0.5 * np.eye(3)
    mu = np.array([0.3, -0.2, 0.1])
    out = plan_for(hp, B, Bx, nd).density_mf_gauss(U, s, V, mu, Sigma)
    R = so3.rotation_grid(B)
    fR = np.exp(np.einsum('ij,abcij->abc', U @ np.diag(s) @ V.T, R)) / pd.mf_normaliser(s)
    x = np.moveaxis(pd.omega_grid(Bx, L, nd), 0, -1) - mu
    fx = np.exp(-0.5 * np.einsum('...i,ij,...j->...', x, np.linalg.inv(Sigma), x)) / math.sqrt(
        (2 * math.pi) ** 3 * np.linalg.det(Sigma))
    assert rel(out, fR[..., None, None, None] * fx) < 1e-12


@pytest.mark.parametrize('precision', [0, 1])
def test_state_init(hp, precision):
    B, Bx, nd = 5, 3, 3
    f, prm = pd.seeded_density(B, Bx, nd, 8.0, seed=3)
    plan = plan_for(hp, B, Bx, nd, precision)
    st = hp.State(plan)
    st.init_mf_gauss(prm['U'], prm['s'], prm['V'], prm['mu'], 0.25 * np.eye(nd))
    assert rel(st.store(), so3.fftSO3R_forward(f)) < 1e-11

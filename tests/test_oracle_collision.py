"""CPU checks of the oracle's hybrid collision operator."""
import math

import numpy as np

from oracle import collision as co
from oracle import pendulum as pd
from oracle import so3

PARAMS = dict(d=0.12, h=0.2, r=0.025, theta_t=5 * math.pi / 180, lambda_max=100.0, epsilon=0.8)


def _setup(B=5, Bx=4, L=3.4, nD=10):
    R = so3.rotation_grid(B)
    x = pd.omega_grid(Bx, L, 2)
    lam, indR, PC = co.get_lambda(R, x, PARAMS['d'], PARAMS['h'], PARAMS['r'], PARAMS['theta_t'],
                                  PARAMS['lambda_max'])
    Om = co.get_omega_new(R, x, indR, PARAMS['epsilon'])
    Gd = (np.eye(2) * 0.05) @ (np.eye(2) * 0.05).T
    fcL, idx = co.get_fcL(x, Om, lam, Gd.ravel(order='F'), nD)
    return R, x, lam, indR, PC, Om, fcL, idx


def test_tables_shapes_and_ranges():
    R, x, lam, indR, PC, Om, fcL, idx = _setup()
    nx = x.shape[1] * x.shape[2]
    assert len(indR) > 0
    assert lam.shape == (nx, len(indR)) and Om.shape == (nx, len(indR), 2)
    assert fcL.shape == (nx, len(indR), 10) and idx.min() >= 0 and idx.max() < nx
    assert lam.min() >= 0 and lam.max() <= PARAMS['lambda_max'] + 1e-12


def test_collision_conserves_mass_per_attitude():
    """sum_x df(R, x) = 0 for every attitude whose sources all keep taps."""
    R, x, lam, indR, PC, Om, fcL, idx = _setup()
    rng = np.random.default_rng(0)
    nx = x.shape[1] * x.shape[2]
    f = rng.random((nx, R.shape[0] ** 3))
    df = co.propagate_noise(f, lam, indR, fcL, idx)
    kept = np.zeros((nx, len(indR)), bool)
    for k in range(len(indR)):
        kept[np.unique(idx[:, k, :]), k] = True
    ok = np.all(kept | (lam == 0), axis=0)
    s = df[:, indR].sum(axis=0)
    assert np.abs(s[ok]).max() < 1e-10 * np.abs(f).max() * PARAMS['lambda_max']
    others = np.setdiff1d(np.arange(f.shape[1]), indR)
    assert np.abs(df[:, others]).max() == 0.0


def test_reset_map_restitution_and_momentum():
    """discrete/test.m:45-53: with the contact geometry of the pendulum, the reset
    omega+ = omega - (1+eps)(omega.t)t gives vC+ . e1 = -eps vC . e1 and changes
    the angular momentum only along J^-1 (PC x e1)."""
    d, h, r, eps = 1.5, 2.0, 0.4, 0.7
    pc = math.hypot(r, h)
    rc = math.sqrt(pc * pc - d * d)
    PC = np.array([d, math.cos(math.pi / 4) * rc, math.sin(math.pi / 4) * rc])
    thr = math.asin(d / pc) - math.asin(r / pc)
    r3 = math.sin(thr) * np.array([1.0, 0, 0]) + math.cos(thr) * np.array([0, PC[1], PC[2]]) / rc
    t = np.cross(r3, [1.0, 0, 0])
    t /= np.linalg.norm(t)
    vC_old = t + np.cross(t, PC) / pc
    A = np.array([r3, [0, PC[2], -PC[1]], [-PC[2], 0, PC[0]]])
    omega_old = np.linalg.solve(A, np.array([0, vC_old[0], vC_old[1]]))
    omega_new = omega_old - (1 + eps) * (omega_old @ t) * t
    vC_new = np.cross(omega_new, PC)
    vC_o = np.cross(omega_old, PC)
    assert abs(vC_new[0] + eps * vC_o[0]) < 1e-12
    # omega+ - omega is parallel to t, and t is parallel to (PC x e1) projected:
    assert np.linalg.norm(np.cross(omega_new - omega_old, t)) < 1e-12

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


def test_3d_omega_extension_properties():
    """The 3-D Omega extension: lambda does not depend on the spin x3 about the
    pendulum axis; with x3 = 0 the reset map equals the 2-D one; the reset
    leaves the axial spin's contribution to omega unchanged."""
    B, Bx, L = 4, 3, 3.4
    R = so3.rotation_grid(B)
    x2 = pd.omega_grid(Bx, L, 2)
    x3 = pd.omega_grid(Bx, L, 3)
    a = (PARAMS['d'], PARAMS['h'], PARAMS['r'], PARAMS['theta_t'], PARAMS['lambda_max'])
    lam2, ind2, _ = co.get_lambda(R, x2, *a)
    lam3, ind3, _ = co.get_lambda(R, x3, *a)
    N = 2 * Bx
    assert np.array_equal(ind2, ind3)
    lam3 = lam3.reshape(N, N * N, -1)                 # [k3][i + N j][k]
    for k3 in range(N):
        assert np.array_equal(lam3[k3], lam2)
    Om2 = co.get_omega_new(R, x2, ind2, PARAMS['epsilon'])
    Om3 = co.get_omega_new(R, x3, ind3, PARAMS['epsilon']).reshape(N, N * N, len(ind3), 3)
    z = N // 2                                         # x3 = 0 plane
    assert np.abs(Om3[z, :, :, :2] - Om2).max() < 1e-13
    # a spin-only state (x1 = x2 = 0) is not reset: Omega+ = Omega
    c = N // 2
    spin = Om3[:, c + N * c, :, :]                     # x1 = x2 = 0, every x3
    xs = -L / 2 + L / N * np.arange(N)
    assert np.abs(spin[:, :, 2] - xs[:, None]).max() < 1e-12
    assert np.abs(spin[:, :, :2]).max() < 1e-12


def test_3d_fcl_never_nan_and_normalised():
    """A narrow 3-D landing kernel underflows at far landing points: those taps
    are 0 (no 0/0), and every source that keeps a tap still loses exactly lambda."""
    B, Bx, L = 4, 3, 4.0
    R = so3.rotation_grid(B)
    x = pd.omega_grid(Bx, L, 3)
    lam, indR, _ = co.get_lambda(R, x, PARAMS['d'], PARAMS['h'], PARAMS['r'], PARAMS['theta_t'],
                                 PARAMS['lambda_max'])
    Om = co.get_omega_new(R, x, indR, PARAMS['epsilon'])
    fcL, idx = co.get_fcL(x, Om, lam, (0.0025 * np.eye(3)).ravel(order='F'), 8)
    assert np.isfinite(fcL).all()
    nx, k = lam.shape
    out = np.zeros((nx, k))
    for d in range(8):
        np.add.at(out, (idx[:, :, d].astype(np.int64), np.arange(k)[None, :]), fcL[:, :, d])
    kept = out > 0
    assert np.allclose(out[kept], lam[kept], rtol=1e-12)

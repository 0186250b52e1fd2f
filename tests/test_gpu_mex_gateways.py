"""The MATLAB gateways of hybridpendulum-up_b200/mex/hp_mex.c, executed: each is
built against the host-memory MEX runtime of tests/mex_stub and libhp.so,
called with MATLAB-layout arrays through its mexFunction, and compared with the
FP64 oracle (<= 1e-10 relative L2 in FP64).  The loop body of
pendulum_reduced_hybrid.m:224-234 is run through the gateway calls alone.

Where oracle/build_ref.py has compiled the reference's own collision table
builders (oracle/_ref/getOmega_mex.so, getFcL_mex.so), the gateways and the
oracle restatement are also compared with the reference itself on the same
inputs."""
import math
import os

import numpy as np
import pytest

import mexrt
from oracle import collision as co
from oracle import gyro_bias as gb
from oracle import pendulum as pd
from oracle import so3

pytestmark = pytest.mark.gpu

TOL64 = 1e-10
PRM = dict(d=0.12, h=0.2, r=0.025, theta_t=5 * math.pi / 180, lambda_max=100.0, epsilon=0.8)
REF_DIR = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), 'oracle', '_ref')


def rel(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return float(np.linalg.norm((a - b).ravel()) / np.linalg.norm(b.ravel()))


def gw(define, name, extra=()):
    return mexrt.Gateway(mexrt.build_gateway(define, name, list(extra)))


@pytest.fixture(scope='module', autouse=True)
def _clear_plans():
    yield
    mexrt.clear_all()


def R_matlab(B):
    """R(3, 3, 2B, 2B, 2B) of fftSO3R.m:30-47, MATLAB order."""
    return np.asfortranarray(np.moveaxis(so3.rotation_grid(B), (3, 4), (0, 1)))


def x_matlab(Bx, L, nd=2):
    return np.asfortranarray(pd.omega_grid(Bx, L, nd))


def to_ixiR(f):
    return np.transpose(f, tuple(range(f.ndim - 1, -1, -1))).reshape(int(np.prod(f.shape[3:])), -1)


def test_propagate3_and_32_gateways(hp):
    B, Bx, dt = 4, 2, 1e-3
    P = pd.pendulum_3d(B, Bx)
    f, _ = pd.seeded_density(B, Bx, 3, P.L, seed=21)
    F = so3.fftSO3R_forward(f)
    ref = pd.integrate(F, lambda G: pd.derivative_fast(G, P), dt, 'RK2')
    u = hp.getu(B - 1)
    out = gw('HP_MEX_PROPAGATE3', 'pendulum_propagate').call(F, P.X, P.OJO, P.MR, P.b, P.G, dt, P.L, u, 0.0, 'RK2')[0]
    assert rel(out - F, ref - F) < TOL64
    out32 = gw('HP_MEX_PROPAGATE3', 'pendulum_propagate32', ['-DHP_MEX_MIXED']).call(
        F, P.X, P.OJO, P.MR, P.b, P.G, dt, P.L, u, 0.0, 'RK2')[0]
    assert rel(out32 - F, ref - F) < 1e-6


def test_propagate_reduced_gateway(hp):
    B, Bx, dt = 5, 3, 1e-3
    P = pd.pendulum_reduced(B, Bx)
    f, _ = pd.seeded_density(B, Bx, 2, P.L, seed=22, sigma=0.4)
    F = so3.fftSO3R_forward(f)
    ref = pd.integrate(F, lambda G: pd.derivative_fast(G, P), dt, 'midpoint')
    out = gw('HP_MEX_PROPAGATE2', 'pendulum_propagate_reduced').call(
        F, P.X, P.MR, P.b, P.G, dt, P.L, hp.getu(B - 1), 0.0, 'midpoint')[0]
    assert rel(out - F, ref - F) < TOL64


def test_fftSO3R_gateway(hp):
    B, Bx = 5, 3
    f, _ = pd.seeded_density(B, Bx, 2, 3.2, seed=23)
    g = gw('HP_MEX_FFTSO3R', 'fftSO3R_mex')
    F = g.call('forward', f, 0.0, 0.0)[0]
    assert rel(F, so3.fftSO3R_forward(f)) < TOL64
    f2 = g.call('backward', F, 0.0)[0]
    assert rel(f2, so3.ifftSO3R_backward(F, real=True)) < TOL64


def test_gyrobias_gateway(hp):
    B, Bx, L, dt = 4, 3, 2.0, 0.01
    f, _ = pd.seeded_density(B, Bx, 3, L, seed=24, sigma=0.3)
    F = so3.fftSO3R_forward(f)
    rng = np.random.default_rng(5)
    A = rng.standard_normal((3, 3))
    G1 = 0.05 * A @ A.T
    A = rng.standard_normal((3, 3))
    G2 = 0.01 * A @ A.T
    X = pd.make_X(pd.omega_grid(Bx, L, 3))
    ref = F + dt * gb.derivative_fast(F, L, G1, G2)
    out = gw('HP_MEX_GYROBIAS', 'gyrobias_propagate').call(F, X, dt, hp.getu(B - 1), G1, G2)[0]
    assert rel(out - F, ref - F) < TOL64


def test_propagate_reduced_den_gateway(hp):
    B, Bx, dt = 5, 4, 0.01
    P = pd.pendulum_reduced(B, Bx)
    f, _ = pd.seeded_density(B, Bx, 2, P.L, seed=25, sigma=0.4)
    F = so3.fftSO3R_forward(f)
    calls = []

    def deriv(Fx):
        fx = f if not calls else None
        calls.append(1)
        return pd.derivative_den(Fx, fx, P)
    ref = pd.integrate(F, deriv, dt, 'RK4')
    d = so3.wigner_d_table(B)
    w = so3.quad_weights(B)
    out = gw('HP_MEX_PROPAGATE_DEN', 'pendulum_propagate_reduced_den').call(
        F, f, P.X, np.asfortranarray(P.mR), P.b, P.G, dt, P.L, hp.getu(B - 1), d, w, 'RK4')[0]
    assert rel(out - F, ref - F) < TOL64


def collision_inputs(B, Bx, L):
    R = R_matlab(B)
    x = x_matlab(Bx, L)
    Gd = (0.05 * np.eye(2)) @ (0.05 * np.eye(2)).T
    return R, x, Gd


def test_collision_table_gateways_vs_oracle(hp):
    B, Bx, L, nD = 4, 3, 3.4, 10
    R, x, Gd = collision_inputs(B, Bx, L)
    lam, indR, PC = gw('HP_MEX_GETLAMBDA', 'getLambda_mex').call(
        R, x, PRM['d'], PRM['h'], PRM['r'], PRM['theta_t'], PRM['lambda_max'], False, nlhs=3)
    Rg = so3.rotation_grid(B)
    xg = pd.omega_grid(Bx, L, 2)
    lam_o, ind_o, PC_o = co.get_lambda(Rg, xg, PRM['d'], PRM['h'], PRM['r'], PRM['theta_t'], PRM['lambda_max'])
    assert indR.dtype == np.int32 and np.array_equal(indR.ravel(), ind_o)
    assert lam.shape == (len(ind_o), 2 * Bx, 2 * Bx)
    assert np.abs(lam.reshape(len(ind_o), -1, order='F').T - lam_o).max() < 1e-10 * PRM['lambda_max']
    assert np.abs(PC.reshape(3, -1, order='F').T - PC_o).max() < 1e-13
    Om = gw('HP_MEX_GETOMEGA', 'getOmega_mex').call(R, x, indR, PRM['epsilon'], PC, 'new')[0]
    Om_o = co.get_omega_new(Rg, xg, ind_o, PRM['epsilon'])                  # [ix][k][2]
    assert Om.shape == (2, len(ind_o), 2 * Bx, 2 * Bx)
    assert np.abs(np.transpose(Om.reshape(2, len(ind_o), -1, order='F'), (2, 1, 0)) - Om_o).max() < 1e-12
    fcL, idx = gw('HP_MEX_GETFCL', 'getFcL_mex').call(x, Om, lam, Gd, np.int32(nD), nlhs=2)
    fcL_o, idx_o = co.get_fcL(xg, Om_o, lam_o, Gd.ravel(order='F'), nD)       # [ix][k][d]
    assert fcL.shape == idx.shape == (nD, len(ind_o), 2 * Bx, 2 * Bx) and idx.dtype == np.int16
    f_l = np.transpose(fcL.reshape(nD, len(ind_o), -1, order='F'), (2, 1, 0))
    i_l = np.transpose(idx.reshape(nD, len(ind_o), -1, order='F'), (2, 1, 0))
    # taps of mirror-image source points tie in exact arithmetic; their order
    # (and so which one is kept at the nD boundary) follows the last bit of exp
    assert np.mean(i_l == idx_o) > 0.95
    # df through the discrete-propagate gateway vs the oracle propagate on the oracle's tables
    f, _ = pd.seeded_density(B, Bx, 2, L, seed=26, sigma=0.4)
    df = gw('HP_MEX_DISCRETE', 'pendulum_reduced_discrete_propagate').call(True, f, lam, indR, fcL, idx)[0]
    ref = co.propagate_noise(to_ixiR(f), lam_o, ind_o, fcL_o, idx_o)
    assert rel(to_ixiR(df), ref) < 1e-6
    # exactly the oracle propagate on the gateway's own tables
    ref_same = co.propagate_noise(to_ixiR(f), lam.reshape(len(ind_o), -1, order='F').T, indR.ravel(), f_l, i_l)
    assert rel(to_ixiR(df), ref_same) < 1e-13


def test_discrete_gateway_rejects_bad_tables(hp):
    B, Bx = 3, 2
    f = np.ones((6, 6, 6, 4, 4))
    lam = np.ones((2, 4, 4))
    fcL = np.ones((3, 2, 4, 4))
    bad_idx = np.full((3, 2, 4, 4), 99, np.int16)                          # beyond the 16 omega points
    g = gw('HP_MEX_DISCRETE', 'pendulum_reduced_discrete_propagate')
    with pytest.raises(mexrt.MexError, match='out of range'):
        g.call(True, f, lam, np.array([3, 5], np.int32), fcL, bad_idx)
    with pytest.raises(mexrt.MexError, match='out of range'):
        g.call(True, f, lam, np.array([5, 3], np.int32), fcL, np.zeros((3, 2, 4, 4), np.int16))


def test_hybrid_loop_body_through_gateways(hp):
    """pendulum_reduced_hybrid.m:224-234 with MEX calls only: propagate_den,
    fftSO3R backward, discrete propagate, Euler update of f, fftSO3R forward,
    against the oracle composition."""
    B, Bx, nD = 4, 3, 10
    L = 3.4
    P = pd.pendulum_reduced(B, Bx, L=L)
    R, x, Gd = collision_inputs(B, Bx, L)
    lam, indR, PC = gw('HP_MEX_GETLAMBDA', 'getLambda_mex').call(
        R, x, PRM['d'], PRM['h'], PRM['r'], PRM['theta_t'], PRM['lambda_max'], False, nlhs=3)
    Om = gw('HP_MEX_GETOMEGA', 'getOmega_mex').call(R, x, indR, PRM['epsilon'], PC, 'new')[0]
    fcL, idx = gw('HP_MEX_GETFCL', 'getFcL_mex').call(x, Om, lam, Gd, np.int32(nD), nlhs=2)
    f, _ = pd.seeded_density(B, Bx, 2, L, seed=27, sigma=0.4)
    F = so3.fftSO3R_forward(f)
    d, w = so3.wigner_d_table(B), so3.quad_weights(B)
    u = hp.getu(B - 1)
    prop = gw('HP_MEX_PROPAGATE_DEN', 'pendulum_propagate_reduced_den')
    fft = gw('HP_MEX_FFTSO3R', 'fftSO3R_mex')
    disc = gw('HP_MEX_DISCRETE', 'pendulum_reduced_discrete_propagate')
    dt = 0.01
    Fr, fr = F.copy(), f.copy()
    lam_l = lam.reshape(len(indR), -1, order='F').T
    f_l = np.transpose(fcL.reshape(nD, len(indR), -1, order='F'), (2, 1, 0))
    i_l = np.transpose(idx.reshape(nD, len(indR), -1, order='F'), (2, 1, 0))
    for _ in range(3):
        F = prop.call(F, f, P.X, np.asfortranarray(P.mR), P.b, P.G, dt, L, u, d, w, 'euler')[0]
        f = fft.call('backward', F, d)[0]
        df = disc.call(True, f, lam, indR, fcL, idx)[0]
        f = f + df * dt
        F = fft.call('forward', f, d, w)[0]
        # oracle
        Fr = pd.integrate(Fr, lambda G, f0=fr: pd.derivative_den(G, f0, P), dt, 'euler')
        fr = so3.ifftSO3R_backward(Fr, real=True)
        fl = to_ixiR(fr)
        fl = fl + dt * co.propagate_noise(fl, lam_l, indR.ravel(), f_l, i_l)
        fr = np.transpose(fl.reshape(2 * Bx, 2 * Bx, 2 * B, 2 * B, 2 * B), (4, 3, 2, 1, 0))
        Fr = so3.fftSO3R_forward(fr)
    assert rel(F, Fr) < TOL64
    assert rel(f, fr) < TOL64


# ---------------------------------------------- against the reference itself ----
def _ref_gateway(name):
    path = os.path.join(REF_DIR, name + '.so')
    if not os.path.exists(path):
        pytest.skip(f'{path} not built (oracle/build_ref.py needs the reference sources)')
    return mexrt.Gateway(path)


def test_omega_new_vs_reference_build(hp):
    """getOmega_mex('new') compiled from the reference's getOmega.cu against the
    library's gateway and the oracle restatement, same inputs."""
    B, Bx, L = 4, 3, 3.4
    R, x, _ = collision_inputs(B, Bx, L)
    lam, indR, PC = gw('HP_MEX_GETLAMBDA', 'getLambda_mex').call(
        R, x, PRM['d'], PRM['h'], PRM['r'], PRM['theta_t'], PRM['lambda_max'], False, nlhs=3)
    ref = _ref_gateway('getOmega_mex').call(R, x, indR, PRM['epsilon'], PC, 'new')[0]
    ours = gw('HP_MEX_GETOMEGA', 'getOmega_mex').call(R, x, indR, PRM['epsilon'], PC, 'new')[0]
    assert ref.shape == ours.shape
    assert np.abs(ours - ref).max() < 1e-12
    Om_o = co.get_omega_new(so3.rotation_grid(B), pd.omega_grid(Bx, L, 2), indR.ravel(), PRM['epsilon'])
    assert np.abs(np.transpose(ref.reshape(2, len(indR), -1, order='F'), (2, 1, 0)) - Om_o).max() < 1e-12


def test_fcL_vs_reference_build(hp):
    """getFcL_mex compiled from the reference's getFcL.cu (per-point thrust
    stable sort, host-side normalisation) against the library's gateway and the
    oracle restatement, on the same Omega+ and lambda."""
    B, Bx, L, nD = 4, 3, 3.4, 10
    R, x, Gd = collision_inputs(B, Bx, L)
    lam, indR, PC = gw('HP_MEX_GETLAMBDA', 'getLambda_mex').call(
        R, x, PRM['d'], PRM['h'], PRM['r'], PRM['theta_t'], PRM['lambda_max'], False, nlhs=3)
    Om = gw('HP_MEX_GETOMEGA', 'getOmega_mex').call(R, x, indR, PRM['epsilon'], PC, 'new')[0]
    fr, ir = _ref_gateway('getFcL_mex').call(x, Om, lam, Gd, np.int32(nD), nlhs=2)
    fo, io = gw('HP_MEX_GETFCL', 'getFcL_mex').call(x, Om, lam, Gd, np.int32(nD), nlhs=2)
    assert fr.shape == fo.shape and ir.dtype == io.dtype == np.int16
    same = ir == io
    assert same.mean() > 0.95
    assert np.abs(fo[same] - fr[same]).max() < 1e-12 * np.abs(fr).max()
    # the oracle restatement against the reference
    xg = pd.omega_grid(Bx, L, 2)
    Om_l = np.transpose(Om.reshape(2, len(indR), -1, order='F'), (2, 1, 0))
    lam_l = lam.reshape(len(indR), -1, order='F').T
    f_o, i_o = co.get_fcL(xg, Om_l, lam_l, Gd.ravel(order='F'), nD)
    i_r = np.transpose(ir.reshape(nD, len(indR), -1, order='F'), (2, 1, 0))
    f_r = np.transpose(fr.reshape(nD, len(indR), -1, order='F'), (2, 1, 0))
    s2 = i_o == i_r
    assert s2.mean() > 0.95
    assert np.abs(f_o[s2] - f_r[s2]).max() < 1e-12 * np.abs(f_r).max()
    # and the df each table set gives on one density agrees
    f, _ = pd.seeded_density(B, Bx, 2, L, seed=28, sigma=0.4)
    d_ref = co.propagate_noise(to_ixiR(f), lam_l, indR.ravel(), f_r, i_r)
    d_our = co.propagate_noise(to_ixiR(f), lam_l, indR.ravel(),
                               np.transpose(fo.reshape(nD, len(indR), -1, order='F'), (2, 1, 0)),
                               np.transpose(io.reshape(nD, len(indR), -1, order='F'), (2, 1, 0)))
    assert rel(d_our, d_ref) < 1e-6

"""CPU pins of the FP64 oracle's pendulum derivative and integrators."""
import os

import numpy as np
import pytest

from oracle import pendulum as pd
from oracle import so3

GOLD = os.path.join(os.path.dirname(__file__), 'golden', 'pendulum_small.npz')


def rel(a, b):
    return float(np.linalg.norm((a - b).ravel()) / np.linalg.norm(b.ravel()))


@pytest.mark.parametrize('B,Bx', [(3, 2), (4, 2)])
def test_literal_vs_fast_3d(B, Bx):
    """pendulum.m:388-527 restated literally (O(nx^2) convolutions, dense CG over
    every l2) equals the omega-FFT form with the degree-1 gravity block."""
    P = pd.pendulum_3d(B, Bx)
    f, _ = pd.seeded_density(B, Bx, 3, P.L, seed=B)
    F = so3.fftSO3R_forward(f)
    assert rel(pd.derivative_fast(F, P), pd.derivative_literal(F, P)) < 1e-13


def test_literal_vs_fast_reduced():
    P = pd.pendulum_reduced(4, 3)
    f, _ = pd.seeded_density(4, 3, 2, P.L, seed=1)
    F = so3.fftSO3R_forward(f)
    assert rel(pd.derivative_fast(F, P), pd.derivative_literal(F, P)) < 1e-13


def test_reference_scaled_setup():
    P, dtt = pd.pendulum_3d_reference_scaled(3, 2)
    f, _ = pd.seeded_density(3, 2, 3, P.L, seed=2)
    F = so3.fftSO3R_forward(f)
    assert rel(pd.derivative_fast(F, P), pd.derivative_literal(F, P)) < 1e-13
    assert abs(dtt - 1 / 400 / P.params['tscale']) < 1e-15


def test_density_gravity_equals_cg_gravity():
    """pendulum_reduced_den.m's f.mR gravity == pendulum_reduced.m's CG gravity
    (the multiplier is degree 1, so the B-grid quadrature is exact)."""
    P = pd.pendulum_reduced(5, 3)
    f, _ = pd.seeded_density(5, 3, 2, P.L, seed=3)
    F = so3.fftSO3R_forward(f)
    assert rel(pd.derivative_den(F, None, P), pd.derivative_fast(F, P)) < 1e-13


def test_gravity_multiplier_structure():
    """MR = fftSO3(J^-1(-m g rho x R^T e3)) lives in l2 = 1, m2 = 0 only."""
    P = pd.pendulum_3d(5, 2)
    lmax = 4
    big = np.abs(P.MR).max()
    for l2 in range(lmax + 1):
        for m2 in range(-l2, l2 + 1):
            blk = np.abs(P.MR[m2 + lmax, :, l2]).max()
            if not (l2 == 1 and m2 == 0):
                assert blk < 1e-13 * big


def test_mass_conservation_and_lie_l0():
    """d/dt F^0_00[k=0] = 0 (notes/6 pendulum/pendulum.tex:108-162)."""
    P = pd.pendulum_3d(4, 2)
    f, _ = pd.seeded_density(4, 2, 3, P.L, seed=4)
    F = so3.fftSO3R_forward(f)
    dF = pd.derivative_fast(F, P)
    lmax = 3
    assert abs(dF[lmax, lmax, 0, 0, 0, 0]) < 1e-12 * np.abs(dF).max()


def test_derivative_preserves_hermitian_symmetry():
    P = pd.pendulum_3d(3, 2)
    f, _ = pd.seeded_density(3, 2, 3, P.L, seed=5)
    dF = pd.derivative_fast(so3.fftSO3R_forward(f), P)
    df = so3.ifftSO3R_backward(dF, real=False)
    assert np.abs(df.imag).max() < 1e-12 * np.abs(df.real).max()


def test_rk_orders():
    """Euler / RK2 / RK4 of pendulum.m:346-385 converge at orders 1 / 2 / 4."""
    P = pd.pendulum_reduced(3, 2)
    f, _ = pd.seeded_density(3, 2, 2, P.L, seed=6)
    F0 = so3.fftSO3R_forward(f)
    der = lambda G: pd.derivative_fast(G, P)
    T = 0.02

    def run(meth, n):
        F = F0
        for _ in range(n):
            F = pd.integrate(F, der, T / n, meth)
        return F

    ref = run('rk4', 64)
    for meth, order in (('euler', 1), ('rk2', 2), ('rk4', 4)):
        e1 = np.linalg.norm(run(meth, 4) - ref)
        e2 = np.linalg.norm(run(meth, 8) - ref)
        assert abs(np.log2(e1 / e2) - order) < 0.35, (meth, np.log2(e1 / e2))


def test_golden_derivatives():
    z = np.load(GOLD)
    P = pd.pendulum_3d(3, 2)
    assert np.abs(P.MR - z['p3_MR']).max() < 1e-13 * np.abs(z['p3_MR']).max()
    assert rel(pd.derivative_fast(z['p3_F'], P), z['p3_dF']) < 1e-13
    for meth in ('euler', 'midpoint', 'RK2', 'RK4'):
        out = pd.integrate(z['p3_F'], lambda G: pd.derivative_fast(G, P), 1e-3, meth)
        assert rel(out, z[f'p3_Fnew_{meth}']) < 1e-14
    Q = pd.pendulum_reduced(3, 3)
    assert rel(pd.derivative_fast(z['p2_F'], Q), z['p2_dF']) < 1e-13
    assert rel(pd.derivative_den(z['p2_F'], None, Q), z['p2_dF_den']) < 1e-13

"""The gyro-bias restatement on CPU: the literal form of gyro_bias.m:226-300
against the FFT form, and known answers of the attitude diffusion."""
import numpy as np
import pytest

from oracle import gyro_bias as gb
from oracle import pendulum as pd
from oracle import so3


def sym(rng, scale):
    A = rng.standard_normal((3, 3))
    return scale * 0.5 * (A @ A.T)


@pytest.mark.parametrize('B,Bx', [(2, 2), (3, 2), (3, 3)])
def test_literal_equals_fast(B, Bx):
    rng = np.random.default_rng(B * 10 + Bx)
    f, _ = pd.seeded_density(B, Bx, 3, 2.0, seed=B + Bx, sigma=0.4)
    F = so3.fftSO3R_forward(f)
    G1, G2 = sym(rng, 0.01), sym(rng, 0.003)
    X = pd.make_X(gb.bias_grid(Bx, 2.0))
    d1 = gb.derivative_literal(F, X, G1, G2)
    d2 = gb.derivative_fast(F, 2.0, G1, G2)
    assert np.linalg.norm(d1 - d2) <= 1e-13 * np.linalg.norm(d1)


def test_isotropic_attitude_diffusion_is_casimir():
    """sum_i u_i u_i = -l(l+1) I, so G1 = g I gives -g l(l+1) F^l."""
    B, Bx = 4, 2
    f, _ = pd.seeded_density(B, Bx, 3, 2.0, seed=3)
    F = so3.fftSO3R_forward(f)
    g = 0.37
    D = gb.so3_diffusion(F, g * np.eye(3))
    l = np.arange(B).reshape(1, 1, B, 1, 1, 1)
    assert np.abs(D + g * l * (l + 1) * F).max() <= 1e-13 * np.abs(F).max()


def test_mass_is_conserved():
    """The l = 0, k = 0 coefficient (total mass) has zero derivative."""
    B, Bx = 3, 3
    rng = np.random.default_rng(5)
    f, _ = pd.seeded_density(B, Bx, 3, 2.0, seed=9)
    F = so3.fftSO3R_forward(f)
    d = gb.derivative_fast(F, 2.0, sym(rng, 0.02), sym(rng, 0.01))
    lmax = B - 1
    assert abs(d[lmax, lmax, 0, 0, 0, 0]) <= 1e-13 * abs(F[lmax, lmax, 0, 0, 0, 0])

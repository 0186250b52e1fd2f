"""The oracle's real-harmonic transforms (fftSO3.m / ifftSO3.m / getu.m isreal
branches) pinned against the complex-harmonic restatement: round trips, the
same band-limited function from both expansions, and the real Lie-derivative
matrices against the complex ones through fftSO3_deriv.m's identity."""
import numpy as np
import pytest

from oracle import real_harmonics as rh
from oracle import so3


def band_limited(B, seed):
    lmax = B - 1
    rng = np.random.default_rng(seed)
    F = np.zeros((2 * lmax + 1, 2 * lmax + 1, lmax + 1), complex)
    for l in range(lmax + 1):
        s = slice(lmax - l, lmax + l + 1)
        F[s, s, l] = rng.standard_normal((2 * l + 1, 2 * l + 1)) + 1j * rng.standard_normal((2 * l + 1, 2 * l + 1))
    return so3.ifftSO3R_backward(F, real=True)


@pytest.mark.parametrize('B', [2, 3, 5])
def test_round_trips(B):
    f = band_limited(B, B)
    F = rh.forward(f)
    assert np.abs(rh.backward(F) - f).max() <= 1e-12 * np.abs(f).max()
    assert np.abs(rh.forward(rh.backward(F)) - F).max() <= 1e-12 * np.abs(F).max()


def test_psi_symmetry_and_zero_block():
    B = 4
    P = rh.psi_table(B)
    lmax = B - 1
    for l in range(lmax + 1):
        for n in range(1, l + 1):
            assert np.array_equal(P[:, n + lmax, l, :], P[:, -n + lmax, l, :])
    d = so3.wigner_d_table(B)
    assert np.array_equal(P[lmax, lmax], d[lmax, lmax])


@pytest.mark.parametrize('eta', [(0.3, -0.5, 0.7), (1.0, 0.0, 0.0), (0.0, 0.0, -2.0)])
def test_real_lie_derivative_matches_complex(eta):
    B = 4
    lmax = B - 1
    f = band_limited(B, 11)
    Fc = so3.fftSO3R_forward(f)
    u = so3.getu(lmax)
    dFc = np.zeros_like(Fc)
    for l in range(lmax + 1):
        s = slice(lmax - l, lmax + l + 1)
        for i in range(3):
            dFc[s, s, l] += eta[i] * Fc[s, s, l] @ u[s, s, l, i].T
    df_c = so3.ifftSO3R_backward(dFc, real=True)
    df_r = rh.backward(rh.deriv(rh.forward(f), eta))
    assert np.abs(df_r - df_c).max() <= 1e-12 * np.abs(df_c).max()


def test_real_product_literal_equals_basis_change():
    """fftSO3_prod.m's real Clebsch-Gordan route = Re T (complex product) T^H."""
    B = 4
    lmax = B - 1
    f, g = band_limited(B, 1), band_limited(B, 2)
    FGr = rh.prod_literal(rh.forward(f), rh.forward(g))
    FGc = so3.fftSO3_prod(so3.fftSO3R_forward(f), so3.fftSO3R_forward(g))
    ref = np.zeros_like(FGr)
    for l in range(lmax + 1):
        s = slice(lmax - l, lmax + l + 1)
        T = rh.t_matrix(l)
        ref[s, s, l] = (T @ FGc[s, s, l] @ T.conj().T).real
    assert np.abs(FGr - ref).max() <= 1e-13 * np.abs(FGr).max()

"""get_stat restatement: the coefficient-space moments (the library's method)
against the reference's grid sums, and the moment-to-parameter map of the
matrix Fisher density."""

import numpy as np
import pytest

from oracle import pendulum as pd
from oracle import so3
from oracle import stats as st

pytestmark = pytest.mark.filterwarnings('ignore::scipy.integrate.IntegrationWarning')

@pytest.mark.parametrize('B,Bx,nd', [(3, 2, 3), (4, 3, 2), (5, 2, 3)])
def test_coefficient_moments_equal_grid_sums(B, Bx, nd):
    L = 4.0
    f, _ = pd.seeded_density(B, Bx, nd, L, seed=B + nd)
    F = so3.fftSO3R_forward(f)
    a = st.raw_moments_grid(f, L)
    b = st.moments_from_coeffs(F, L)
    for k in a:
        assert np.abs(np.asarray(a[k]) - np.asarray(b[k])).max() < 1e-13 * max(1.0, np.abs(a[k]).max()), k

def test_moments_of_a_non_bandlimited_grid_density():
    """The hybrid loop takes statistics of f after a grid-side update; the
    coefficients of its forward transform are the same discrete sums."""
    B, Bx, nd, L = 4, 3, 2, 4.0
    f, _ = pd.seeded_density(B, Bx, nd, L, seed=9)
    f = f * (1 + 0.1 * np.random.default_rng(0).standard_normal(f.shape))
    F = so3.fftSO3R_forward(f)
    a, b = st.raw_moments_grid(f, L), st.moments_from_coeffs(F, L)
    for k in a:
        assert np.abs(np.asarray(a[k]) - np.asarray(b[k])).max() < 1e-13 * max(1.0, np.abs(a[k]).max()), k

@pytest.mark.parametrize('s', [(5.0, 3.0, 1.0), (12.0, 8.0, -2.0), (0.5, 0.2, 0.1)])
def test_mf_moment_map_round_trip(s):
    d = st.mf_dlogc(s)
    assert np.abs(st.mf_M2S(d) - np.array(s)).max() < 1e-7 * max(1.0, max(abs(v) for v in s))

def test_mf_first_moment_matches_quadrature():
    """d_i of the normalised density exp(tr(S R)) / c(S) equals E[R_ii] on a fine grid."""
    s = np.array([6.0, 4.0, 2.0])
    B = 12
    R = so3.rotation_grid(B)
    w = so3.quad_weights(B)
    fR = np.exp(np.einsum('ii,abcii->abc', np.diag(s), R))
    fR /= np.einsum('b,abc->', w, fR)
    ER = np.einsum('abcij,b,abc->ij', R, w, fR)
    assert np.abs(np.diag(ER) - st.mf_dlogc(s)).max() < 1e-8

@pytest.mark.parametrize('nd', [2, 3])
def test_get_stat_fit_from_coefficients(nd):
    B, Bx, L = 5, 3, 4.0
    f, _ = pd.seeded_density(B, Bx, nd, L, seed=2)
    F = so3.fftSO3R_forward(f)
    ref = st.get_stat_grid(f, L)
    out = st.fit_from_moments(st.moments_from_coeffs(F, L), nd)
    for k in ('ER', 'Ex', 'Varx', 'EvR', 'ExvR', 'EvRvR', 'U', 'S', 'V', 'P', 'Miu', 'Sigma'):
        assert np.abs(out[k] - ref[k]).max() < 1e-9 * max(1.0, np.abs(ref[k]).max()), k

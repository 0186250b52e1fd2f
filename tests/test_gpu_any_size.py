"""Bandlimits and omega grids off the 2/3/5 sizes: every B in 2..32 and every
even omega grid of 4..64 points per axis is accepted.  FFT lengths with a
prime factor above 5 (2B = 14, 22, 26, 34, 62; 2Bx = 10 is 2*5, 14, 22, 26,
28, 34, 38) run a direct DFT for that factor.  Against the FP64 oracle:
transforms (real and complex, FP64 <= 1e-10, mixed <= 1e-6 relative L2), the
3-D derivative, the 2-D derivative on grids above 32 points (whole-array
omega FFTs), the tensor-core forward contraction where the padded node count
changes (2B = 26 -> 32, 2B = 50 -> 64), and propagation steps."""
import numpy as np
import pytest

from oracle import pendulum as pd
from oracle import so3

pytestmark = pytest.mark.gpu

TOL64 = 1e-10
TOLMIX = 1e-6


def rel(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return float(np.linalg.norm((a - b).ravel()) / np.linalg.norm(b.ravel()))


def coeffs(B, xs, seed, hermitian):
    rng = np.random.default_rng(seed)
    lmax = B - 1
    F = np.zeros((2 * lmax + 1, 2 * lmax + 1, lmax + 1) + xs, np.complex128)
    for l in range(lmax + 1):
        s = slice(lmax - l, lmax + l + 1)
        F[s, s, l] = (rng.standard_normal((2 * l + 1, 2 * l + 1) + xs)
                      + 1j * rng.standard_normal((2 * l + 1, 2 * l + 1) + xs)) / (2 * l + 1)
    if hermitian:
        F = so3.fftSO3R_forward(so3.ifftSO3R_backward(F, real=True))
    return F


def gyro_of(P):
    J = np.diag(P.params['J'])
    return ((J[1] - J[2]) / J[0], (J[2] - J[0]) / J[1], (J[0] - J[1]) / J[2])


@pytest.mark.parametrize('B,Bx,ndim', [(7, 5, 2), (9, 3, 3), (11, 7, 2), (13, 2, 3), (14, 5, 3), (17, 2, 2),
                                       (31, 2, 2)])
@pytest.mark.parametrize('precision', [0, 1])
def test_transforms_any_size(hp, B, Bx, ndim, precision):
    F = coeffs(B, (2 * Bx,) * ndim, seed=B + Bx, hermitian=True)
    f_ref = so3.ifftSO3R_backward(F, real=True)
    plan = hp.Plan(B, Bx, ndim, precision, hp.HP_REAL)
    tol = TOL64 if precision == 0 else TOLMIX
    f = plan.backward(F)
    assert rel(f, f_ref) < tol
    assert rel(plan.forward(f_ref), F) < tol


@pytest.mark.parametrize('B,Bx,ndim', [(7, 3, 3), (9, 5, 2)])
@pytest.mark.parametrize('precision', [0, 1])
def test_complex_roundtrip_any_size(hp, B, Bx, ndim, precision):
    F = coeffs(B, (2 * Bx,) * ndim, seed=3 * B, hermitian=False)
    plan = hp.Plan(B, Bx, ndim, precision, hp.HP_COMPLEX)
    f = plan.backward(F)
    tol = TOL64 if precision == 0 else TOLMIX
    assert rel(f, so3.ifftSO3R_backward(F, real=False)) < tol
    assert rel(plan.forward(f), F) < tol


@pytest.mark.parametrize('B,Bx', [(7, 5), (9, 7), (5, 9), (4, 13)])
@pytest.mark.parametrize('precision', [0, 1])
def test_derivative_3d_any_size(hp, B, Bx, precision):
    P = pd.pendulum_3d(B, Bx)
    f, _ = pd.seeded_density(B, Bx, 3, P.L, seed=B * Bx)
    F = so3.fftSO3R_forward(f)
    ref = pd.derivative_fast(F, P)
    plan = hp.Plan(B, Bx, 3, precision, hp.HP_REAL)
    plan.set_model(P.L, P.b, P.G, P.MR, gyro_of(P))
    assert rel(plan.derivative(F), ref) < (TOL64 if precision == 0 else TOLMIX)


@pytest.mark.parametrize('B,Bx', [(3, 17), (5, 19), (4, 27)])
@pytest.mark.parametrize('precision', [0, 1])
def test_derivative_2d_large_grid_any_size(hp, B, Bx, precision):
    # 2Bx = 34, 38, 54 > 32: the whole-array omega-FFT path of the 2-D derivative
    P = pd.pendulum_reduced(B, Bx)
    f, _ = pd.seeded_density(B, Bx, 2, P.L, seed=B + Bx)
    F = so3.fftSO3R_forward(f)
    ref = pd.derivative_fast(F, P)
    plan = hp.Plan(B, Bx, 2, precision, hp.HP_REAL)
    plan.set_model(P.L, P.b, P.G, P.MR)
    assert rel(plan.derivative(F), ref) < (TOL64 if precision == 0 else TOLMIX)


@pytest.mark.parametrize('engine', ['HP_BETA_TENSOR', 'HP_BETA_TENSOR_BF16'])
@pytest.mark.parametrize('B', [13, 25, 27])
def test_tensor_core_forward_any_size(hp, B, engine):
    F = coeffs(B, (4, 4), seed=B, hermitian=True)
    f = so3.ifftSO3R_backward(F, real=True)
    plan = hp.Plan(B, 2, 2, hp.HP_MIXED, hp.HP_REAL)
    plan.set_beta_engine(getattr(hp, engine))
    plan.profile(True)
    out = plan.forward(f)
    assert any(k.startswith('tf.anal.beta.tc') for k in plan.profile_read())
    assert plan.tc_errors() == 0
    assert rel(out, F) < TOLMIX


@pytest.mark.parametrize('precision', [0, 1])
def test_propagation_any_size(hp, precision):
    """Five Euler steps at B=7 on a 10^3 grid against the oracle's steps."""
    B, Bx, dt = 7, 5, 1e-3
    P = pd.pendulum_3d(B, Bx)
    f, _ = pd.seeded_density(B, Bx, 3, P.L, seed=77)
    F = so3.fftSO3R_forward(f)
    ref = F.copy()
    for _ in range(5):
        ref = ref + dt * pd.derivative_fast(ref, P)
    plan = hp.Plan(B, Bx, 3, precision, hp.HP_REAL)
    plan.set_model(P.L, P.b, P.G, P.MR, gyro_of(P))
    st = hp.State(plan)
    st.load(F)
    st.step(dt, 'euler', 5)
    assert rel(st.store(), ref) < (TOL64 if precision == 0 else TOLMIX)

"""Parity of the CUDA library (through its C ABI) with the FP64 oracle.

Tolerances: FP64 plans <= 1e-10 relative L2 (the bar for FP64 mode); mixed
plans <= 1e-6 relative L2 (the mixed-precision bar).  Sizes are small enough
for the oracle to finish in seconds.
"""
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


def random_coeffs(B, xs, seed, hermitian=False):
    rng = np.random.default_rng(seed)
    lmax = B - 1
    F = np.zeros((2 * lmax + 1, 2 * lmax + 1, lmax + 1) + xs, np.complex128)
    for l in range(lmax + 1):
        s = slice(lmax - l, lmax + l + 1)
        F[s, s, l] = (rng.standard_normal((2 * l + 1, 2 * l + 1) + xs)
                      + 1j * rng.standard_normal((2 * l + 1, 2 * l + 1) + xs)) / (2 * l + 1)
    if hermitian:
        f = so3.ifftSO3R_backward(F, real=True)
        F = so3.fftSO3R_forward(f)
    return F


def gyro_of(P):
    J = np.diag(P.params['J'])
    return ((J[1] - J[2]) / J[0], (J[2] - J[0]) / J[1], (J[0] - J[1]) / J[2])


@pytest.mark.parametrize('B', [2, 3, 5, 10, 15])
def test_wigner_d_and_weights(hp, B):
    plan = hp.get_plan(B, 2, 3)
    assert np.abs(plan.wigner_d() - so3.wigner_d_table(B)).max() < 1e-13
    assert np.abs(plan.quad_weights() - so3.quad_weights(B)).max() < 1e-16


@pytest.mark.parametrize('B,Bx,ndim', [(3, 2, 3), (5, 2, 3), (4, 3, 2), (10, 4, 3), (6, 4, 2)])
@pytest.mark.parametrize('precision', [0, 1])
def test_forward_real_density(hp, B, Bx, ndim, precision):
    f, _ = pd.seeded_density(B, Bx, ndim, 8.0, seed=B + 10 * Bx)
    ref = so3.fftSO3R_forward(f)
    out = hp.get_plan(B, Bx, ndim, precision, hp.HP_REAL).forward(f)
    assert rel(out, ref) < (TOL64 if precision == 0 else TOLMIX)


@pytest.mark.parametrize('B,Bx,ndim', [(3, 2, 3), (5, 2, 3), (4, 3, 2), (10, 4, 3), (6, 4, 2)])
@pytest.mark.parametrize('precision', [0, 1])
def test_backward_real_density(hp, B, Bx, ndim, precision):
    F = random_coeffs(B, (2 * Bx,) * ndim, seed=B, hermitian=True)
    ref = so3.ifftSO3R_backward(F, real=True)
    out = hp.get_plan(B, Bx, ndim, precision, hp.HP_REAL).backward(F)
    assert rel(out, ref) < (TOL64 if precision == 0 else TOLMIX)


@pytest.mark.parametrize('B,Bx,ndim', [(3, 2, 3), (4, 3, 2), (8, 2, 3)])
@pytest.mark.parametrize('precision', [0, 1])
def test_complex_roundtrip(hp, B, Bx, ndim, precision):
    F = random_coeffs(B, (2 * Bx,) * ndim, seed=7 + B)
    plan = hp.get_plan(B, Bx, ndim, precision, hp.HP_COMPLEX)
    f = plan.backward(F)
    ref = so3.ifftSO3R_backward(F, real=False)
    tol = TOL64 if precision == 0 else TOLMIX
    assert rel(f, ref) < tol
    F2 = plan.forward(ref)
    assert rel(F2, F) < tol


def _model3(hp, P, precision):
    plan = hp.get_plan(P.B, P.Bx, 3, precision, hp.HP_REAL)
    plan.set_model(P.L, P.b, P.G, P.MR, gyro_of(P))
    return plan


@pytest.mark.parametrize('B,Bx', [(3, 2), (5, 2), (4, 4), (6, 8)])
@pytest.mark.parametrize('precision', [0, 1])
def test_derivative_3d(hp, B, Bx, precision):
    P = pd.pendulum_3d(B, Bx)
    f, _ = pd.seeded_density(B, Bx, 3, P.L, seed=3)
    F = so3.fftSO3R_forward(f)
    ref = pd.derivative_fast(F, P)
    out = _model3(hp, P, precision).derivative(F)
    assert rel(out, ref) < (TOL64 if precision == 0 else TOLMIX)


def test_derivative_3d_literal(hp):
    """Against the statement-by-statement restatement of pendulum.m:388-527."""
    P = pd.pendulum_3d(3, 2)
    f, _ = pd.seeded_density(3, 2, 3, P.L, seed=11)
    F = so3.fftSO3R_forward(f)
    ref = pd.derivative_literal(F, P)
    out = _model3(hp, P, 0).derivative(F)
    assert rel(out, ref) < TOL64


def test_derivative_reference_scaled_setup(hp):
    """The exact scaled model of pendulum.m:41-208 through the MEX-shaped drop-in."""
    P, dtt = pd.pendulum_3d_reference_scaled(4, 2)
    f, _ = pd.seeded_density(4, 2, 3, P.L, seed=5)
    F = so3.fftSO3R_forward(f)
    ref = pd.integrate(F, lambda G: pd.derivative_fast(G, P), dtt, 'euler')
    u = hp.getu(3)
    out = hp.pendulum_propagate(F, P.X, P.OJO, P.MR, P.b, P.G, dtt, P.L, u, None, 'euler')
    assert rel(out, ref) < TOL64


@pytest.mark.parametrize('B,Bx', [(3, 2), (5, 3), (6, 8)])
@pytest.mark.parametrize('precision', [0, 1])
def test_derivative_reduced(hp, B, Bx, precision):
    P = pd.pendulum_reduced(B, Bx)
    f, _ = pd.seeded_density(B, Bx, 2, P.L, seed=4)
    F = so3.fftSO3R_forward(f)
    ref = pd.derivative_fast(F, P)
    plan = hp.get_plan(B, Bx, 2, precision, hp.HP_REAL)
    plan.set_model(P.L, P.b, P.G, P.MR)
    assert rel(plan.derivative(F), ref) < (TOL64 if precision == 0 else TOLMIX)


def test_reduced_dropin(hp):
    P = pd.pendulum_reduced(4, 3)
    f, _ = pd.seeded_density(4, 3, 2, P.L, seed=9)
    F = so3.fftSO3R_forward(f)
    ref = pd.integrate(F, lambda G: pd.derivative_fast(G, P), 1e-3, 'rk4')
    out = hp.pendulum_propagate_reduced(F, P.X, P.MR, P.b, P.G, 1e-3, P.L, None, None, 'RK4')
    assert rel(out, ref) < TOL64


@pytest.mark.parametrize('method', ['euler', 'midpoint', 'RK2', 'RK4'])
@pytest.mark.parametrize('precision', [0, 1])
def test_propagate_methods(hp, method, precision):
    P = pd.pendulum_3d(4, 2)
    f, _ = pd.seeded_density(4, 2, 3, P.L, seed=6)
    F = so3.fftSO3R_forward(f)
    dt = 1e-3
    ref = pd.integrate(F, lambda G: pd.derivative_fast(G, P), dt, method)
    out = _model3(hp, P, precision).propagate(F, dt, method)
    # compare the increments: the step itself must match, not just F
    assert rel(out - F, ref - F) < (TOL64 * 1e3 if precision == 0 else TOLMIX * 10)
    assert rel(out, ref) < (TOL64 if precision == 0 else TOLMIX)


def test_state_multistep_and_mass(hp):
    P = pd.pendulum_3d(4, 4)
    f, _ = pd.seeded_density(4, 4, 3, P.L, seed=8)
    F = so3.fftSO3R_forward(f)
    plan = _model3(hp, P, 0)
    st = hp.State(plan)
    st.load(F)
    m0 = st.mass()
    st.step(1e-3, 'euler', 5)
    ref = F
    for _ in range(5):
        ref = pd.integrate(ref, lambda G: pd.derivative_fast(G, P), 1e-3, 'euler')
    assert rel(st.store(), ref) < TOL64
    lmax = 3
    assert abs(m0 - F[lmax, lmax, 0, 0, 0, 0].real) < 1e-12 * abs(m0)
    assert abs(st.mass() - m0) < 1e-12 * abs(m0)


def test_state_normalize(hp):
    P = pd.pendulum_3d(3, 2)
    f, _ = pd.seeded_density(3, 2, 3, P.L, seed=12)
    F = so3.fftSO3R_forward(f)
    st = hp.State(_model3(hp, P, 0))
    st.load(F)
    m0 = st.mass()
    fac = st.normalize(2.0 * m0)
    assert abs(fac - 2.0) < 1e-14
    assert abs(st.mass() - 2.0 * m0) < 1e-13 * abs(m0)
    assert rel(st.store(), 2.0 * F) < 1e-14


@pytest.mark.parametrize('B', [2, 4, 6])
def test_fftSO3_prod(hp, B):
    F = random_coeffs(B, (), seed=B)
    G = random_coeffs(B, (), seed=B + 1)
    ref = so3.fftSO3_prod(F, G)
    out = hp.fftSO3_prod(F, G)
    assert rel(out, ref) < 1e-12


def test_gravity_rejects_alpha_dependent_multiplier(hp):
    P = pd.pendulum_3d(3, 2)
    MR = P.MR.copy()
    lmax = 2
    MR[lmax + 1, lmax, 1, 0] = 1.0   # an m2 = 1 component
    plan = hp.Plan(3, 2, 3)
    with pytest.raises(hp.HPError) as e:
        plan.set_model(P.L, P.b, P.G, MR, gyro_of(P))
    assert e.value.code == hp.HP_ERR_UNSUPPORTED


def test_errors(hp):
    with pytest.raises(hp.HPError) as e:
        hp.Plan(33, 2, 3)
    assert e.value.code == hp.HP_ERR_INVALID
    plan = hp.Plan(3, 2, 3)
    F = np.zeros(plan.F_shape, np.complex128)
    with pytest.raises(hp.HPError) as e:
        plan.propagate(F, 1e-3)
    assert e.value.code == hp.HP_ERR_NO_MODEL


@pytest.mark.parametrize('B,Bx', [(15, 2), (6, 3), (5, 2)])
def test_density_store_paths_agree(hp, B, Bx):
    """The mixed synthesis writes its runs by bulk copies (16-byte aligned
    buffer, even beta groups) or by plain stores (any other buffer): a density
    written one float past an aligned address equals the aligned one exactly,
    and both match the oracle."""
    import torch
    F = random_coeffs(B, (2 * Bx,) * 3, seed=B + 1, hermitian=True)
    ref = so3.ifftSO3R_backward(F, real=True)
    plan = hp.Plan(B, Bx, 3, hp.HP_MIXED, hp.HP_REAL)
    st = hp.State(plan)
    st.load(F)
    n = int(np.prod(plan.f_shape))
    buf = torch.zeros(n + 4, dtype=torch.float32, device='cuda')
    st.density_into(buf.data_ptr())
    a = buf[:n].clone()
    buf.zero_()
    st.density_into(buf.data_ptr() + 4)          # one float off the 16-byte grid
    torch.cuda.synchronize()
    assert torch.equal(buf[1:n + 1], a) and float(buf[0]) == 0.0 and float(buf[n + 1:].abs().sum()) == 0.0
    f = a.double().cpu().numpy().reshape(tuple(reversed(plan.f_shape))).transpose()
    assert rel(f, ref) < TOLMIX

"""The largest bandlimit, B=32 (64^3 Euler grid), where the transforms read
their d tables from global memory: parity with the oracle on a small omega
grid (FP64 <= 1e-10, mixed <= 1e-6 relative L2), complex and real plans."""
import numpy as np
import pytest

from oracle import so3

pytestmark = pytest.mark.gpu


def rel(a, b):
    return float(np.linalg.norm((np.asarray(a) - np.asarray(b)).ravel()) / np.linalg.norm(np.asarray(b).ravel()))


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


@pytest.mark.parametrize('precision', [0, 1])
def test_b32_complex_round_trip(hp, precision):
    B, Bx = 32, 2
    F = coeffs(B, (4, 4), 1, False)
    plan = hp.Plan(B, Bx, 2, precision, hp.HP_COMPLEX)
    f = plan.backward(F)
    tol = 1e-10 if precision == 0 else 1e-6
    assert rel(f, so3.ifftSO3R_backward(F, real=False)) < tol
    assert rel(plan.forward(f), F) < tol


@pytest.mark.parametrize('precision', [0, 1])
def test_b32_real(hp, precision):
    B, Bx = 32, 2
    F = coeffs(B, (4, 4), 2, True)
    plan = hp.Plan(B, Bx, 2, precision, hp.HP_REAL)
    f = plan.backward(F)
    tol = 1e-10 if precision == 0 else 1e-6
    assert rel(f, so3.ifftSO3R_backward(F, real=True)) < tol
    assert rel(plan.forward(f), F) < tol

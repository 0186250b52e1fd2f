"""CPU pins of the FP64 oracle's SO(3) harmonic analysis.

The reference has no tests or golden vectors; these checks pin the restatement
against the closed forms the reference ships beside its recursions and against
exact identities of the transforms.
"""
import math

import numpy as np
import pytest

from oracle import so3


def test_wigner_recursion_matches_closed_form():
    """Wigner_d.m's recursion (lines 11-47) vs its Jacobi closed form (lines 7-9)."""
    B = 6
    lmax = B - 1
    _, beta, _ = so3.so3_grid(B)
    d = so3.wigner_d(beta, lmax)
    err = 0.0
    for l in range(lmax + 1):
        for m in range(-l, l + 1):
            for n in range(-l, l + 1):
                for j in (0, 3, 2 * B - 1):
                    err = max(err, abs(d[m + lmax, n + lmax, l, j] - so3.wigner_d_closed(beta[j], l, m, n)))
    assert err < 1e-12


def test_wigner_identity_and_symmetry():
    lmax = 6
    d0 = so3.wigner_d(0.0, lmax)
    for l in range(lmax + 1):
        s = slice(lmax - l, lmax + l + 1)
        assert np.allclose(d0[s, s, l], np.eye(2 * l + 1), atol=1e-14)
    d = so3.wigner_d(0.7, lmax)
    for l in range(lmax + 1):
        for m in range(-l, l + 1):
            for n in range(-l, l + 1):
                assert abs(d[-m + lmax, -n + lmax, l] - (-1) ** (m - n) * d[m + lmax, n + lmax, l]) < 1e-14


@pytest.mark.parametrize('B', [3, 5, 8])
def test_quadrature_orthogonality(B):
    """sum_j w_j d^l_mn(b_j) d^l'_mn(b_j) = delta_ll' / (4 B^2 (2l+1))."""
    lmax = B - 1
    d = so3.wigner_d_table(B)
    w = so3.quad_weights(B)
    for m in range(-lmax, lmax + 1):
        for n in range(-lmax, lmax + 1):
            lo = max(abs(m), abs(n))
            G = np.einsum('j,lj,kj->lk', w, d[m + lmax, n + lmax, lo:], d[m + lmax, n + lmax, lo:])
            ref = np.diag([1.0 / (4 * B * B * (2 * l + 1)) for l in range(lo, lmax + 1)])
            assert np.abs(G - ref).max() < 1e-15


def _random_F(B, xs, seed):
    rng = np.random.default_rng(seed)
    lmax = B - 1
    F = np.zeros((2 * lmax + 1, 2 * lmax + 1, lmax + 1) + xs, np.complex128)
    for l in range(lmax + 1):
        s = slice(lmax - l, lmax + l + 1)
        F[s, s, l] = rng.standard_normal((2 * l + 1, 2 * l + 1) + xs) + 1j * rng.standard_normal((2 * l + 1, 2 * l + 1) + xs)
    return F


@pytest.mark.parametrize('xs', [(), (4,), (2, 2, 2)])
def test_round_trip(xs):
    F = _random_F(5, xs, 1)
    f = so3.ifftSO3R_backward(F, real=False)
    assert np.abs(so3.fftSO3R_forward(f) - F).max() < 1e-12 * np.abs(F).max()


def test_real_density_hermitian_symmetry():
    """Real f => F^l_{-m,-n}[-k] = (-1)^(m-n) conj F^l_{mn}[k]."""
    rng = np.random.default_rng(2)
    B, N = 4, 4
    f = rng.standard_normal((2 * B,) * 3 + (N, N))
    F = so3.fftSO3R_forward(f)
    lmax = B - 1
    mir = lambda a: np.roll(np.flip(a, axis=(-2, -1)), 1, axis=(-2, -1))   # k -> -k mod N
    for l in range(lmax + 1):
        for m in range(-l, l + 1):
            for n in range(-l, l + 1):
                lhs = F[-m + lmax, -n + lmax, l]
                rhs = (-1) ** (m - n) * np.conj(mir(F[m + lmax, n + lmax, l]))
                assert np.abs(lhs - rhs).max() < 1e-12 * np.abs(F).max()


def test_getu_matches_spectral_derivative():
    """fftSO3_deriv.m:7-27: sum_i eta_i F (u_i)^T is the transform of
    d/dt f(R exp(t hat(eta))) at t = 0; f is a degree-2 polynomial in R."""
    B = 4
    lmax = B - 1
    R = so3.rotation_grid(B)
    A = np.array([[0.3, -1.2, 0.5], [0.7, 0.1, -0.4], [1.1, 0.2, 0.9]])
    f = np.einsum('ij,abcji->abc', A, R) + R[..., 0, 1] ** 2 + R[..., 2, 0] * R[..., 1, 2]
    F = so3.fftSO3_forward(f)
    u = so3.getu(lmax)
    hat = lambda e: np.array([[0, -e[2], e[1]], [e[2], 0, -e[0]], [-e[1], e[0], 0]])
    for i in range(3):
        eta = np.eye(3)[i]
        dR = R @ hat(eta)            # d/dt R exp(t hat(eta))
        df = (np.einsum('ij,abcji->abc', A, dR) + 2 * R[..., 0, 1] * dR[..., 0, 1]
              + dR[..., 2, 0] * R[..., 1, 2] + R[..., 2, 0] * dR[..., 1, 2])
        dF = so3.fftSO3_forward(df)
        spec = np.zeros_like(F)
        for l in range(lmax + 1):
            s = slice(lmax - l, lmax + l + 1)
            spec[s, s, l] = F[s, s, l] @ u[s, s, l, i].T
        assert np.abs(spec - dF).max() < 1e-12 * max(1.0, np.abs(dF).max())


def test_getu_elementwise_branch():
    """getu.m's element-wise branch (lines 118-130) agrees with the array branch
    used by the propagation (lines 132-163) on the diagonal and the m-1 == n
    entries; its m+1 == n entries use sqrt((1+n)(l-n+1)) with the opposite sign
    and are not the Lie-derivative coefficients (the array branch is, as the
    spectral-derivative identity above shows)."""
    lmax = 5
    u = so3.getu(lmax)
    for l in range(lmax + 1):
        for m in range(-l, l + 1):
            for n in range(-l, l + 1):
                for ei in (1, 2, 3):
                    if m + 1 == n:
                        continue
                    assert abs(u[m + lmax, n + lmax, l, ei - 1] - so3.getu_element(l, m, n, ei)) < 1e-14


def _cg_racah(j1, m1, j2, m2, j, m):
    """Condon-Shortley Clebsch-Gordan coefficient from Racah's formula."""
    if m1 + m2 != m or abs(m1) > j1 or abs(m2) > j2 or abs(m) > j or not (abs(j1 - j2) <= j <= j1 + j2):
        return 0.0
    f = math.factorial
    pref = math.sqrt((2 * j + 1) * f(j + j1 - j2) * f(j - j1 + j2) * f(j1 + j2 - j) / f(j1 + j2 + j + 1))
    pref *= math.sqrt(f(j + m) * f(j - m) * f(j1 - m1) * f(j1 + m1) * f(j2 - m2) * f(j2 + m2))
    s = 0.0
    for k in range(0, j1 + j2 - j + 1):
        den = [k, j1 + j2 - j - k, j1 - m1 - k, j2 + m2 - k, j - j2 + m1 + k, j - j1 - m2 + k]
        if min(den) < 0:
            continue
        s += (-1) ** k / np.prod([float(f(x)) for x in den])
    return pref * s


@pytest.mark.parametrize('l1,l2', [(0, 0), (1, 1), (2, 1), (3, 2), (4, 4), (5, 1)])
def test_clebsch_gordan(l1, l2):
    """clebsch_gordan.m: orthogonal, and equal to Condon-Shortley up to one sign
    per (l1, l2, l) column block (the product rule only needs consistent signs
    across m, which the next test checks)."""
    CG = so3.clebsch_gordan(l1, l2)
    assert np.abs(CG.T @ CG - np.eye(CG.shape[0])).max() < 1e-12
    for l in range(abs(l1 - l2), l1 + l2 + 1):
        signs = set()
        for m in range(-l, l + 1):
            for m1 in range(-l1, l1 + 1):
                a = so3.cg_coeff(l1, m1, l2, m - m1, l, m)
                b = _cg_racah(l1, m1, l2, m - m1, l, m)
                assert abs(abs(a) - abs(b)) < 1e-12
                if abs(b) > 1e-8:
                    signs.add(int(np.sign(a * b)))
        assert len(signs) == 1


def test_product_rule_vs_grid_product():
    """fftSO3_prod.m:50 check: FG from the CG rule equals the transform of f.g
    when the product is band-limited (deg f + deg g <= lmax)."""
    B = 5
    R = so3.rotation_grid(B)
    f = R[..., 0, 0] + 0.5 * R[..., 2, 1] * R[..., 1, 1]          # degree 2
    g = 0.3 + R[..., 1, 2] - R[..., 0, 2] ** 2                    # degree 2
    F, G = so3.fftSO3_forward(f), so3.fftSO3_forward(g)
    FG = so3.fftSO3_prod(F, G)
    ref = so3.fftSO3_forward(f * g)
    assert np.abs(FG - ref).max() < 1e-12 * np.abs(ref).max()


def test_golden_transforms():
    import os
    z = np.load(os.path.join(os.path.dirname(__file__), 'golden', 'pendulum_small.npz'))
    assert np.abs(so3.fftSO3R_forward(z['p3_f']) - z['p3_F']).max() < 1e-13 * np.abs(z['p3_F']).max()
    assert np.abs(so3.ifftSO3R_backward(z['p3_F']) - z['p3_fback']).max() < 1e-13 * np.abs(z['p3_fback']).max()
    assert np.abs(so3.fftSO3_prod(z['prod_F'], z['prod_G']) - z['prod_FG']).max() < 1e-12 * np.abs(z['prod_FG']).max()

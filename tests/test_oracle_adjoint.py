"""The oracle's reverse mode on CPU: the adjoint identity <lam, A x> = <A^H lam, x>
and trajectory gradients against central finite differences."""
import numpy as np
import pytest

from oracle import adjoint as adj
from oracle import pendulum as pd
from oracle import so3


def rcoef(B, xs, rng, hermitian):
    lmax = B - 1
    F = np.zeros((2 * lmax + 1, 2 * lmax + 1, lmax + 1) + xs, np.complex128)
    for l in range(lmax + 1):
        s = slice(lmax - l, lmax + l + 1)
        F[s, s, l] = rng.standard_normal((2 * l + 1, 2 * l + 1) + xs) + 1j * rng.standard_normal((2 * l + 1, 2 * l + 1) + xs)
    if hermitian:
        F = so3.fftSO3R_forward(so3.ifftSO3R_backward(F, real=True))
    return F


def models():
    return [pd.pendulum_3d(3, 2, L=4.0), pd.pendulum_reduced(3, 2)]


@pytest.mark.parametrize('k', [0, 1])
def test_adjoint_identity(k):
    P = models()[k]
    rng = np.random.default_rng(3 + k)
    xs = (2 * P.Bx,) * P.ndim
    x = rcoef(P.B, xs, rng, False)
    lam = rcoef(P.B, xs, rng, False)
    lhs = adj.dot(lam, pd.derivative_fast(x, P))
    rhs = adj.dot(adj.derivative_adjoint(lam, P), x)
    assert abs(lhs - rhs) < 1e-11 * max(abs(lhs), 1.0)


def test_mirror_is_involution_and_fixes_real_densities():
    P = pd.pendulum_3d(3, 2, L=4.0)
    rng = np.random.default_rng(0)
    F = rcoef(3, (4, 4, 4), rng, True)
    assert np.abs(adj.mirror(F, 3) - F).max() < 1e-12 * np.abs(F).max()
    G = rcoef(3, (4, 4, 4), rng, False)
    assert np.abs(adj.mirror(adj.mirror(G, 3), 3) - G).max() < 1e-14 * np.abs(G).max()


@pytest.mark.parametrize('k', [0, 1])
def test_trajectory_gradients_vs_fd(k):
    P = models()[k]
    nd = P.ndim
    rng = np.random.default_rng(10 + k)
    xs = (2 * P.Bx,) * nd
    F0 = rcoef(P.B, xs, rng, True)
    C = rcoef(P.B, xs, rng, True)          # loss L = <C, F_T>
    dt, n = 0.01, 4
    lam0, grads, _ = adj.euler_adjoint(F0, C, P, dt, n)

    def loss(Pm, F=F0):
        Fx = F
        for _ in range(n):
            Fx = Fx + dt * pd.derivative_fast(Fx, Pm)
        return adj.dot(C, Fx)

    h = 1e-6
    # damping
    for i in range(nd):
        bp, bm = P.b.copy(), P.b.copy()
        bp[i] += h
        bm[i] -= h
        Pp = pd.Pendulum(**{**P.__dict__, 'b': bp})
        Pm = pd.Pendulum(**{**P.__dict__, 'b': bm})
        fd = (loss(Pp) - loss(Pm)) / (2 * h)
        assert abs(fd - grads[('b', i)]) < 1e-5 * max(abs(fd), 1e-3)
    # noise (independent entry G_ij)
    for i in range(nd):
        for j in range(i, nd):
            Gp, Gm = P.G.copy(), P.G.copy()
            Gp[i, j] += h
            Gm[i, j] -= h
            fd = (loss(pd.Pendulum(**{**P.__dict__, 'G': Gp})) - loss(pd.Pendulum(**{**P.__dict__, 'G': Gm}))) / (2 * h)
            assert abs(fd - grads[('G', i, j)]) < 1e-5 * max(abs(fd), 1e-3)
    # gravity scale of component 0
    MRp, MRm = P.MR.copy(), P.MR.copy()
    MRp[..., 0] *= 1 + h
    MRm[..., 0] *= 1 - h
    fd = (loss(pd.Pendulum(**{**P.__dict__, 'MR': MRp})) - loss(pd.Pendulum(**{**P.__dict__, 'MR': MRm}))) / (2 * h)
    assert abs(fd - grads[('gscale', 0)]) < 1e-5 * max(abs(fd), 1e-3)
    # gyroscopic coefficients: OJO_i = fftn(g_i x_j x_k)
    if nd == 3:
        pairs = [(1, 2), (0, 2), (0, 1)]
        for i in range(3):
            j, k2 = pairs[i]
            dO = np.zeros_like(P.OJO)
            dO[..., i] = np.fft.fftn(P.x[j] * P.x[k2])
            fd = (loss(pd.Pendulum(**{**P.__dict__, 'OJO': P.OJO + h * dO}))
                  - loss(pd.Pendulum(**{**P.__dict__, 'OJO': P.OJO - h * dO}))) / (2 * h)
            assert abs(fd - grads[('gyro', i)]) < 1e-5 * max(abs(fd), 1e-3)
    # initial coefficients along a real-density direction
    V = rcoef(P.B, xs, rng, True)
    fd = (loss(P, F0 + h * V) - loss(P, F0 - h * V)) / (2 * h)
    assert abs(fd - adj.dot(lam0, V)) < 1e-5 * max(abs(fd), 1e-3)


def test_measurement_weights_identity():
    """Re <(2l+1)/nx (L/N)^n fftSO3R(p), F> equals the grid quadrature of p f."""
    B, Bx, nd, L = 4, 2, 3, 8.0
    f, _ = pd.seeded_density(B, Bx, nd, L, seed=1)
    F = so3.fftSO3R_forward(f)
    fb = so3.ifftSO3R_backward(F, real=True)
    p, _ = pd.seeded_density(B, Bx, nd, L, seed=2)
    w = so3.quad_weights(B)
    c0 = (L / (2 * Bx)) ** nd
    I_grid = np.sum(w[None, :, None, None, None, None] * c0 * p * fb)
    W = (2 * np.arange(B) + 1).reshape(1, 1, B, 1, 1, 1) / (2 * Bx) ** nd * c0
    I_coef = adj.dot(so3.fftSO3R_forward(p) * W, F)
    assert abs(I_grid - I_coef) < 1e-13 * abs(I_grid)

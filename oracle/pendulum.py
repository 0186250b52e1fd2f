"""FP64 CPU restatement of the reference's pendulum Fokker-Planck step.

TEST INFRASTRUCTURE ONLY (see ``oracle/so3.py`` for the rules and the parity
status).  Two forms of the derivative are restated:

* ``derivative_literal`` follows ``propagation/pendulum.m:388-527`` (3-D Omega)
  and ``propagation/pendulum_reduced.m:362-465`` (2-D Omega) statement by
  statement: the omega-circular convolutions with flipped, shifted X / bX / OJO
  tables, the page-wise ``temp * u.'`` Lie term, the dense Clebsch-Gordan
  gravity loop over every (l, l2, l1, m, n) and the noise loop.  Its cost is
  O(nx^2) and O(B^7), so it only runs at small sizes.
* ``derivative_fast`` computes the same quantities with omega FFTs
  ((1/nx) X (*) F == fftn(x . ifftn(F)) exactly) and the gravity term with the
  degree-1 block of MR only (MR is the transform of a degree-1 function of R,
  so its l2 != 1 blocks are round-off; the literal form keeps them).  The two
  forms are cross-checked in ``tests/test_oracle_pendulum.py``.

Arrays use the reference's full layout F[m+lmax, n+lmax, l, i, j(, k)].
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np
import scipy.fft as sfft

from . import so3


# --------------------------------------------------------------- models ----
@dataclass
class Pendulum:
    """Derivative inputs of pendulum_propagate / pendulum_propagate_reduced
    (mex/pendulum_propagate/kernel.cu:16-76): X, OJO, MR, b, G, L plus sizes."""
    B: int
    Bx: int
    ndim: int                      # 3 (pendulum.m) or 2 (pendulum_reduced.m)
    L: float
    X: np.ndarray                  # (N,)*ndim + (ndim,) complex: fftn of the grid coordinates
    OJO: np.ndarray | None         # (N,)*3 + (3,) complex, None for ndim=2
    MR: np.ndarray                 # (2lmax+1, 2lmax+1, lmax+1, ndim) complex
    b: np.ndarray                  # (ndim,)
    G: np.ndarray                  # (ndim, ndim)
    x: np.ndarray = field(repr=False, default=None)   # (ndim, N, ...) grid
    mR: np.ndarray = field(repr=False, default=None)  # (ndim, 2B, 2B, 2B) samples
    params: dict = field(default_factory=dict)

    @property
    def lmax(self):
        return self.B - 1

    @property
    def N(self):
        return 2 * self.Bx


def omega_grid(Bx: int, L: float, ndim: int) -> np.ndarray:
    """x[:, i, j(, k)] = -L/2 + L/(2Bx) * index (pendulum.m:90-99)."""
    N = 2 * Bx
    g1 = -L / 2 + L / N * np.arange(N)
    return np.stack(np.meshgrid(*([g1] * ndim), indexing='ij'), 0)


def make_X(x: np.ndarray) -> np.ndarray:
    """X(..., i) = fftn(x_i) (pendulum.m:141-143)."""
    return np.stack([sfft.fftn(x[i]) for i in range(x.shape[0])], -1)


def make_OJO(x: np.ndarray, J: np.ndarray) -> np.ndarray:
    """OJO(..., i) = fftn((J^-1 (-x cross J x))_i) (pendulum.m:146-158)."""
    xv = np.moveaxis(x, 0, -1)                      # (..., 3)
    ojo = -np.cross(xv, xv @ J.T)
    ojo = ojo @ np.linalg.inv(J).T
    return np.stack([sfft.fftn(ojo[..., i]) for i in range(3)], -1)


def gravity_samples(B: int, mR_matrix: np.ndarray) -> np.ndarray:
    """mR_i(R) = sum_j A[i, j] R[2, j] on the SO(3) grid (third row of R; the
    reference's J^-1 [R32, -R31, 0] at pendulum.m:167-168 is A = J^-1 [[0,1,0],[-1,0,0],[0,0,0]])."""
    R = so3.rotation_grid(B)                         # (2B,2B,2B,3,3)
    r3 = R[..., 2, :]                                # third row
    return np.moveaxis(r3 @ mR_matrix.T, -1, 0)      # (ndim, 2B, 2B, 2B)


def make_MR(B: int, mR: np.ndarray) -> np.ndarray:
    """MR(:,:,:,i) = fftSO3(mR_i) (pendulum.m:176-192)."""
    return np.stack([so3.fftSO3_forward(mR[i]) for i in range(mR.shape[0])], -1)


def pendulum_3d(B: int, Bx: int, *, J=(0.02, 0.02, 0.01), rho=(0.0, 0.0, 0.1), mass=1.0,
                g=9.8, b=0.05, H=0.2, L=8.0) -> Pendulum:
    """Dimensional 3-D pendulum (Omega in R^3): Omega-dot = J^-1(-Omega x J Omega)
    - b Omega + J^-1(-m g rho x R^T e3) + noise H dW, the model of pendulum.m
    written without its time scaling (pendulum.m:41-58)."""
    J = np.diag(J) if np.ndim(J) == 1 else np.asarray(J, float)
    rho = np.asarray(rho, float)
    x = omega_grid(Bx, L, 3)
    # -m g rho x v  ==  A v  with A = -m g hat(rho)
    hat = np.array([[0, -rho[2], rho[1]], [rho[2], 0, -rho[0]], [-rho[1], rho[0], 0]])
    A = np.linalg.inv(J) @ (-mass * g * hat)
    mR = gravity_samples(B, A)
    bvec = np.full(3, b) if np.ndim(b) == 0 else np.asarray(b, float)
    Hm = H * np.eye(3) if np.ndim(H) == 0 else np.asarray(H, float)
    return Pendulum(B=B, Bx=Bx, ndim=3, L=L, X=make_X(x), OJO=make_OJO(x, J),
                    MR=make_MR(B, mR), b=bvec, G=0.5 * Hm @ Hm.T, x=x, mR=mR,
                    params=dict(J=J, rho=rho, mass=mass, g=g, A=A))


def pendulum_reduced(B: int, Bx: int, *, b=0.2, H=1.0, L=3.2, A=None) -> Pendulum:
    """2-D reduced pendulum of pendulum_reduced.m:41-182 (Omega in R^2, mR =
    [R32; -R31], no gyroscopic term)."""
    x = omega_grid(Bx, L, 2)
    A = np.array([[0.0, 1.0, 0.0], [-1.0, 0.0, 0.0]]) if A is None else np.asarray(A, float)
    mR = gravity_samples(B, A)
    bvec = np.full(2, b) if np.ndim(b) == 0 else np.asarray(b, float)
    Hm = H * np.eye(2) if np.ndim(H) == 0 else np.asarray(H, float)
    return Pendulum(B=B, Bx=Bx, ndim=2, L=L, X=make_X(x), OJO=None,
                    MR=make_MR(B, mR), b=bvec, G=0.5 * Hm @ Hm.T, x=x, mR=mR,
                    params=dict(A=A))


def pendulum_3d_reference_scaled(B: int, Bx: int) -> tuple[Pendulum, float]:
    """The exact scaled setup of pendulum.m:41-208 (J, rho, m of the reference,
    L=4, tscale-scaled b, H and time).  Returns (model, dtt)."""
    J = np.diag([0.0152492, 0.0142639, 0.00380233])
    rho3, mass, g = 0.0679878, 1.85480, 9.8
    Jt = J / J[0, 0]
    tscale = math.sqrt(J[0, 0] / (mass * g * rho3))
    dtt = 1 / 400 / tscale
    L = 4.0
    x = omega_grid(Bx, L, 3)
    A = np.linalg.inv(Jt) @ np.array([[0.0, 1.0, 0.0], [-1.0, 0.0, 0.0], [0.0, 0.0, 0.0]])
    mR = gravity_samples(B, A)
    bt = np.array([0.2, 0.2, 0.2]) * tscale
    Ht = np.eye(3) * 2 * tscale ** 1.5
    return Pendulum(B=B, Bx=Bx, ndim=3, L=L, X=make_X(x), OJO=make_OJO(x, Jt),
                    MR=make_MR(B, mR), b=bt, G=0.5 * Ht @ Ht.T, x=x, mR=mR,
                    params=dict(J=Jt, A=A, tscale=tscale)), dtt


# ------------------------------------------------------ initial density ----
def mf_normaliser(s) -> float:
    """c(s) = int_{-1}^{1} 1/2 exp(s3 u) I0((s1-s2)(1-u)/2) I0((s1+s2)(1+u)/2) du
    (pdf_MF_normal.m:38, integrand 205-211)."""
    from scipy.integrate import quad
    from scipy.special import iv
    s = np.asarray(s, float)
    val, _ = quad(lambda u: 0.5 * math.exp(s[2] * u) * iv(0, 0.5 * (s[0] - s[1]) * (1 - u))
                  * iv(0, 0.5 * (s[0] + s[1]) * (1 + u)), -1, 1, epsabs=0, epsrel=1e-13, limit=200)
    return val


def haar_rotation(rng) -> np.ndarray:
    """Haar-random rotation: QR of a Gaussian with sign fix, det = +1."""
    Q, Rr = np.linalg.qr(rng.standard_normal((3, 3)))
    Q = Q * np.sign(np.diag(Rr))
    if np.linalg.det(Q) < 0:
        Q[:, 0] = -Q[:, 0]
    return Q


def seeded_density(B: int, Bx: int, ndim: int, L: float, seed: int, sigma: float = 0.5):
    """Seeded matrix-Fisher(R; U diag(s) V^T) x Gaussian(omega; mu, sigma^2 I) on the
    grid, with U, V Haar-random, s ~ U[5, 20], mu ~ U[-1, 1]^ndim (the density family
    of pendulum.m:210-220 with seeded parameters).  Returns f[a, j, c, *x]."""
    rng = np.random.default_rng(seed)
    U, V = haar_rotation(rng), haar_rotation(rng)
    s = np.sort(rng.uniform(5, 20, 3))[::-1]
    mu = rng.uniform(-1, 1, ndim)
    Fm = U @ np.diag(s) @ V.T
    R = so3.rotation_grid(B)
    fR = np.exp(np.einsum('ij,abcij->abc', Fm, R)) / mf_normaliser(s)
    x = omega_grid(Bx, L, ndim)
    r2 = np.sum((np.moveaxis(x, 0, -1) - mu) ** 2, -1)
    fx = np.exp(-0.5 * r2 / sigma ** 2) / math.sqrt((2 * math.pi * sigma ** 2) ** ndim)
    return fR.reshape(fR.shape + (1,) * ndim) * fx, dict(U=U, V=V, s=s, mu=mu)


# ----------------------------------------------------------- derivative ----
def deriv_x(n1: int, B: int, L: float) -> complex:
    """deriv_x of pendulum.m:530-544 (1-based index n1; Nyquist -> 0)."""
    n = n1 - 1
    if n < B:
        return 2j * math.pi * n / L
    if n == B:
        return 0.0
    if B < n < 2 * B:
        return 2j * math.pi * (n - 2 * B) / L
    raise ValueError('n out of range')


def _c_first(Bx: int, L: float) -> np.ndarray:
    """2 pi i [0:Bx-1, 0, -Bx+1:-1] / L  (pendulum.m:504)."""
    k = np.concatenate([np.arange(Bx), [0], np.arange(-Bx + 1, 0)])
    return 2j * np.pi * k / L


def _noise_mult(Bx: int, L: float, ndim: int, G: np.ndarray) -> np.ndarray:
    """sum_ij G_ij c_ij of pendulum.m:510-523 on the omega grid."""
    N = 2 * Bx
    kd = np.concatenate([np.arange(Bx), np.arange(-Bx, 0)])
    kf = np.concatenate([np.arange(Bx), [0], np.arange(-Bx + 1, 0)])
    out = np.zeros((N,) * ndim)
    for i in range(ndim):
        for j in range(ndim):
            if i == j:
                c = -(4 * np.pi ** 2 * kd ** 2 / L ** 2)
                sh = [1] * ndim
                sh[i] = N
                out = out + G[i, j] * c.reshape(sh)
            else:
                c = 2 * np.pi * kf / L
                shi = [1] * ndim
                shi[i] = N
                shj = [1] * ndim
                shj[j] = N
                out = out + G[i, j] * (-(c.reshape(shi) * c.reshape(shj)))
    return out


def _circ_conv_literal(T: np.ndarray, F: np.ndarray, ndim: int) -> np.ndarray:
    """temp(:,:,:,ix,jx[,kx]) = sum(T_ijk .* F, x-axes) / N^ndim with T_ijk =
    circshift(flip(T), (ix, jx[, kx])) (pendulum.m:400-414)."""
    N = T.shape[0]
    out = np.zeros_like(F)
    idx = np.arange(N)
    for o in np.ndindex(*(N,) * ndim):
        # T_ijk[a, b, c] = T[(o1 - a) mod N, (o2 - b) mod N, (o3 - c) mod N]
        sel = np.ix_(*[(oi - idx) % N for oi in o])
        Ts = T[sel]
        out[(Ellipsis,) + o] = np.tensordot(F, Ts, axes=(list(range(3, 3 + ndim)),
                                                         list(range(ndim)))) / N ** ndim
    return out


def _gravity_literal(F: np.ndarray, MRi: np.ndarray) -> np.ndarray:
    """temp_i of the CG loop of pendulum.m:470-502 (every l2, dense CG)."""
    lmax = F.shape[2] - 1
    temp = np.zeros_like(F)
    for l in range(lmax + 1):
        for l2 in range(lmax + 1):
            ind2 = slice(lmax - l2, lmax + l2 + 1)
            l1_all = [l1 for l1 in range(lmax + 1) if abs(l1 - l2) <= l <= l1 + l2]
            for l1 in l1_all:
                cl = (2 * l1 + 1) * (2 * l2 + 1) / (2 * l + 1)
                col = l * l - (l1 - l2) ** 2
                ind1 = slice(lmax - l1, lmax + l1 + 1)
                CG = so3.clebsch_gordan(l1, l2)
                MRb = MRi[ind2, ind2, l2]
                for m in range(-l, l + 1):
                    CGm = CG[:, col + m + l].reshape(2 * l1 + 1, 2 * l2 + 1).T
                    for n in range(-l, l + 1):
                        CGn = CG[:, col + n + l].reshape(2 * l1 + 1, 2 * l2 + 1).T
                        K = CGm.T @ MRb @ CGn                    # (2l1+1, 2l1+1)
                        temp[m + lmax, n + lmax, l] += cl * np.tensordot(
                            K, F[ind1, ind1, l1], axes=([0, 1], [0, 1]))
    return temp


def derivative_literal(F: np.ndarray, P: Pendulum) -> np.ndarray:
    """dF of pendulum.m:388-527 (ndim=3) / pendulum_reduced.m:362-465 (ndim=2)."""
    lmax, Bx, L, nd = P.lmax, P.Bx, P.L, P.ndim
    u = so3.getu(lmax)
    dF = np.zeros_like(F)
    temps = [_circ_conv_literal(P.X[..., i], F, nd) for i in range(nd)]
    for l in range(lmax + 1):
        s = slice(lmax - l, lmax + l + 1)
        for i in range(nd):
            blk = np.moveaxis(temps[i][s, s, l], (0, 1), (-2, -1))
            dF[s, s, l] -= np.moveaxis(blk @ u[s, s, l, i].T, (-2, -1), (0, 1))
    N = 2 * Bx
    cx = np.array([deriv_x(n1, Bx, L) for n1 in range(1, N + 1)])

    def conv_term(T):
        out = np.zeros_like(F)
        for i in range(nd):
            t = _circ_conv_literal(T[..., i], F, nd)
            sh = [1] * (3 + nd)
            sh[3 + i] = N
            out -= t * cx.reshape(sh)
        return out

    dF += conv_term(-P.b * P.X)
    if nd == 3 and P.OJO is not None:
        dF += conv_term(P.OJO)
    c = _c_first(Bx, L)
    for i in range(nd):
        t = _gravity_literal(F, P.MR[..., i])
        sh = [1] * (3 + nd)
        sh[3 + i] = N
        dF -= t * c.reshape(sh)
    dF += F * _noise_mult(Bx, L, nd, P.G)
    return dF


# --- fast form ---
def _xaxes(nd):
    return tuple(range(3, 3 + nd))


def gravity_taps(lmax: int, MR1: np.ndarray):
    """Sparse degree-1 product: Grav^l_{mn} = sum_{l1, m2, n2} W F^{l1}_{m-m2, n-n2} with
    W = (2l1+1)*3/(2l+1) <l1 m-m2; 1 m2|l m><l1 n-n2; 1 n2|l n> MR^1_{m2 n2}
    (the l2 = 1 terms of pendulum.m:474-502).  MR1: (3, 3) block MR[lmax-1:lmax+2,
    lmax-1:lmax+2, 1].  Returns a list of (l, m, n, l1, m1, n1, W)."""
    taps = []
    for l in range(lmax + 1):
        for l1 in (l - 1, l, l + 1):
            if l1 < 0 or l1 > lmax or l1 + 1 < l:
                continue
            cl = (2 * l1 + 1) * 3 / (2 * l + 1)
            for m in range(-l, l + 1):
                for m2 in (-1, 0, 1):
                    m1 = m - m2
                    if abs(m1) > l1:
                        continue
                    cm = so3.cg_coeff(l1, m1, 1, m2, l, m)
                    if cm == 0.0:
                        continue
                    for n in range(-l, l + 1):
                        for n2 in (-1, 0, 1):
                            n1 = n - n2
                            if abs(n1) > l1:
                                continue
                            cn = so3.cg_coeff(l1, n1, 1, n2, l, n)
                            w = cl * cm * cn * MR1[m2 + 1, n2 + 1]
                            if w != 0:
                                taps.append((l, m, n, l1, m1, n1, w))
    return taps


def gravity_fast(F: np.ndarray, MRi: np.ndarray) -> np.ndarray:
    lmax = F.shape[2] - 1
    MR1 = MRi[lmax - 1:lmax + 2, lmax - 1:lmax + 2, 1]
    out = np.zeros_like(F)
    for (l, m, n, l1, m1, n1, w) in gravity_taps(lmax, MR1):
        out[m + lmax, n + lmax, l] += w * F[m1 + lmax, n1 + lmax, l1]
    return out


def derivative_fast(F: np.ndarray, P: Pendulum, *, gravity: str = 'l2=1') -> np.ndarray:
    """Same dF as ``derivative_literal`` with omega FFTs.  ``gravity='full'``
    keeps every l2 block of MR (slow), 'l2=1' the degree-1 block only."""
    lmax, Bx, L, nd = P.lmax, P.Bx, P.L, P.ndim
    N = 2 * Bx
    ax = _xaxes(nd)
    u = so3.getu(lmax)
    Fp = sfft.ifftn(F, axes=ax)
    xs = [sfft.ifftn(P.X[..., i]) for i in range(nd)]          # grid coordinates
    dF = np.zeros_like(F)
    PF = [sfft.fftn(Fp * xs[i], axes=ax) for i in range(nd)]   # F_omega[x_i f]
    for l in range(lmax + 1):
        s = slice(lmax - l, lmax + l + 1)
        for i in range(nd):
            blk = np.moveaxis(PF[i][s, s, l], (0, 1), (-2, -1))
            dF[s, s, l] -= np.moveaxis(blk @ u[s, s, l, i].T, (-2, -1), (0, 1))
    c = _c_first(Bx, L)

    def cmul(T, i):
        sh = [1] * (3 + nd)
        sh[3 + i] = N
        return T * c.reshape(sh)

    for i in range(nd):
        dF -= cmul(-P.b[i] * PF[i], i)
    if nd == 3 and P.OJO is not None:
        for i in range(3):
            ojo = sfft.ifftn(P.OJO[..., i])
            dF -= cmul(sfft.fftn(Fp * ojo, axes=ax), i)
    for i in range(nd):
        g = _gravity_literal(F, P.MR[..., i]) if gravity == 'full' else gravity_fast(F, P.MR[..., i])
        dF -= cmul(g, i)
    dF += F * _noise_mult(Bx, L, nd, P.G)
    return dF


def derivative_fast_mgroup(Fm: np.ndarray, m: int, P: Pendulum) -> np.ndarray:
    """The rows of one order m of ``derivative_fast``, from the rows of that m alone.

    Every term of the pendulum derivative keeps m (the alpha frequency):
    the Lie matrices u^l_i act on n by right multiplication (pendulum.m:418-420,
    getu.m:132-163); damping, gyroscopic and noise terms are pointwise in
    (l, m, n) (pendulum.m:424-466, 510-523); and the gravity multiplier
    mR_i(R) = sum_j A_ij R_3j depends on R only through its third row
    (-sin b cos g, sin b sin g, cos b), which does not involve alpha, so MR^1 is
    non-zero only at m2 = 0 and the l2 = 1 product of pendulum.m:474-502 keeps m.
    This lets the full-size workload (B = 15 on a 32^3 omega grid, 6.6 GB per
    full coefficient array) be checked one m group at a time.
    Fm = F[m + lmax] (shape (2lmax+1, lmax+1, *x)); returns dF[m + lmax]."""
    lmax, Bx, L, nd = P.lmax, P.Bx, P.L, P.ndim
    N = 2 * Bx
    ax = tuple(range(2, 2 + nd))
    u = so3.getu(lmax)
    MR1 = [P.MR[lmax - 1:lmax + 2, lmax - 1:lmax + 2, 1, i] for i in range(nd)]
    for blk in MR1:
        scale = max(np.abs(blk).max(), 1e-300)
        if max(np.abs(blk[0]).max(), np.abs(blk[2]).max()) > 1e-12 * scale:
            raise ValueError('gravity multiplier depends on alpha: m groups are coupled')
    Fp = sfft.ifftn(Fm, axes=ax)
    xs = [sfft.ifftn(P.X[..., i]) for i in range(nd)]
    PF = [sfft.fftn(Fp * xs[i], axes=ax) for i in range(nd)]
    dF = np.zeros_like(Fm)
    for l in range(abs(m), lmax + 1):
        s = slice(lmax - l, lmax + l + 1)
        for i in range(nd):
            blk = np.moveaxis(PF[i][s, l], 0, -1)                  # (*x, n)
            dF[s, l] -= np.moveaxis(blk @ u[s, s, l, i].T, -1, 0)
    c = _c_first(Bx, L)

    def cmul(T, i):
        sh = [1] * (2 + nd)
        sh[2 + i] = N
        return T * c.reshape(sh)

    for i in range(nd):
        dF -= cmul(-P.b[i] * PF[i], i)
    if nd == 3 and P.OJO is not None:
        for i in range(3):
            ojo = sfft.ifftn(P.OJO[..., i])
            dF -= cmul(sfft.fftn(Fp * ojo, axes=ax), i)
    for i in range(nd):
        g = np.zeros_like(Fm)
        for (l, mm, n, l1, m1, n1, w) in gravity_taps(lmax, MR1[i]):
            if mm == m and m1 == m:
                g[n + lmax, l] += w * Fm[n1 + lmax, l1]
        dF -= cmul(g, i)
    dF += Fm * _noise_mult(Bx, L, nd, P.G)
    return dF


def integrate(F: np.ndarray, deriv, dt: float, method: str = 'euler') -> np.ndarray:
    """Time integrators of pendulum.m:346-385 (euler, midpoint, RK2, RK4)."""
    method = method.lower()
    dF1 = deriv(F)
    if method == 'euler':
        return F + dt * dF1
    if method in ('midpoint', 'rk4'):
        dF2 = deriv(F + dF1 * dt / 2)
        if method == 'midpoint':
            return F + dt * dF2
    elif method == 'rk2':
        dF2 = deriv(F + dF1 * dt)
        return F + dt / 2 * (dF1 + dF2)
    else:
        raise ValueError("method must be one of 'euler', 'midpoint', 'RK2', 'RK4'")
    dF3 = deriv(F + dF2 * dt / 2)
    dF4 = deriv(F + dF3 * dt)
    return F + 1 / 6 * dt * (dF1 + 2 * dF2 + 2 * dF3 + dF4)


# ------------------------------------------------------- density gravity ----
def derivative_den(F: np.ndarray, f: np.ndarray | None, P: Pendulum) -> np.ndarray:
    """dF of pendulum_reduced_den.m:401-533: the Lie, damping and noise terms of
    the reduced model with the gravity term formed on the grid,
    FMR_i = fftSO3R(f . mR_i).  When ``f`` is None it is recomputed from F by
    the complex backward transform (pendulum_reduced_den.m:454-475)."""
    assert P.ndim == 2
    lmax, Bx, L = P.lmax, P.Bx, P.L
    N = 2 * Bx
    Pn = Pendulum(B=P.B, Bx=Bx, ndim=2, L=L, X=P.X, OJO=None, MR=np.zeros_like(P.MR),
                  b=P.b, G=np.zeros_like(P.G))
    dF = derivative_fast(F, Pn)
    if f is None:
        f = so3.ifftSO3R_backward(F, real=False)
    c = _c_first(Bx, L)
    for i in range(2):
        fm = f * P.mR[i].reshape(P.mR[i].shape + (1, 1))
        FMR = so3.fftSO3R_forward(fm)
        sh = [1] * 5
        sh[3 + i] = N
        dF -= FMR * c.reshape(sh)
    dF += F * _noise_mult(Bx, L, 2, P.G)
    return dF

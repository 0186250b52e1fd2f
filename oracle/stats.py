"""FP64 restatement of the per-step statistics get_stat (test infrastructure only).

``get_stat_grid`` follows propagation/pendulum.m:547-594 (3-D omega) and
propagation/pendulum_reduced_hybrid.m:304-351 (2-D omega, also returns fx)
statement by statement on the grid density f, with the proper SVD of
'matrix Fisher/psvd.m' and the moment-to-parameter map of
'matrix Fisher/pdf_MF_M2S.m' (solved here with a root finder on
grad log c(s) = d; the reference uses Newton-Armijo on the same equations,
pdf_MF_M2S.m:55-104 with func() at :137-165, so both land on the unique root
up to the solver tolerance).

``moments_from_coeffs`` computes the same raw moments from the transform
coefficients F = fftSO3R(f): every moment in get_stat integrates f against a
polynomial of degree <= 2 in the entries of R and in omega, so it is a finite
combination of F^l_{mn}[k] with l <= 2 (k = 0) or l <= 1 (k on the omega axes):
  E[h(R)]     = c0 sum_{lmn} a^h_{lmn} F^l_{mn}[0],   h = sum a^h conj(D^l_mn)
  E[x_i h(R)] = c0 / N sum_q sum_{lmn} a^h_{lmn} F^l_{mn}[q e_i] conj(xi(q))
with c0 = (L/2Bx)^n and xi the DFT of the grid coordinate.  This is the
library's method (no pass over f); this module pins it to the grid form.
"""
from __future__ import annotations

import math

import numpy as np
from scipy import integrate, optimize, special

from . import so3
from .pendulum import omega_grid


# ----------------------------------------------------------- MF helpers ----
def psvd(F: np.ndarray):
    """Proper SVD ('matrix Fisher/psvd.m:1-15'): F = U S V^T with U, V in SO(3)."""
    U, s, Vh = np.linalg.svd(F)
    V = Vh.T
    S = np.diag(s) @ np.diag([1, 1, np.linalg.det(U @ V)])
    U = U @ np.diag([1, 1, np.linalg.det(U)])
    V = V @ np.diag([1, 1, np.linalg.det(V)])
    return U, S, V


def _kunze(s, order):
    """c(s) and its gradient, scaled by a common exponential (ratios only):
    c(s) = int_{-1}^{1} 1/2 e^{s3 u} I0((s1-s2)(1-u)/2) I0((s1+s2)(1+u)/2) du
    ('matrix Fisher/pdf_MF_normal.m:38', integrand :205-211)."""
    s1, s2, s3 = (float(v) for v in s)
    a, b = 0.5 * (s1 - s2), 0.5 * (s1 + s2)
    M = max(s3 * u + abs(a) * (1 - u) + abs(b) * (1 + u) for u in (-1.0, 1.0))

    def parts(u):
        za, zb = a * (1 - u), b * (1 + u)
        e = math.exp(s3 * u + abs(za) + abs(zb) - M)
        return e, special.ive(0, za), special.ive(0, zb), special.ive(1, za), special.ive(1, zb)

    def g(u, k):
        e, i0a, i0b, i1a, i1b = parts(u)
        if k == 0:
            return 0.5 * e * i0a * i0b
        if k == 1:
            return 0.5 * e * (i1a * 0.5 * (1 - u) * i0b + i0a * i1b * 0.5 * (1 + u))
        if k == 2:
            return 0.5 * e * (-i1a * 0.5 * (1 - u) * i0b + i0a * i1b * 0.5 * (1 + u))
        return 0.5 * e * u * i0a * i0b

    return [integrate.quad(g, -1, 1, args=(k,), epsabs=0, epsrel=1e-13, limit=200)[0]
            for k in range(1 + 3 * order)]


def mf_dlogc(s) -> np.ndarray:
    """grad log c(s): the first moments d_i of the matrix Fisher density."""
    c, d1, d2, d3 = _kunze(s, 1)
    return np.array([d1, d2, d3]) / c


def mf_M2S(d, s0=(0.0, 0.0, 0.0)) -> np.ndarray:
    """pdf_MF_M2S(d, s0): s with grad log c(s) = d."""
    d = np.asarray(d, float)
    sol = optimize.root(lambda s: mf_dlogc(s) - d, np.asarray(s0, float), method='hybr',
                        options=dict(xtol=1e-14, maxfev=2000))
    return sol.x


# ----------------------------------------------------------- get_stat -----
def _fit(ER, Ex, Varx, m_vR, nd):
    """The part of get_stat after the raw moments (pendulum.m:561-592).
    m_vR(U, s, V) returns (EvR, EvRvR, ExvR)."""
    U, D, V = psvd(ER)
    s = mf_M2S(np.diag(D), [0.0, 0.0, 0.0])
    S = np.diag(s)
    EvR, EvRvR, ExvR = m_vR(U, s, V)
    covxvR = ExvR - np.outer(Ex, EvR)
    covvRvR = EvRvR - np.outer(EvR, EvR)
    P = covxvR @ np.linalg.inv(covvRvR)
    Miu = Ex - P @ EvR
    Sigma = Varx - P @ covxvR.T + P @ (np.trace(S) * np.eye(3) - S) @ P.T
    return dict(ER=ER, Ex=Ex, Varx=Varx, EvR=EvR, ExvR=ExvR, EvRvR=EvRvR, U=U, S=S, V=V, P=P,
                Miu=Miu, Sigma=Sigma)


def vR_of(R, U, s, V):
    """vR of pendulum.m:569-572 from Q = U^T R V: (..., 3)."""
    Q = np.einsum('ki,...kl,lj->...ij', U, R, V)
    return np.stack([s[1] * Q[..., 2, 1] - s[2] * Q[..., 1, 2],
                     s[2] * Q[..., 0, 2] - s[0] * Q[..., 2, 0],
                     s[0] * Q[..., 1, 0] - s[1] * Q[..., 0, 1]], -1)


def get_stat_grid(f: np.ndarray, L: float) -> dict:
    """get_stat of pendulum.m:547-594 / pendulum_reduced_hybrid.m:304-351 on the
    grid density f(a, b, c, x...) (FP64, the reference's grid sums)."""
    B = f.shape[0] // 2
    nd = f.ndim - 3
    Bx = f.shape[3] // 2
    c0 = (L / (2 * Bx)) ** nd
    R = so3.rotation_grid(B)
    w = so3.quad_weights(B)
    x = omega_grid(Bx, L, nd)
    ax = tuple(range(3, 3 + nd))
    fR = f.sum(axis=ax) * c0
    ER = np.einsum('abcij,b,abc->ij', R, w, fR)
    fx = np.einsum('b,abc...->...', w, f)
    xf, fxf = x.reshape(nd, -1), fx.reshape(-1)
    Ex = xf @ fxf * c0
    Varx = (xf * fxf) @ xf.T * c0 - np.outer(Ex, Ex)

    def m_vR(U, s, V):
        vR = vR_of(R, U, s, V)
        EvR = np.einsum('abci,b,abc->i', vR, w, fR)
        EvRvR = np.einsum('abci,abcj,b,abc->ij', vR, vR, w, fR)
        g = np.einsum('abcj,b,abc...->j...', vR, w, f).reshape(3, -1)
        ExvR = xf @ g.T * c0
        return EvR, EvRvR, ExvR

    out = _fit(ER, Ex, Varx, m_vR, nd)
    out['fx'] = fx
    return out


def raw_moments_grid(f: np.ndarray, L: float) -> dict:
    """mass, E[R], E[R (x) R], E[x], E[x x^T], E[x R] as grid sums (the inputs of _fit)."""
    B = f.shape[0] // 2
    nd = f.ndim - 3
    Bx = f.shape[3] // 2
    c0 = (L / (2 * Bx)) ** nd
    R = so3.rotation_grid(B)
    w = so3.quad_weights(B)
    x = omega_grid(Bx, L, nd)
    fw = f * w.reshape((1, -1, 1) + (1,) * nd)
    ax = tuple(range(3, 3 + nd))
    fwR = fw.sum(axis=ax)                                          # (2B, 2B, 2B)
    fwx = fw.sum(axis=(0, 1, 2))                                   # omega grid
    gR = np.einsum('abckl,abc...->kl...', R, fw).reshape(9, -1)    # (9, omega)
    xf, fxf = x.reshape(nd, -1), fwx.reshape(-1)
    return dict(mass=c0 * fwR.sum(),
                ER=c0 * np.einsum('abcij,abc->ij', R, fwR),
                ERR=c0 * np.einsum('abcij,abckl,abc->ijkl', R, R, fwR),
                Ex=c0 * xf @ fxf,
                Exx=c0 * (xf * fxf) @ xf.T,
                ExR=c0 * (xf @ gR.T).reshape(nd, 3, 3))


# ------------------------------------------------- coefficient moments ----
BASIS = [(l, m, n) for l in range(3) for m in range(-l, l + 1) for n in range(-l, l + 1)]


def expansion_tables():
    """a^h_{lmn} (h = sum a conj(D^l_mn), l <= 2) for h = R_kq (9) and R_kq R_k'q' (81),
    computed by exact quadrature on the B = 3 grid: a = (2l+1) sum_g w h D^l_mn."""
    B, lmax = 3, 2
    R = so3.rotation_grid(B)
    w = so3.quad_weights(B)
    d = so3.wigner_d_table(B)
    al = np.pi * np.arange(2 * B) / B
    W = np.broadcast_to(w[None, :, None], (2 * B,) * 3)
    D = np.stack([np.exp(-1j * m * al)[:, None, None] * d[m + lmax, n + lmax, l][None, :, None]
                  * np.exp(-1j * n * al)[None, None, :] for (l, m, n) in BASIS], -1)   # D^l_mn(g)
    scale = np.array([2 * l + 1 for (l, _, _) in BASIS])
    hR = R.reshape((2 * B,) * 3 + (9,))
    aR = np.einsum('abc,abch,abct->ht', W, hR, D) * scale
    hRR = np.einsum('abci,abcj->abcij', hR, hR).reshape((2 * B,) * 3 + (81,))
    aRR = np.einsum('abc,abch,abct->ht', W, hRR, D) * scale
    return aR, aRR


def moments_from_coeffs(F: np.ndarray, L: float) -> dict:
    """The raw moments of raw_moments_grid from F (full layout, lmax >= 2)."""
    lmax = F.shape[2] - 1
    nd = F.ndim - 3
    N = F.shape[3]
    c0 = (L / N) ** nd
    aR, aRR = expansion_tables()
    z = (0,) * nd
    F0 = np.array([F[m + lmax, n + lmax, l][z] for (l, m, n) in BASIS])
    t = np.arange(N)
    xt = -L / 2 + L * t / N
    E = np.exp(-2j * np.pi * np.outer(t, t) / N)
    xi, xi2 = E @ xt, E @ (xt * xt)

    def axis(row, i):
        idx = [0] * nd
        out = []
        for q in range(N):
            idx[i] = q
            out.append(row[tuple(idx)])
        return np.array(out)

    r000 = F[lmax, lmax, 0]
    Ex = np.array([c0 / N * np.sum(axis(r000, i) * np.conj(xi)) for i in range(nd)])
    Exx = np.zeros((nd, nd), complex)
    for i in range(nd):
        Exx[i, i] = c0 / N * np.sum(axis(r000, i) * np.conj(xi2))
        for j in range(i + 1, nd):
            idx = [slice(0, 1)] * nd
            idx[i] = slice(None)
            idx[j] = slice(None)
            plane = r000[tuple(idx)].reshape(N, N)
            Exx[i, j] = Exx[j, i] = c0 / N ** 2 * np.einsum('qr,q,r->', plane, np.conj(xi), np.conj(xi))
    ExR = np.zeros((nd, 9), complex)
    for i in range(nd):
        ax = np.array([axis(F[m + lmax, n + lmax, l], i) if l <= 1 else np.zeros(N)
                       for (l, m, n) in BASIS])                       # (35, N)
        ExR[i] = c0 / N * (aR @ (ax @ np.conj(xi)))
    return dict(mass=float(np.real(c0 * F0[0])), ER=np.real(c0 * aR @ F0).reshape(3, 3),
                ERR=np.real(c0 * aRR @ F0).reshape(3, 3, 3, 3), Ex=np.real(Ex), Exx=np.real(Exx),
                ExR=np.real(ExR).reshape(nd, 3, 3))


def fit_from_moments(mo: dict, nd: int) -> dict:
    """get_stat's outputs from the raw moments: vR is linear in R, so
    E[vR] and E[vR vR^T] follow from E[R] and E[R (x) R], E[x vR^T] from E[x R]."""
    ER, Ex, Exx, ERR, ExR = (np.asarray(mo[k]) for k in ('ER', 'Ex', 'Exx', 'ERR', 'ExR'))
    Varx = Exx - np.outer(Ex, Ex)

    def m_vR(U, s, V):
        # vR_j = sum_kq C[j, k, q] R_kq with Q = U^T R V
        C = np.zeros((3, 3, 3))
        terms = [((2, 1), s[1], (1, 2), s[2]), ((0, 2), s[2], (2, 0), s[0]), ((1, 0), s[0], (0, 1), s[1])]
        for j, ((a1, b1), c1, (a2, b2), c2) in enumerate(terms):
            C[j] += c1 * np.outer(U[:, a1], V[:, b1]) - c2 * np.outer(U[:, a2], V[:, b2])
        Cf = C.reshape(3, 9)
        EvR = Cf @ ER.reshape(9)
        EvRvR = Cf @ ERR.reshape(9, 9) @ Cf.T
        ExvR = ExR.reshape(nd, 9) @ Cf.T
        return EvR, EvRvR, ExvR

    return _fit(ER, Ex, Varx, m_vR, nd)

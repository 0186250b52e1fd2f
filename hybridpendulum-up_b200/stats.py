"""Per-step statistics get_stat (propagation/pendulum.m:547-594 and
pendulum_reduced_hybrid.m:304-351) on top of the library's coefficient-space
moments (``hp_moments`` / ``hp_state_moments``).

The GPU returns the raw moments E[R], E[R (x) R], E[x], E[x x^T], E[x R]; the
fit below is the small host computation of the reference:
  * proper SVD of E[R] ('matrix Fisher/psvd.m');
  * matrix-Fisher parameters s from the first moments, i.e. the root of
    grad log c(s) = d ('matrix Fisher/pdf_MF_M2S.m', a damped Newton
    iteration here, on the normalising constant of 'pdf_MF_normal.m:38');
  * E[vR], E[vR vR^T], E[x vR^T] (vR is linear in R, pendulum.m:569-579) and
    the Gaussian part P, Miu, Sigma (pendulum.m:581-587).
"""
from __future__ import annotations

import math

import numpy as np
from scipy import integrate, special

__all__ = ['psvd', 'mf_first_moments', 'mf_parameters', 'get_stat']


def psvd(F: np.ndarray):
    """F = U S V^T with U, V rotations (psvd.m:9-13)."""
    U, s, Vh = np.linalg.svd(np.asarray(F, float))
    V = Vh.T
    dU, dV = np.linalg.det(U), np.linalg.det(V)
    S = np.diag(s * np.array([1.0, 1.0, dU * dV]))
    return U @ np.diag([1.0, 1.0, dU]), S, V @ np.diag([1.0, 1.0, dV])


def _integrals(s):
    """c(s) and dc/ds_i up to one common positive factor (Kunze's integral of
    pdf_MF_normal.m with exponentially scaled Bessel functions)."""
    s1, s2, s3 = (float(v) for v in s)
    a, b = 0.5 * (s1 - s2), 0.5 * (s1 + s2)
    shift = max(s3 * u + abs(a) * (1 - u) + abs(b) * (1 + u) for u in (-1.0, 1.0))

    def integrand(u, k):
        za, zb = a * (1 - u), b * (1 + u)
        e = 0.5 * math.exp(s3 * u + abs(za) + abs(zb) - shift)
        i0a, i0b = special.ive(0, za), special.ive(0, zb)
        if k == 0:
            return e * i0a * i0b
        if k == 3:
            return e * u * i0a * i0b
        i1a, i1b = special.ive(1, za), special.ive(1, zb)
        sa = -1.0 if k == 2 else 1.0
        return e * (sa * i1a * 0.5 * (1 - u) * i0b + i0a * i1b * 0.5 * (1 + u))

    return [integrate.quad(integrand, -1.0, 1.0, args=(k,), epsabs=0.0, epsrel=1e-13, limit=200)[0]
            for k in range(4)]


def mf_first_moments(s) -> np.ndarray:
    """d = grad log c(s): diag(E[Q]) of the matrix Fisher density with proper
    singular values s."""
    c, *dc = _integrals(s)
    return np.array(dc) / c


def mf_parameters(d, s0=(0.0, 0.0, 0.0), tol=1e-12, max_iter=100) -> np.ndarray:
    """s with grad log c(s) = d (pdf_MF_M2S.m): Newton steps on the residual
    with a finite-difference Jacobian and step halving until the residual drops."""
    d = np.asarray(d, float)
    s = np.asarray(s0, float).copy()
    r = mf_first_moments(s) - d
    for _ in range(max_iter):
        if np.max(np.abs(r)) < tol:
            break
        J = np.zeros((3, 3))
        for j in range(3):
            h = 1e-6 * max(1.0, abs(s[j]))
            e = np.zeros(3)
            e[j] = h
            J[:, j] = (mf_first_moments(s + e) - mf_first_moments(s - e)) / (2 * h)
        step = -np.linalg.solve(J, r)
        lam = 1.0
        while True:
            s_new = s + lam * step
            r_new = mf_first_moments(s_new) - d
            if np.linalg.norm(r_new) < (1 - 1e-4 * lam) * np.linalg.norm(r) or lam < 1e-6:
                break
            lam *= 0.5
        s, r = s_new, r_new
    return s


def get_stat(moments: dict) -> dict:
    """get_stat's outputs (ER, Ex, Varx, EvR, ExvR, EvRvR, U, S, V, P, Miu,
    Sigma, and fx when present) from ``Plan.moments`` / ``State.moments``."""
    ER, Ex, Exx = moments['ER'], moments['Ex'], moments['Exx']
    nd = len(Ex)
    Varx = Exx - np.outer(Ex, Ex)
    U, D, V = psvd(ER)
    s = mf_parameters(np.diag(D))
    S = np.diag(s)
    # vR_j = sum_kq C[j, k, q] R_kq for Q = U^T R V (pendulum.m:569-572)
    C = np.zeros((3, 3, 3))
    for j, (a1, b1, c1, a2, b2, c2) in enumerate([(2, 1, s[1], 1, 2, s[2]), (0, 2, s[2], 2, 0, s[0]),
                                                   (1, 0, s[0], 0, 1, s[1])]):
        C[j] = c1 * np.outer(U[:, a1], V[:, b1]) - c2 * np.outer(U[:, a2], V[:, b2])
    Cf = C.reshape(3, 9)
    EvR = Cf @ ER.reshape(9)
    EvRvR = Cf @ moments['ERR'].reshape(9, 9) @ Cf.T
    ExvR = moments['ExR'].reshape(nd, 9) @ Cf.T
    covxvR = ExvR - np.outer(Ex, EvR)
    covvRvR = EvRvR - np.outer(EvR, EvR)
    P = covxvR @ np.linalg.inv(covvRvR)
    Miu = Ex - P @ EvR
    Sigma = Varx - P @ covxvR.T + P @ (np.trace(S) * np.eye(3) - S) @ P.T
    out = dict(ER=ER, Ex=Ex, Varx=Varx, EvR=EvR, ExvR=ExvR, EvRvR=EvRvR, U=U, S=S, V=V, P=P, Miu=Miu,
               Sigma=Sigma)
    if 'fx' in moments:
        out['fx'] = moments['fx']
    return out

"""FP64 CPU restatement of the reference's SO(3) harmonic analysis.

TEST INFRASTRUCTURE ONLY.  Nothing in the product path imports this module:
only ``tests/``, ``__graft_entry__.smoke()`` and the ``cpu_baseline`` /
``--impl reference`` legs of ``bench.py`` may use it, and only as the checker.

Parity status: the reference is MATLAB code with no tests, fixtures or golden
vectors, and neither MATLAB nor Octave exists on the build or GPU machines, so
this restatement cannot be compared with outputs of the reference itself
("parity unpinned" against reference runs).  It is pinned instead against the
closed forms the reference itself ships beside its recursions
(``Wigner_d.m:7-9`` Jacobi-polynomial branch, ``getu.m:118-130`` element-wise
branch), against ``fftSO3_prod``'s own grid-product cross-check
(``fftSO3_prod.m:50``) and against exact identities (orthogonality, round
trips, Hermitian symmetry); see ``tests/test_oracle_so3.py``.

Array conventions follow the MATLAB code exactly (0-based here):
  d[m+lmax, n+lmax, l, j]      Wigner-d at beta_j            (Wigner_d.m)
  F[m+lmax, n+lmax, l, *x]     Fourier coefficients          (fftSO3R.m:98-106)
  f[a, j, c, *x]               samples at (alpha_a, beta_j, gamma_c, x)
  u[m+lmax, n+lmax, l, i]      Lie-derivative matrices       (getu.m:132-163)
"""
from __future__ import annotations

import math
from functools import lru_cache

import numpy as np
import scipy.fft as sfft


# ---------------------------------------------------------------- grids ----
def so3_grid(B: int):
    """Euler-angle grid of the reference (fftSO3R.m:26-28): alpha_a = pi a/B,
    beta_j = pi (2j+1)/(4B), gamma_c = pi c/B for a, j, c in [0, 2B)."""
    k = np.arange(2 * B, dtype=np.float64)
    return np.pi / B * k, np.pi / (4 * B) * (2 * k + 1), np.pi / B * k


def quad_weights(B: int) -> np.ndarray:
    """Quadrature weights (fftSO3R.m:62-66, pendulum.m:101-105):
    w_j = 1/(4B^3) sin(beta_j) sum_{k<B} sin((2k+1) beta_j)/(2k+1)."""
    _, beta, _ = so3_grid(B)
    k = np.arange(B, dtype=np.float64)
    return np.array([1.0 / (4 * B ** 3) * np.sin(b) *
                     np.sum(np.sin((2 * k + 1) * b) / (2 * k + 1)) for b in beta])


def rotation_grid(B: int) -> np.ndarray:
    """R[a, j, c] = Rz(alpha_a) Ry(beta_j) Rz(gamma_c), shape (2B,2B,2B,3,3)
    (fftSO3R.m:30-47)."""
    al, be, ga = so3_grid(B)

    def rz(t):
        c, s = np.cos(t), np.sin(t)
        z, o = np.zeros_like(t), np.ones_like(t)
        return np.stack([np.stack([c, -s, z], -1), np.stack([s, c, z], -1),
                         np.stack([z, z, o], -1)], -2)

    def ry(t):
        c, s = np.cos(t), np.sin(t)
        z, o = np.zeros_like(t), np.ones_like(t)
        return np.stack([np.stack([c, z, s], -1), np.stack([z, o, z], -1),
                         np.stack([-s, z, c], -1)], -2)

    Ra, Rb, Rg = rz(al), ry(be), rz(ga)
    return np.einsum('aij,bjk,ckl->abcil', Ra, Rb, Rg)


# ------------------------------------------------------------ Wigner-d ----
def _symm(d, l, lmax):
    """Symmetry fill of Wigner_d.m:50-63 (in place), vectorised over beta."""
    for m in range(1, l + 1):
        for n in range(-m + 1, m + 1):
            d[m + lmax, n + lmax, l] = d[-n + lmax, -m + lmax, l]
    for m in range(-l, l):
        for n in range(m + 1, l + 1):
            d[m + lmax, n + lmax, l] = d[n + lmax, m + lmax, l] * (-1.0) ** (m - n)


def wigner_d(beta, lmax: int) -> np.ndarray:
    """d^l_{mn}(beta) for l <= lmax by the reference's three-term recursion in l
    (Wigner_d.m:11-44) plus symmetry fill (Wigner_d.m:50-63).

    ``beta`` may be a scalar or a 1-D array; the result has shape
    (2lmax+1, 2lmax+1, lmax+1[, nbeta])."""
    scalar = np.ndim(beta) == 0
    beta = np.atleast_1d(np.asarray(beta, dtype=np.float64))
    cb, cb2, sb2 = np.cos(beta), np.cos(beta / 2), np.sin(beta / 2)
    L = 2 * lmax + 1
    d = np.zeros((L, L, lmax + 1, beta.size))
    d[lmax, lmax, 0] = 1.0
    if lmax >= 1:
        d[lmax - 1, lmax - 1, 1] = cb2 ** 2
        d[lmax, lmax - 1, 1] = -math.sqrt(2) * cb2 * sb2
        d[lmax, lmax, 1] = cb
        d[lmax + 1, lmax - 1, 1] = sb2 ** 2
        _symm(d, 1, lmax)
    for l in range(2, lmax + 1):
        for n in range(-l, 1):
            for m in range(n, -n + 1):
                if n == -l:
                    c = math.sqrt(float(math.factorial(2 * l)) / float(math.factorial(l + m))
                                  / float(math.factorial(l - m)))
                    v = c * cb2 ** (l - m) * (-sb2) ** (l + m)
                elif n == -l + 1:
                    v = (l * (2 * l - 1) / math.sqrt((l * l - m * m) * (l * l - n * n))
                         * (cb - m * n / (l - 1) / l) * d[m + lmax, n + lmax, l - 1])
                else:
                    v = (l * (2 * l - 1) / math.sqrt((l * l - m * m) * (l * l - n * n))
                         * (cb - m * n / (l - 1) / l) * d[m + lmax, n + lmax, l - 1]
                         - math.sqrt(((l - 1) ** 2 - m * m) * ((l - 1) ** 2 - n * n))
                         / math.sqrt((l * l - m * m) * (l * l - n * n))
                         * l / (l - 1) * d[m + lmax, n + lmax, l - 2])
                d[m + lmax, n + lmax, l] = v
        _symm(d, l, lmax)
    return d[..., 0] if scalar else d


def wigner_d_closed(beta: float, l: int, m: int, n: int) -> float:
    """Closed form of Wigner_d.m:7-9:
    sqrt((l+n)!(l-n)!/((l+m)!(l-m)!)) sin(b/2)^(n-m) cos(b/2)^(n+m) P_{l-n}^{(n-m, n+m)}(cos b),
    evaluated with an exact-coefficient Jacobi polynomial (valid for any sign of
    the Jacobi parameters, as MATLAB's symbolic jacobiP is)."""
    from fractions import Fraction
    a, b_, k = n - m, n + m, l - n
    x = math.cos(beta)
    # P_k^{(a,b)}(x) = sum_s C(k+a, k-s) C(k+b, s) ((x-1)/2)^s ((x+1)/2)^(k-s),
    # with generalised binomials C(r, j) = r (r-1) ... (r-j+1) / j!.
    def gbin(r, j):
        if j < 0:
            return Fraction(0)
        num = Fraction(1)
        for t in range(j):
            num *= (r - t)
        return num / math.factorial(j)
    P = 0.0
    for s in range(0, k + 1):
        coef = gbin(k + a, k - s) * gbin(k + b_, s)
        P += float(coef) * ((x - 1) / 2) ** s * ((x + 1) / 2) ** (k - s)
    pref = math.sqrt(math.factorial(l + n) * math.factorial(l - n)
                     / (math.factorial(l + m) * math.factorial(l - m)))
    return pref * math.sin(beta / 2) ** (n - m) * math.cos(beta / 2) ** (n + m) * P


@lru_cache(maxsize=16)
def wigner_d_table(B: int) -> np.ndarray:
    """d[m+lmax, n+lmax, l, j] = d^l_{mn}(beta_j) on the grid (fftSO3R.m:68-73)."""
    _, beta, _ = so3_grid(B)
    d = wigner_d(beta, B - 1)
    d.setflags(write=False)
    return d


# ------------------------------------------------------------------ getu ----
def getu(lmax: int) -> np.ndarray:
    """Complex-harmonic Lie-derivative matrices u[., ., l, i] (getu.m:132-163):
    F^l[E_i f] = F^l[f] (u^l_i)^T."""
    L = 2 * lmax + 1
    u = np.zeros((L, L, lmax + 1, 3), dtype=np.complex128)
    for l in range(lmax + 1):
        for n in range(-l, l + 1):
            if n > -l:
                u[n + lmax - 1, n + lmax, l, 0] = -0.5j * math.sqrt((l + n) * (l - n + 1))
                u[n + lmax - 1, n + lmax, l, 1] = 0.5 * math.sqrt((l + n) * (l - n + 1))
            if n < l:
                u[n + lmax + 1, n + lmax, l, 0] = -0.5j * math.sqrt((l - n) * (l + n + 1))
                u[n + lmax + 1, n + lmax, l, 1] = -0.5 * math.sqrt((l - n) * (l + n + 1))
        for m in range(-l, l + 1):
            u[m + lmax, m + lmax, l, 2] = -1j * m
    return u


def getu_element(l: int, m: int, n: int, ei: int) -> complex:
    """Element-wise branch of getu.m:118-130 (an independent statement of the
    same matrices, used to pin ``getu``)."""
    if ei == 1:
        if m - 1 == n:
            return -0.5j * math.sqrt((l - n) * (l + n + 1))
        if m + 1 == n:
            return 0.5j * math.sqrt((1 + n) * (l - n + 1))
        return 0.0
    if ei == 2:
        if m - 1 == n:
            return -0.5 * math.sqrt((l - n) * (l + n + 1))
        if m + 1 == n:
            return 0.5 * math.sqrt((1 + n) * (l - n + 1))
        return 0.0
    return -1j * m if m == n else 0.0


# ------------------------------------------------------- Clebsch-Gordan ----
@lru_cache(maxsize=4096)
def clebsch_gordan(l1: int, l2: int) -> np.ndarray:
    """Dense CG matrix of clebsch_gordan.m:1-43: column l^2-(l2-l1)^2+l+m,
    row (l1+m1)(2l2+1)+l2+m2; each (l, m) column from a tridiagonal solve with
    the last coefficient positive."""
    D = (2 * l1 + 1) * (2 * l2 + 1)
    CG = np.zeros((D, D))
    for l in range(abs(l1 - l2), l1 + l2 + 1):
        for m in range(-l, l + 1):
            m1 = np.arange((m - l1 - l2 + abs(l1 - l2 + m)) // 2,
                           (m + l1 + l2 - abs(l1 - l2 - m)) // 2 + 1)
            m2 = m - m1
            nnz = m1.size
            A = np.zeros((nnz, nnz))
            for k in range(nnz):
                A[k, k] = l1 * (l1 + 1) + l2 * (l2 + 1) + 2 * m1[k] * m2[k] - l * (l + 1)
                if k > 0:
                    A[k - 1, k] = (math.sqrt(l1 * (l1 + 1) - m1[k - 1] * m1[k])
                                   * math.sqrt(l2 * (l2 + 1) - m2[k - 1] * m2[k]))
            A = A + A.T - np.diag(np.diag(A))
            if nnz == 1:
                C = np.ones(1)
            else:
                rhs = np.zeros(nnz - 1)
                rhs[-1] = -A[nnz - 2, nnz - 1]
                CinCn = np.linalg.solve(A[:nnz - 1, :nnz - 1], rhs)
                Cn = math.sqrt(1.0 / (1.0 + np.sum(CinCn ** 2)))
                C = np.concatenate([CinCn * Cn, [Cn]])
            col = l * l - (l2 - l1) ** 2 + l + m
            for k in range(nnz):
                CG[(l1 + m1[k]) * (2 * l2 + 1) + l2 + m2[k], col] = C[k]
    CG.setflags(write=False)
    return CG


def cg_coeff(l1: int, m1: int, l2: int, m2: int, l: int, m: int) -> float:
    """<l1 m1; l2 m2 | l m> read from the reference's CG matrix."""
    if m1 + m2 != m or abs(m1) > l1 or abs(m2) > l2 or not (abs(l1 - l2) <= l <= l1 + l2):
        return 0.0
    CG = clebsch_gordan(l1, l2)
    return float(CG[(l1 + m1) * (2 * l2 + 1) + l2 + m2, l * l - (l2 - l1) ** 2 + l + m])


# ----------------------------------------------------------- transforms ----
def fftSO3R_forward(f: np.ndarray, B: int | None = None) -> np.ndarray:
    """Forward transform of fftSO3R.m:89-106 for samples f[a, j, c, *x]
    (real or complex): FFT over (alpha, gamma) and every x axis, fftshift + flip
    on alpha and gamma, then the weighted beta-contraction with d.
    Returns F[m+lmax, n+lmax, l, *x] (zero outside |m|,|n| <= l)."""
    B = f.shape[0] // 2 if B is None else B
    lmax = B - 1
    d, w = wigner_d_table(B), quad_weights(B)
    axes = (0, 2) + tuple(range(3, f.ndim))
    F1 = sfft.fftn(f, axes=axes)
    F1 = sfft.fftshift(F1, axes=(0, 2))
    F1 = np.flip(F1, axis=(0, 2))
    xs = f.shape[3:]
    F = np.zeros((2 * lmax + 1, 2 * lmax + 1, lmax + 1) + xs, dtype=np.complex128)
    F1 = F1[:2 * lmax + 1, :, :2 * lmax + 1]                  # (m, j, n, *x)
    for l in range(lmax + 1):
        sl = slice(lmax - l, lmax + l + 1)
        dw = d[sl, sl, l, :] * w                               # (m, n, j)
        F[sl, sl, l] = np.einsum('mnj,mjn...->mn...', dw, F1[sl, :, sl])
    return F


def ifftSO3R_backward(F: np.ndarray, real: bool = True) -> np.ndarray:
    """Backward transform of ifftSO3R.m:16-37 / pendulum.m:284-304:
    F1[m, k, n, x] = sum_{l >= max|m|,|n|} (2l+1) F^l_{mn}[x] d^l_{mn}(beta_k),
    zero-pad to 2B, ifftshift + flip, inverse FFT over (alpha, gamma, x) times
    (2B)^2.  ``real=True`` returns the real part (the 'symmetric' option of
    pendulum.m:303, exact for a Hermitian-symmetric F)."""
    lmax = F.shape[2] - 1
    B = lmax + 1
    d = wigner_d_table(B)
    xs = F.shape[3:]
    N = 2 * B
    F1 = np.zeros((N, N, N) + xs, dtype=np.complex128)
    l2p1 = 2 * np.arange(lmax + 1) + 1.0
    # sum over l of (2l+1) F d, vectorised: entries with l < max(|m|,|n|) are 0 in F and d
    F1[:2 * lmax + 1, :, :2 * lmax + 1] = np.einsum(
        'mnl,mnl...,mnlk->mkn...', np.broadcast_to(l2p1, F.shape[:3]), F, d)
    F1 = sfft.ifftshift(F1, axes=(0, 2))
    F1 = np.flip(F1, axis=(0, 2))
    axes = (0, 2) + tuple(range(3, F1.ndim))
    f = sfft.ifftn(F1, axes=axes) * N ** 2
    return f.real if real else f


def fftSO3_forward(f: np.ndarray) -> np.ndarray:
    """SO(3)-only forward transform (no x axes), as used for MR
    (pendulum.m:176-192) and fftSO3_prod.m:212-227."""
    return fftSO3R_forward(f)


def fftSO3_prod(F: np.ndarray, G: np.ndarray) -> np.ndarray:
    """Complex-harmonic product rule of fftSO3_prod.m:247-264:
    FG^l = sum_{l1,l2} (2l1+1)(2l2+1)/(2l+1) [CG^T kron(F^{l1}, G^{l2}) CG]_{l-block},
    truncated to l <= lmax.  F, G: (2lmax+1, 2lmax+1, lmax+1)."""
    lmax = F.shape[2] - 1
    FG = np.zeros_like(F, dtype=np.complex128)
    for l1 in range(lmax + 1):
        for l2 in range(lmax + 1):
            i1 = slice(lmax - l1, lmax + l1 + 1)
            i2 = slice(lmax - l2, lmax + l2 + 1)
            CG = clebsch_gordan(l1, l2)
            A = CG.T @ np.kron(F[i1, i1, l1], G[i2, i2, l2]) @ CG
            A = A * (2 * l1 + 1) * (2 * l2 + 1)
            for l in range(abs(l1 - l2), min(l1 + l2, lmax) + 1):
                s = l * l - (l1 - l2) ** 2
                iF = slice(lmax - l, lmax + l + 1)
                FG[iF, iF, l] += A[s:s + 2 * l + 1, s:s + 2 * l + 1] / (2 * l + 1)
    return FG


# --------------------------------------------------------------- layouts ----
def n_coeff(lmax: int) -> int:
    """Number of (l, m, n) with |m|,|n| <= l <= lmax (init_Size_F's nR_compact)."""
    return (lmax + 1) * (2 * lmax + 1) * (2 * lmax + 3) // 3

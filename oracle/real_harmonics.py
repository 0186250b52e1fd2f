"""FP64 CPU restatement of the reference's real-harmonic SO(3) transforms.

TEST INFRASTRUCTURE ONLY (see ``oracle/so3.py`` for the rules and the parity
status).  The ``isreal`` branches of ``fftSO3.m`` (forward, lines 61-119),
``ifftSO3.m`` (backward, lines 24-84) and ``getu.m`` (lines 9-107) expand a
real function on SO(3) in real harmonics built from Wigner-d through the table

  Psi(m, n, l, beta)   (fftSO3.m:62-88 / ifftSO3.m:24-50), for n <= 0:
     m = n = 0 :  d^l_00
     m = 0 or n = 0 :  (-1)^(m-n) sqrt(2) d^l_{|m| |n|}
     otherwise :  (-1)^(m-n) d^l_{|m| |n|} + (-1)^m sign(m) d^l_{|m|, -|n|}
  and Psi(m, n) = Psi(m, -n) for n > 0,

so the coefficients F(m, n, l) are real.  Both directions are restated as the
reference computes them: the forward one from the fftshift-ed 2-D FFT S12 of
every beta slice over (alpha, gamma), the backward one through the per-beta
sums S1, F1 and the cos/sin tables of ifftSO3.m:69-83.  These functions are SO(3)
only (no omega axes), the setting of the SO(3)-only models (``gyro_nobias.m``)
and of ``fftSO3_deriv.m``.  Arrays: f[a, j, c] (alpha, beta, gamma), F[m+lmax,
n+lmax, l], u[m+lmax, n+lmax, l, i].
"""
from __future__ import annotations

import math

import numpy as np

from . import so3


def psi_table(B: int) -> np.ndarray:
    """Psi[m+lmax, n+lmax, l, j] of fftSO3.m:62-88."""
    lmax = B - 1
    d = so3.wigner_d_table(B)
    P = np.zeros_like(d)
    for l in range(lmax + 1):
        for m in range(-l, l + 1):
            for n in range(-l, 1):
                am, an = abs(m), abs(n)
                if m == 0 and n == 0:
                    v = d[lmax, lmax, l, :]
                elif m == 0 or n == 0:
                    v = (-1.0) ** (m - n) * math.sqrt(2.0) * d[am + lmax, an + lmax, l, :]
                else:
                    v = ((-1.0) ** (m - n) * d[am + lmax, an + lmax, l, :]
                         + (-1.0) ** m * np.sign(m) * d[am + lmax, -an + lmax, l, :])
                P[m + lmax, n + lmax, l, :] = v
                if n < 0:
                    P[m + lmax, -n + lmax, l, :] = v
    return P


def forward(f: np.ndarray) -> np.ndarray:
    """F = fftSO3(f, B, true) (fftSO3.m:90-118) for real samples f[a, j, c]."""
    B = f.shape[0] // 2
    lmax = B - 1
    w = so3.quad_weights(B)
    Psi = psi_table(B)
    # S12[j, kA, kC] = fftshift(fft2(f(:, j, :))): index B + k <-> frequency k
    S12 = np.fft.fftshift(np.fft.fft2(np.transpose(f, (1, 0, 2)), axes=(1, 2)), axes=(1, 2))
    F = np.zeros((2 * lmax + 1, 2 * lmax + 1, lmax + 1))
    for l in range(lmax + 1):
        for m in range(-l, l + 1):
            for n in range(-l, l + 1):
                smn, sm_n = S12[:, m + B, n + B], S12[:, m + B, -n + B]
                p1 = Psi[-m + lmax, n + lmax, l, :]
                p2 = Psi[m + lmax, n + lmax, l, :]
                if (m >= 0 and n >= 0) or (m < 0 and n < 0):
                    c1, c2 = smn.real, sm_n.real
                    F[m + lmax, n + lmax, l] = np.sum(w * (-0.5 * (c2 - c1) * p1 + 0.5 * (c2 + c1) * p2))
                else:
                    s1, s2 = -smn.imag, -sm_n.imag
                    F[m + lmax, n + lmax, l] = np.sum(w * (-0.5 * (s1 + s2) * p1 + 0.5 * (s1 - s2) * p2))
    return F


def backward(F: np.ndarray) -> np.ndarray:
    """f = ifftSO3(F, true) (ifftSO3.m:24-84): real samples f[a, j, c]."""
    lmax = F.shape[2] - 1
    B = lmax + 1
    N = 2 * B
    Psi = psi_table(B)
    alpha, _, gamma = so3.so3_grid(B)
    l2p1 = 2.0 * np.arange(lmax + 1) + 1.0
    # S1[m, j, n] = sum_l (2l+1) F Psi(m, n), F1[m, j, n] = sum_l (2l+1) F Psi(-m, n)
    S1 = np.einsum('l,mnl,mnlj->mjn', l2p1, F, Psi)
    F1 = np.einsum('l,mnl,mnlj->mjn', l2p1, F, Psi[::-1])
    ms = np.arange(-lmax, lmax + 1)
    same = (np.sign(ms)[:, None] >= 0) == (np.sign(ms)[None, :] >= 0)   # m, n of the same sign class
    f = np.zeros((N, N, N))
    for i in range(N):
        sa, ca = np.sin(ms * alpha[i]), np.cos(ms * alpha[i])
        for c in range(N):
            sg, cg = np.sin(ms * gamma[c]), np.cos(ms * gamma[c])
            T1 = -sa[:, None] * np.where(same, sg[None, :], cg[None, :])
            T2 = ca[:, None] * np.where(same, cg[None, :], sg[None, :])
            f[i, :, c] = np.einsum('mjn,mn->j', F1, T1) + np.einsum('mjn,mn->j', S1, T2)
    return f


def getu_real(lmax: int) -> np.ndarray:
    """Real-harmonic Lie-derivative matrices of getu.m:45-107 (isreal branch)."""
    u = np.zeros((2 * lmax + 1, 2 * lmax + 1, lmax + 1, 3))
    o = lmax
    for l in range(lmax + 1):
        for m in range(-l, l + 1):
            am = abs(m)
            if m >= 2:
                u[m + o, -m + 1 + o, l, 0] = 0.5 * math.sqrt((l + am) * (l - am + 1))
            if m <= -2:
                u[m + o, -m - 1 + o, l, 0] = -0.5 * math.sqrt((l + am) * (l - am + 1))
            if 1 <= m <= l - 1:
                u[m + o, -m - 1 + o, l, 0] = 0.5 * math.sqrt((l - am) * (l + am + 1))
            if -l + 1 <= m <= -1:
                u[m + o, -m + 1 + o, l, 0] = -0.5 * math.sqrt((l - am) * (l + am + 1))
            if m == -1:
                u[-1 + o, o, l, 0] = -1 / math.sqrt(2) * math.sqrt(l * (l + 1))
            if m == 0 and l >= 1:
                u[o, -1 + o, l, 0] = 1 / math.sqrt(2) * math.sqrt(l * (l + 1))
        for m in range(-l, l + 1):
            am = abs(m)
            if m >= 2:
                u[m + o, m - 1 + o, l, 1] = 0.5 * math.sqrt((l + am) * (l - am + 1))
            if m <= -2:
                u[m + o, m + 1 + o, l, 1] = 0.5 * math.sqrt((l + am) * (l - am + 1))
            if 1 <= m <= l - 1:
                u[m + o, m + 1 + o, l, 1] = -0.5 * math.sqrt((l - am) * (l + am + 1))
            if -l + 1 <= m <= -1:
                u[m + o, m - 1 + o, l, 1] = -0.5 * math.sqrt((l - am) * (l + am + 1))
            if m == 1:
                u[1 + o, o, l, 1] = 1 / math.sqrt(2) * math.sqrt(l * (l + 1))
            if m == 0:
                u[o, 1 + o, l, 1] = -1 / math.sqrt(2) * math.sqrt(l * (l + 1))
        for m in range(-l, l + 1):
            if m != 0:
                u[m + o, -m + o, l, 2] = -m
    return u


def deriv(F: np.ndarray, eta) -> np.ndarray:
    """dF^l = sum_i eta_i F^l (u^l_i)^T with the real u (fftSO3_deriv.m:14-25)."""
    lmax = F.shape[2] - 1
    u = getu_real(lmax)
    dF = np.zeros_like(F)
    for l in range(lmax + 1):
        s = slice(lmax - l, lmax + l + 1)
        for i in range(3):
            dF[s, s, l] += eta[i] * F[s, s, l] @ u[s, s, l, i].T
    return dF


def t_matrix(l: int) -> np.ndarray:
    """Real-to-complex basis matrix T^l of fftSO3_prod.m:103-120 (unitary):
    the complex coefficients are F_c^l = (T^l)^H F_r^l T^l."""
    T = np.zeros((2 * l + 1, 2 * l + 1), complex)
    for m in range(-l, l + 1):
        if m < 0:
            T[m + l, m + l] = 1j
            T[m + l, -m + l] = -1j * (-1.0) ** (-m)
        elif m == 0:
            T[l, l] = math.sqrt(2.0)
        else:
            T[m + l, m + l] = (-1.0) ** m
            T[m + l, -m + l] = 1.0
    return T / math.sqrt(2.0)


def prod_literal(F: np.ndarray, G: np.ndarray) -> np.ndarray:
    """FG of fftSO3_prod.m:97-205 (isreal) from real coefficients F, G: the
    real Clebsch-Gordan matrices cg = kron(conj T1, conj T2) CG blkdiag(T)^T and
    A = (2l1+1)(2l2+1) cg^T kron(F^l1, G^l2) conj(cg), l-blocks / (2l+1), real part."""
    lmax = F.shape[2] - 1
    FG = np.zeros(F.shape, complex)
    for l1 in range(lmax + 1):
        for l2 in range(lmax + 1):
            CG = so3.clebsch_gordan(l1, l2)
            Tb = np.zeros((CG.shape[1], CG.shape[1]), complex)
            o = 0
            for l in range(abs(l1 - l2), l1 + l2 + 1):
                Tb[o:o + 2 * l + 1, o:o + 2 * l + 1] = t_matrix(l)
                o += 2 * l + 1
            cg = np.kron(np.conj(t_matrix(l1)), np.conj(t_matrix(l2))) @ CG @ Tb.T
            i1 = slice(lmax - l1, lmax + l1 + 1)
            i2 = slice(lmax - l2, lmax + l2 + 1)
            A = cg.T @ np.kron(F[i1, i1, l1], G[i2, i2, l2]) @ np.conj(cg)
            A = A * (2 * l1 + 1) * (2 * l2 + 1)
            for l in range(abs(l1 - l2), min(l1 + l2, lmax) + 1):
                s = l * l - (l1 - l2) ** 2
                iF = slice(lmax - l, lmax + l + 1)
                FG[iF, iF, l] += A[s:s + 2 * l + 1, s:s + 2 * l + 1] / (2 * l + 1)
    return FG.real

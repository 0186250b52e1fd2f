"""FP64 CPU restatement of the gyro-bias attitude model.

TEST INFRASTRUCTURE ONLY (see ``oracle/so3.py`` for the rules and the parity
status).  The state is (R, x): attitude R in SO(3) and gyro bias x in R^3 on
the periodic grid x_i = -L/2 + L*j/(2Bx) (``propagation/gyro_bias.m:57-66``,
L = 2 there).  ``integrate`` of ``propagation/gyro_bias.m:226-300`` (and the
MEX ``gyrobias_propagate``) advances the coefficients by one Euler step of

  dF = -sum_i temp_i^l (u^l_i)^T                 bias drift      (gyro_bias.m:233-265)
       + sum_ij G1_ij F^l (u^l_i)^T (u^l_j)^T     gyro random walk (gyro_bias.m:268-279)
       + sum_ij G2_ij c_ij F                      bias random walk (gyro_bias.m:281-297)

with temp_i the omega-circular convolution (1/N^3) X_i (*) F of
gyro_bias.m:238-256.  Two forms:

* ``derivative_literal`` restates those lines: the flipped, shifted X sums, the
  page-wise products with u.' and the pi-based multipliers c (the reference
  hard-codes pi = 2 pi / L for its L = 2 grid, so this form takes L = 2);
* ``derivative_fast`` reuses ``pendulum.derivative_fast`` (omega FFTs for the
  drift, any L) with no damping, gyroscopic or gravity term, plus the attitude
  diffusion ``so3_diffusion``.
"""
from __future__ import annotations

import math

import numpy as np

from . import so3
from . import pendulum as pd
from .pendulum import Pendulum, _circ_conv_literal, make_X, omega_grid


def bias_grid(Bx: int, L: float = 2.0) -> np.ndarray:
    """x[:, i, j, k] of gyro_bias.m:57-66 (period L)."""
    return omega_grid(Bx, L, 3)


def so3_diffusion(F: np.ndarray, G1: np.ndarray) -> np.ndarray:
    """sum_ij G1_ij F^l (u^l_i)^T (u^l_j)^T per degree (gyro_bias.m:268-279)."""
    lmax = F.shape[2] - 1
    u = so3.getu(lmax)
    out = np.zeros_like(F)
    for l in range(lmax + 1):
        s = slice(lmax - l, lmax + l + 1)
        blk = np.moveaxis(F[s, s, l], (0, 1), (-2, -1))
        acc = np.zeros_like(blk)
        for i in range(3):
            for j in range(3):
                if G1[i, j] != 0:
                    acc += G1[i, j] * (blk @ u[s, s, l, i].T) @ u[s, s, l, j].T
        out[s, s, l] = np.moveaxis(acc, (-2, -1), (0, 1))
    return out


def derivative_literal(F: np.ndarray, X: np.ndarray, G1: np.ndarray, G2: np.ndarray) -> np.ndarray:
    """dF1 of gyro_bias.m:230-297 (small sizes: the drift is O(nx^2))."""
    lmax = F.shape[2] - 1
    Bx = F.shape[3] // 2
    u = so3.getu(lmax)
    temps = [_circ_conv_literal(X[..., i], F, 3) for i in range(3)]
    dF = np.zeros_like(F)
    for l in range(lmax + 1):
        s = slice(lmax - l, lmax + l + 1)
        for i in range(3):
            blk = np.moveaxis(temps[i][s, s, l], (0, 1), (-2, -1))
            dF[s, s, l] -= np.moveaxis(blk @ u[s, s, l, i].T, (-2, -1), (0, 1))
    dF += so3_diffusion(F, G1)
    kd = np.concatenate([np.arange(Bx), np.arange(-Bx, 0)])
    kf = np.concatenate([np.arange(Bx), [0], np.arange(-Bx + 1, 0)])
    for i in range(3):
        for j in range(3):
            if i == j:
                c = -(math.pi ** 2 * kd ** 2)
                sh = [1] * 6
                sh[3 + i] = 2 * Bx
                c = c.reshape(sh)
            else:
                ci = (math.pi * kf).reshape([1] * (3 + i) + [2 * Bx] + [1] * (2 - i))
                cj = (math.pi * kf).reshape([1] * (3 + j) + [2 * Bx] + [1] * (2 - j))
                c = -ci * cj
            dF = dF + G2[i, j] * F * c
    return dF


def model(B: int, Bx: int, L: float, G2: np.ndarray) -> Pendulum:
    """The pendulum restatement with only the drift and the bias random walk."""
    lmax = B - 1
    x = omega_grid(Bx, L, 3)
    return Pendulum(B=B, Bx=Bx, ndim=3, L=L, X=make_X(x), OJO=None,
                    MR=np.zeros((2 * lmax + 1, 2 * lmax + 1, lmax + 1, 3), np.complex128),
                    b=np.zeros(3), G=np.asarray(G2, float), x=x)


def derivative_fast(F: np.ndarray, L: float, G1: np.ndarray, G2: np.ndarray) -> np.ndarray:
    B, Bx = F.shape[2], F.shape[3] // 2
    return pd.derivative_fast(F, model(B, Bx, L, G2)) + so3_diffusion(F, np.asarray(G1, float))


def propagate(F: np.ndarray, X: np.ndarray, dt: float, G1: np.ndarray, G2: np.ndarray) -> np.ndarray:
    """Fnew = Fold + dt dF1 (gyro_bias.m:299), literal form."""
    return F + dt * derivative_literal(F, X, np.asarray(G1, float), np.asarray(G2, float))

"""FP64 CPU restatement of the reference's hybrid collision operator
(propagation/discrete/mex/sources/pendulum_reduced_collision).

TEST INFRASTRUCTURE ONLY (see oracle/so3.py for the rules; parity unpinned
against reference runs: the reference MEX needs mex.h, cuTENSOR 1.x and
Thrust and cannot be built or run here).

Arrays follow the MEX layouts:
  R       (2B, 2B, 2B, 3, 3) rotations, grid index iR = a + 2B b + 4B^2 c
  x       (2, 2Bx, 2Bx) grid, point index ix = i + 2Bx j
          (3-D Omega: (3, 2Bx, 2Bx, 2Bx), ix = i + 2Bx j + 4Bx^2 k)
  lambda  [ix][k]  (numR fastest), k indexes the colliding attitudes indR
  Omega   [ix][k][ndim]
  fcL, fcL_indx  [ix][k][d] (nD fastest)
  f, df   [ix][iR]  (the density f(a, b, c, i, j) in column-major order)
"""
from __future__ import annotations

import math

import numpy as np


def _rows(R):
    """R as (nR, 3, 3) in grid-index order a + 2B b + 4B^2 c."""
    n = R.shape[0] * R.shape[1] * R.shape[2]
    return np.transpose(R, (2, 1, 0, 3, 4)).reshape(n, 3, 3)


def _xpts(x):
    """x (nd, N, ...) as (nx, nd) in point order i + N j (+ N^2 k)."""
    return x.T.reshape(-1, x.shape[0])


def get_lambda(R, x, d, h, r, theta_t, lambda_max):
    """getLambda (getLambda.cu:8-85, kernels 192-267): switching rate lambda(R, x),
    the colliding attitudes indR (lambda category != 0) and the contact point PC."""
    Rr = _rows(R)
    theta0 = math.asin(d / math.sqrt(h * h + r * r)) - math.asin(r / math.sqrt(h * h + r * r))
    theta = np.arcsin(Rr[:, 0, 2])                                 # asin(R13)
    cat = np.where(theta < theta0 - theta_t, 0, np.where(theta > theta0 + theta_t, 2, 1))
    indR = np.nonzero(cat != 0)[0].astype(np.int32)
    lr3 = h - r * np.tan(theta)
    PC = np.stack([lr3 * Rr[:, 0, 2] + r / np.cos(theta), lr3 * Rr[:, 1, 2], lr3 * Rr[:, 2, 2]], -1)
    lam0 = np.where(cat == 2, lambda_max,
                    lambda_max / 2 * np.sin(math.pi / (2 * theta_t) * (theta - theta0)) + lambda_max / 2)
    lam0 = np.where(cat == 0, 0.0, lam0)[indR]
    X = _xpts(x)
    Rk = Rr[indR]                                                   # (numR, 3, 3)
    # omega = R Omega with Omega = [x1, x2, 0] (2-D).  On a 3-D grid the spin x3
    # R e3 about the pendulum axis adds nothing to (omega x PC)_1 (PC's (2, 3)
    # components are lr3 R e3's), so the contact velocity uses x1, x2 alone.
    om0 = Rk[None, :, 1, 0] * X[:, None, 0] + Rk[None, :, 1, 1] * X[:, None, 1]
    om1 = Rk[None, :, 2, 0] * X[:, None, 0] + Rk[None, :, 2, 1] * X[:, None, 1]
    vC = om0 * PC[indR][None, :, 2] - om1 * PC[indR][None, :, 1]
    lam = np.where(vC < 0.0, 0.0, np.broadcast_to(lam0[None, :], vC.shape))
    return lam, indR, PC


def get_omega_new(R, x, indR, epsilon):
    """getOmega(..., 'new') (getOmega.cu:64-103): post-collision angular velocity
    Omega+ = R^T(w - (1+eps)(w.t) t), w = R [x1, x2, 0], t = (R33, -R23)/|.| in
    the (2, 3) components, first ndim components kept.  For a 3-D grid (no
    reference counterpart) w = R [x1, x2, x3] and Omega+ keeps all three."""
    Rk = _rows(R)[indR]
    X = _xpts(x)
    nd = X.shape[1]
    n = np.sqrt(Rk[:, 1, 2] ** 2 + Rk[:, 2, 2] ** 2)
    t1, t2 = Rk[:, 2, 2] / n, -Rk[:, 1, 2] / n
    w = np.einsum('kij,xj->xki', Rk[:, :, :nd], X)                   # (nx, numR, 3)
    ot = (1.0 + epsilon) * (w[..., 1] * t1 + w[..., 2] * t2)
    w1 = w[..., 1] - ot * t1
    w2 = w[..., 2] - ot * t2
    return np.stack([Rk[None, :, 0, c] * w[..., 0] + Rk[None, :, 1, c] * w1 + Rk[None, :, 2, c] * w2
                     for c in range(nd)], -1)


def get_fcL(x, Omega, lam, Gd, nD):
    """getFcL (getFcL.cu:11-166): for every colliding attitude k and landing point
    ix1, the Gaussian density of landing at x[ix1] from every source point ix2
    (mean Omega+(k, ix2), covariance Gd); keep the nD largest (stable descending
    sort), normalise per source point over the kept taps (times dx^2), then scale
    by lambda(k, ix2) dx^2.  Returns fcL, fcL_indx as [ix1][k][d]."""
    X = _xpts(x)
    nd = X.shape[1]
    nx, numR = Omega.shape[0], Omega.shape[1]
    Gd = np.asarray(Gd, float).reshape(nd, nd, order='F')
    det = np.linalg.det(Gd) if nd == 3 else Gd[0, 0] * Gd[1, 1] - Gd[0, 1] * Gd[1, 0]
    cn = 1 / ((2 * math.pi) ** (nd / 2) * math.sqrt(det))
    inv = (np.linalg.inv(Gd) if nd == 3
           else np.array([[Gd[1, 1], -Gd[0, 1]], [-Gd[1, 0], Gd[0, 0]]]) / det)
    dx2 = (X[1, 0] - X[0, 0]) ** nd
    fcL = np.zeros((nx, numR, nD))
    idx = np.zeros((nx, numR, nD), np.int16)
    for k in range(numR):
        dO = X[:, None, :] - Omega[None, :, k, :]                   # (ix1, ix2, nd)
        q = (inv[0, 0] * dO[..., 0] ** 2 + (inv[0, 1] + inv[1, 0]) * dO[..., 0] * dO[..., 1]
             + inv[1, 1] * dO[..., 1] ** 2)
        if nd == 3:
            q = q + ((inv[0, 2] + inv[2, 0]) * dO[..., 0] * dO[..., 2]
                     + (inv[1, 2] + inv[2, 1]) * dO[..., 1] * dO[..., 2] + inv[2, 2] * dO[..., 2] ** 2)
        fc = np.exp(-0.5 * q) * cn                                  # (ix1, ix2)
        order = np.argsort(-fc, axis=1, kind='stable')[:, :nD]
        vals = np.take_along_axis(fc, order, 1)
        norm = np.zeros(nx)
        np.add.at(norm, order.ravel(), vals.ravel())
        norm *= dx2
        nz = norm[order] > 0          # 0/0 (every kept tap of a source underflowed) -> 0
        vals = np.where(nz, vals / np.where(nz, norm[order], 1.0), 0.0)
        vals = vals * lam[order, k] * dx2
        fcL[:, k, :] = vals
        idx[:, k, :] = order
    return fcL, idx


def propagate_noise(f, lam, indR, fcL, fcL_indx):
    """get_df_noise (propagate.cu:6-121): df(R_k, x) = sum_d fcL[x][k][d] f(R_k, idx)
    - lambda(k, x) f(R_k, x) on the colliding attitudes, zero elsewhere.
    f: [ix][iR] (nx, nR)."""
    df = np.zeros_like(f)
    fk = f[:, indR]                                                 # (nx, numR)
    gather = fk[fcL_indx.astype(np.int64), np.arange(len(indR))[None, :, None]]   # (nx, numR, nD)
    df[:, indR] = np.sum(fcL * gather, axis=2) - lam * fk
    return df

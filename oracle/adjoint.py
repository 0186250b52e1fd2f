"""FP64 reverse mode of the pendulum propagation (test infrastructure only).

The reference has no adjoint; this is the checker for the library's reverse
pass.  It takes the adjoint of ``pendulum.derivative_fast`` term by term
(no weighting identities), so it is independent of the library's
formulation:
  Lie      -sum_i L_i M_i F          ->  -sum_i M_i (lam conj(u_i))
  damping  +b_i D_i M_i F            ->  +b_i M_i conj(D_i) lam
  gyro     -D_i M_{ojo_i} F          ->  -M_{ojo_i} conj(D_i) lam
  gravity  -D_i Grav_i F             ->  -Grav_i^T-conj(conj(D_i) lam)   (taps transposed)
  noise    N . F                     ->  N . lam
with <X, Y> = Re sum conj(X) Y over the full layout, M_i = fftn(x_i ifftn .),
D_i the multiplier 2 pi i kappa / L of pendulum.m:504 along omega axis i.
Gradients of a forward-Euler trajectory follow from
lam_n = lam_{n+1} + dt A^H lam_{n+1} and dL/dtheta = sum_n dt <lam_{n+1}, dA/dtheta F_n>.
"""
from __future__ import annotations

import numpy as np
import scipy.fft as sfft

from . import so3
from .pendulum import (Pendulum, _c_first, _noise_mult, _xaxes, derivative_fast,
                       gravity_taps)


def _cmul(T, c, i, nd):
    sh = [1] * (3 + nd)
    sh[3 + i] = len(c)
    return T * c.reshape(sh)


def _mx(F, xi, nd):
    ax = _xaxes(nd)
    return sfft.fftn(sfft.ifftn(F, axes=ax) * xi, axes=ax)


def _grav_T(lam, MRi):
    """Transpose-conjugate of gravity_fast: out[l1,m1,n1] += conj(w) lam[l,m,n]."""
    lmax = lam.shape[2] - 1
    MR1 = MRi[lmax - 1:lmax + 2, lmax - 1:lmax + 2, 1]
    out = np.zeros_like(lam)
    for (l, m, n, l1, m1, n1, w) in gravity_taps(lmax, MR1):
        out[m1 + lmax, n1 + lmax, l1] += np.conj(w) * lam[m + lmax, n + lmax, l]
    return out


def _grav(F, MRi):
    lmax = F.shape[2] - 1
    MR1 = MRi[lmax - 1:lmax + 2, lmax - 1:lmax + 2, 1]
    out = np.zeros_like(F)
    for (l, m, n, l1, m1, n1, w) in gravity_taps(lmax, MR1):
        out[m + lmax, n + lmax, l] += w * F[m1 + lmax, n1 + lmax, l1]
    return out


def xs_of(P: Pendulum):
    return [sfft.ifftn(P.X[..., i]) for i in range(P.ndim)]


def derivative_adjoint(lam: np.ndarray, P: Pendulum) -> np.ndarray:
    """A^H lam for A = derivative_fast(., P)."""
    lmax, Bx, L, nd = P.lmax, P.Bx, P.L, P.ndim
    u = so3.getu(lmax)
    c = _c_first(Bx, L)
    cc = np.conj(c)
    xs = xs_of(P)
    out = np.zeros_like(lam)
    for i in range(nd):
        t = np.zeros_like(lam)
        for l in range(lmax + 1):
            s = slice(lmax - l, lmax + l + 1)
            blk = np.moveaxis(lam[s, s, l], (0, 1), (-2, -1))
            t[s, s, l] = np.moveaxis(blk @ np.conj(u[s, s, l, i]), (-2, -1), (0, 1))
        out -= _mx(t, xs[i], nd)
    for i in range(nd):
        out += P.b[i] * _mx(_cmul(lam, cc, i, nd), xs[i], nd)
    if nd == 3 and P.OJO is not None:
        for i in range(3):
            ojo = sfft.ifftn(P.OJO[..., i])
            out -= _mx(_cmul(lam, cc, i, nd), ojo, nd)
    for i in range(nd):
        out -= _grav_T(_cmul(lam, cc, i, nd), P.MR[..., i])
    out += lam * _noise_mult(Bx, L, nd, P.G)
    return out


def mirror(lam: np.ndarray, nd: int) -> np.ndarray:
    """C lam: F^l_{mn}[k] -> (-1)^(m-n) conj F^l_{-m,-n}[-k]."""
    D = lam.shape[0]
    lmax = (D - 1) // 2
    r = np.conj(lam[::-1, ::-1])
    for a in range(nd):
        r = np.roll(np.flip(r, 3 + a), 1, axis=3 + a)
    m = np.arange(-lmax, lmax + 1)
    sg = (-1.0) ** (m[:, None] - m[None, :])
    return r * sg.reshape((D, D) + (1,) * (lam.ndim - 2))


def symmetrise(lam: np.ndarray, nd: int) -> np.ndarray:
    return 0.5 * (lam + mirror(lam, nd))


def dot(a, b):
    return float(np.real(np.vdot(a, b)))


def param_terms(F: np.ndarray, P: Pendulum) -> dict:
    """dA/dtheta F for theta = b_i, gyro_i (3-D), gscale_i, G_ij."""
    lmax, Bx, L, nd = P.lmax, P.Bx, P.L, P.ndim
    c = _c_first(Bx, L)
    xs = xs_of(P)
    out = {}
    for i in range(nd):
        out[('b', i)] = _cmul(_mx(F, xs[i], nd), c, i, nd)
    if nd == 3:
        pairs = [(1, 2), (0, 2), (0, 1)]
        for i in range(3):
            j, k = pairs[i]
            out[('gyro', i)] = -_cmul(_mx(F, xs[j] * xs[k], nd), c, i, nd)
    for i in range(nd):
        out[('gscale', i)] = -_cmul(_grav(F, P.MR[..., i]), c, i, nd)
    for i in range(nd):
        for j in range(i, nd):
            E = np.zeros((nd, nd))
            E[i, j] = 1.0
            out[('G', i, j)] = F * _noise_mult(Bx, L, nd, E)
    return out


def euler_adjoint(F0: np.ndarray, lamT: np.ndarray, P: Pendulum, dt: float, nsteps: int,
                  real: bool = True):
    """(lam0, grads) of nsteps Euler steps; grads keyed as in ``param_terms``."""
    traj = [F0]
    for _ in range(nsteps):
        traj.append(traj[-1] + dt * derivative_fast(traj[-1], P))
    lam = symmetrise(lamT, P.ndim) if real else lamT.copy()
    grads = {}
    for n in range(nsteps - 1, -1, -1):
        for k, Y in param_terms(traj[n], P).items():
            grads[k] = grads.get(k, 0.0) + dt * dot(lam, Y)
        lam = lam + dt * derivative_adjoint(lam, P)
    return lam, grads, traj[-1]

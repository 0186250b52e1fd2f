"""Parity at the sizes of the benchmark workloads, against the FP64 oracle.

* Plain FP64 single step, B = 10 on a 16^3 omega grid: fftSO3R -> pendulum
  derivative -> Euler (dt = 1e-3) -> ifftSO3R, each stage against the oracle
  at full size (<= 1e-10 relative L2).
* Plain vs mixed propagation, B = 15 on a 32^3 omega grid, 200 Euler steps:
  at every step the mixed step from the FP64 state is compared with the FP64
  step from the same state (<= 1e-6).  The oracle cannot hold the full state
  (6.6 GB per coefficient array) in the time a test allows, but every term of
  the derivative keeps the order m (``oracle.pendulum.derivative_fast_mgroup``),
  so the one-step map is checked against it at full size on whole m groups
  (m = 0, 7, 14) at steps 0, 100 and 199: FP64 <= 1e-10, mixed <= 1e-6; the
  density at two omega points against the oracle's synthesis of the
  omega-inverse-FFT of the same coefficients.  With HP_TRAJECTORY_TABLE=<path>
  the test writes the per-step table (errors, trajectory separation, l = 0
  mass drift) as JSON.
* Transform stress, B = 32 on a 24^3 omega grid, complex coefficients
  N(0,1)/(2l+1): backward then forward (round trip) for every beta engine of
  the forward transform (FP32 CUDA cores, 3xTF32 and BF16x3 tensor cores),
  the density at two omega points against the oracle's synthesis.
"""
import json
import math
import os

import numpy as np
import pytest
import scipy.fft as sfft

from oracle import pendulum as pd
from oracle import so3

pytestmark = pytest.mark.gpu

TOL64 = 1e-10
TOLMIX = 1e-6


def rel(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return float(np.linalg.norm((a - b).ravel()) / np.linalg.norm(b.ravel()))


def gyro_of(P):
    J = np.diag(P.params['J'])
    return ((J[1] - J[2]) / J[0], (J[2] - J[0]) / J[1], (J[0] - J[1]) / J[2])


def seeded_factors(seed):
    """U, s, V, mu of oracle.pendulum.seeded_density for the same seed."""
    rng = np.random.default_rng(seed)
    U, V = pd.haar_rotation(rng), pd.haar_rotation(rng)
    s = np.sort(rng.uniform(5, 20, 3))[::-1]
    mu = rng.uniform(-1, 1, 3)
    return U, s, V, mu


# ------------------------------------------------- device-side slicing ----
def _full_view(Fdev, B, N):
    """Full MATLAB layout F(m, n, l, i, j, k) (column-major) of a flat device
    tensor as a C-order view [k][j][i][l][n][m]."""
    lmax = B - 1
    D = 2 * lmax + 1
    return Fdev.view(N, N, N, lmax + 1, D, D)


def mgroup_host(Fdev, B, N, m):
    """Rows of order m as the oracle's F[m + lmax] (n, l, i, j, k), on the host."""
    v = _full_view(Fdev, B, N)[..., m + B - 1]              # [k][j][i][l][n]
    return v.permute(4, 3, 2, 1, 0).contiguous().cpu().numpy()


def coeffs_at_point(Fdev, B, N, x):
    """F^l_mn at the omega grid point x = (i, j, k): (1/nx) sum_k F[k] e^{+2 pi i k.x / N}
    (the omega part of ifftn), computed on the device in FP64.  Returns
    (2lmax+1, 2lmax+1, lmax+1) in the oracle layout."""
    import torch
    v = _full_view(Fdev, B, N)
    kk = torch.arange(N, device=Fdev.device, dtype=torch.float64)

    def e(t):
        return torch.exp(2j * math.pi * kk * t / N).to(torch.complex128)

    i, j, k = x
    r = torch.tensordot(e(k), v, dims=([0], [0]))           # [j][i][l][n][m]
    r = torch.tensordot(e(j), r, dims=([0], [0]))
    r = torch.tensordot(e(i), r, dims=([0], [0]))           # [l][n][m]
    return (r / N ** 3).permute(2, 1, 0).contiguous().cpu().numpy()


def density_at_point(fdev, B, N, x):
    """f[a, b, c] at omega point x from a device density [w][c][b][a], w = i + N j + N^2 k."""
    i, j, k = x
    w = i + N * j + N * N * k
    n3 = (2 * B) ** 3
    return fdev[w * n3:(w + 1) * n3].view(2 * B, 2 * B, 2 * B).permute(2, 1, 0).double().cpu().numpy()


# ------------------------------------------------------------ config 1 ----
def test_config1_fp64_single_step_full_size(hp):
    """B = 10, 16^3: every stage of the plain FP64 step against the oracle."""
    B, Bx, dt = 10, 8, 1e-3
    P = pd.pendulum_3d(B, Bx)
    f, _ = pd.seeded_density(B, Bx, 3, P.L, seed=1)
    F_ref = so3.fftSO3R_forward(f)
    plan = hp.get_plan(B, Bx, 3, hp.HP_FP64, hp.HP_REAL)
    F = plan.forward(f)
    assert rel(F, F_ref) < TOL64
    F1_ref = pd.integrate(F_ref, lambda G: pd.derivative_fast(G, P), dt, 'euler')
    F1 = hp.pendulum_propagate(F_ref, P.X, P.OJO, P.MR, P.b, P.G, dt, P.L, hp.getu(B - 1), None, 'euler')
    assert rel(F1, F1_ref) < TOL64
    # the step increment itself, not only the state (dt dF is ~1e-3 of F)
    assert rel(F1 - F_ref, F1_ref - F_ref) < 1e-9
    f1_ref = so3.ifftSO3R_backward(F1_ref, real=True)
    f1 = plan.backward(F1_ref)
    assert rel(f1, f1_ref) < TOL64


# ------------------------------------------------------------ config 2 ----
def test_config2_trajectory_full_size(hp):
    """Per-step error of the mixed step against the FP64 step from the same
    state at every one of 200 steps (<= 1e-6 relative L2 on the new state and
    on the increment), the FP64 step pinned to the oracle on whole m groups at
    steps 0, 100, 199, and the density at two omega points.

    The mixed and FP64 trajectories are also compared, beside an FP64
    trajectory started from a 1e-9 relative perturbation of the same state: at
    dt = 1e-3 the forward-Euler step amplifies the highest omega wavenumbers
    (the drift and gyroscopic operators there have |lambda| dt of order 0.1-1,
    and |1 + i lambda dt| > 1), so any difference between two trajectories
    grows, whatever its origin; the table records both growths."""
    import torch
    B, Bx, dt, nsteps = 15, 16, 1e-3, 200
    N = 2 * Bx
    mgroups = (0, 7, 14)
    checks = (0, 100, 199)
    points = ((16, 16, 16), (12, 19, 17))
    P = pd.pendulum_3d(B, Bx)
    dev = torch.device('cuda', 0)
    nfull = (2 * B - 1) ** 2 * B * N ** 3

    def plan_for(prec):
        pl = hp.Plan(B, Bx, 3, prec, hp.HP_REAL)
        pl.set_model(P.L, P.b, P.G, P.MR, gyro_of(P))
        return pl

    def norm(t):
        return float(torch.linalg.vector_norm(t))

    p64, pmix = plan_for(hp.HP_FP64), plan_for(hp.HP_MIXED)
    s64, spert, smix, sone = hp.State(p64), hp.State(p64), hp.State(pmix), hp.State(pmix)
    U, s, V, mu = seeded_factors(2)
    s64.init_mf_gauss(U, s, V, mu, 0.25 * np.eye(3))
    F64 = torch.empty(nfull, dtype=torch.complex128, device=dev)
    Fprev = torch.empty_like(F64)
    Fone = torch.empty_like(F64)
    Ftr = torch.empty_like(F64)
    s64.store(F64)
    smix.load(F64)
    g = torch.Generator(device=dev).manual_seed(3)
    noise = torch.randn(nfull, dtype=torch.complex128, device=dev, generator=g)
    Ftr.copy_(F64 + 1e-9 * norm(F64) / norm(noise) * noise)
    spert.load(Ftr)                  # the real-density projection keeps the perturbation ~1e-9
    mass0 = s64.mass()
    f64 = torch.empty((2 * B) ** 3 * N ** 3, dtype=torch.float64, device=dev)
    fmx = torch.empty((2 * B) ** 3 * N ** 3, dtype=torch.float32, device=dev)
    table = []
    worst = {'mixed_step_rel_l2': 0.0, 'mixed_increment_rel_l2': 0.0, 'mixed_step_max_rel': 0.0,
             'fp64_step_vs_oracle': 0.0, 'mixed_step_vs_oracle': 0.0, 'density64_vs_oracle': 0.0,
             'density_mixed_vs_fp64': 0.0}
    for k in range(nsteps):
        Fprev.copy_(F64)
        if k in checks:
            before = {m: mgroup_host(F64, B, N, m) for m in mgroups}
        sone.load(F64)
        sone.step(dt, 'euler', 1)
        sone.store(Fone)
        s64.step(dt, 'euler', 1)
        s64.store(F64)
        d = Fone - F64
        row = {'step': k + 1, 'mixed_step_rel_l2': norm(d) / norm(F64),
               'mixed_increment_rel_l2': norm(d) / norm(F64 - Fprev),
               'mixed_step_max_rel': float(d.abs().max() / F64.abs().max())}
        del d
        for key in ('mixed_step_rel_l2', 'mixed_increment_rel_l2', 'mixed_step_max_rel'):
            worst[key] = max(worst[key], row[key])
        assert row['mixed_step_rel_l2'] < TOLMIX and row['mixed_increment_rel_l2'] < TOLMIX, row
        if k in checks:
            for m in mgroups:
                Fm = before[m]
                with sfft.set_workers(os.cpu_count() or 1):
                    ref = Fm + dt * pd.derivative_fast_mgroup(Fm, m, P)
                e64 = rel(mgroup_host(F64, B, N, m), ref)
                emx = rel(mgroup_host(Fone, B, N, m), ref)
                worst['fp64_step_vs_oracle'] = max(worst['fp64_step_vs_oracle'], e64)
                worst['mixed_step_vs_oracle'] = max(worst['mixed_step_vs_oracle'], emx)
                assert e64 < TOL64, (k, m, e64)
                assert emx < TOLMIX, (k, m, emx)
            s64.density_into(f64.data_ptr())
            sone.density_into(fmx.data_ptr())
            for x in points:
                fref = so3.ifftSO3R_backward(coeffs_at_point(F64, B, N, x), real=True)
                d64 = rel(density_at_point(f64, B, N, x), fref)
                worst['density64_vs_oracle'] = max(worst['density64_vs_oracle'], d64)
                assert d64 < TOL64, (k, x, d64)
            dmx = float(torch.linalg.vector_norm(fmx.double() - f64) / torch.linalg.vector_norm(f64))
            worst['density_mixed_vs_fp64'] = max(worst['density_mixed_vs_fp64'], dmx)
            assert dmx < TOLMIX, (k, dmx)
        smix.step(dt, 'euler', 1)
        smix.store(Ftr)
        row['mixed_trajectory_rel_l2'] = norm(Ftr - F64) / norm(F64)
        spert.step(dt, 'euler', 1)
        spert.store(Ftr)
        row['fp64_perturbed_trajectory_rel_l2'] = norm(Ftr - F64) / norm(F64)
        row['mass_drift_mixed'] = abs(smix.mass() - mass0) / abs(mass0)
        row['mass_drift_fp64'] = abs(s64.mass() - mass0) / abs(mass0)
        table.append(row)
        assert math.isfinite(row['mixed_trajectory_rel_l2'])
        assert row['mass_drift_mixed'] < 1e-12 and row['mass_drift_fp64'] < 1e-12, row
    out = os.environ.get('HP_TRAJECTORY_TABLE')
    if out:
        with open(out, 'w') as fh:
            json.dump({'workload': 'B=15, omega 32^3 over [-4,4]^3, 200 Euler steps, dt=1e-3, seeded matrix-Fisher '
                                   'x Gaussian (seed 2, Sigma 0.25 I), J=diag(0.02,0.02,0.01), rho=(0,0,0.1), b=0.05, '
                                   'H=0.2 I', 'worst': worst,
                       'oracle_checks': {'steps': list(checks), 'm_groups': list(mgroups),
                                         'density_points': [list(p) for p in points]},
                       'per_step': table}, fh, indent=1)


def test_config2_rk4_trajectory_stays_close(hp):
    """The same density and model over 200 RK4 steps of dt = 1e-3, whose
    stability region covers the imaginary-axis spectrum that forward Euler
    amplifies: the mixed trajectory stays within 1e-5 relative L2 of the FP64
    trajectory over all 200 steps (and both keep the l = 0 mass)."""
    import torch
    B, Bx, dt, nsteps = 15, 16, 1e-3, 200
    N = 2 * Bx
    P = pd.pendulum_3d(B, Bx)
    dev = torch.device('cuda', 0)
    nfull = (2 * B - 1) ** 2 * B * N ** 3

    def plan_for(prec):
        pl = hp.Plan(B, Bx, 3, prec, hp.HP_REAL)
        pl.set_model(P.L, P.b, P.G, P.MR, gyro_of(P))
        return pl

    p64, pmix = plan_for(hp.HP_FP64), plan_for(hp.HP_MIXED)
    s64, smix = hp.State(p64), hp.State(pmix)
    U, s, V, mu = seeded_factors(2)
    s64.init_mf_gauss(U, s, V, mu, 0.25 * np.eye(3))
    F64 = torch.empty(nfull, dtype=torch.complex128, device=dev)
    Fmx = torch.empty_like(F64)
    s64.store(F64)
    smix.load(F64)
    n0 = float(torch.linalg.vector_norm(F64))
    mass0 = s64.mass()
    table = []
    for k in range(nsteps):
        s64.step(dt, 'RK4', 1)
        smix.step(dt, 'RK4', 1)
        s64.store(F64)
        smix.store(Fmx)
        n64 = float(torch.linalg.vector_norm(F64))
        row = {'step': k + 1, 'mixed_vs_fp64_rel_l2': float(torch.linalg.vector_norm(Fmx - F64)) / n64,
               'fp64_norm_growth': n64 / n0,
               'mass_drift_mixed': abs(smix.mass() - mass0) / abs(mass0)}
        table.append(row)
        assert row['mixed_vs_fp64_rel_l2'] < 1e-5, row
        assert row['mass_drift_mixed'] < 1e-12, row
    out = os.environ.get('HP_TRAJECTORY_TABLE')
    if out:
        with open(out + '.rk4.json', 'w') as fh:
            json.dump({'workload': 'as the Euler table, RK4 steps', 'per_step': table}, fh, indent=1)


# ------------------------------------------------------------ config 3 ----
@pytest.mark.parametrize('engine', ['simt', 'tensor', 'tensor_bf16'])
def test_config3_roundtrip_full_size(hp, engine):
    import torch
    B, Bx = 32, 12
    lmax, N = B - 1, 2 * Bx
    D = 2 * lmax + 1
    dev = torch.device('cuda', 0)
    g = torch.Generator(device=dev).manual_seed(7)
    F = torch.empty((N, N, N, lmax + 1, D, D), dtype=torch.complex128, device=dev)
    Fr = torch.view_as_real(F)
    Fr.normal_(generator=g)
    l = torch.arange(lmax + 1, device=dev).view(-1, 1, 1)
    m = (torch.arange(D, device=dev) - lmax).view(1, 1, -1)
    n = (torch.arange(D, device=dev) - lmax).view(1, -1, 1)
    scale = (((m.abs() <= l) & (n.abs() <= l)).to(torch.float64) / (2 * l + 1)).view(1, lmax + 1, D, D, 1)
    Fr.view(N ** 3, lmax + 1, D, D, 2).mul_(scale)
    del Fr
    F = F.view(-1)
    nF = torch.linalg.vector_norm(F).item()
    plan = hp.Plan(B, Bx, 3, hp.HP_MIXED, hp.HP_COMPLEX)
    plan.set_beta_engine({'simt': hp.HP_BETA_SIMT, 'tensor': hp.HP_BETA_TENSOR,
                          'tensor_bf16': hp.HP_BETA_TENSOR_BF16}[engine])
    st = hp.State(plan)
    f = torch.empty((2 * B) ** 3 * N ** 3, dtype=torch.complex64, device=dev)
    st.load(F)
    st.density_into(f.data_ptr())
    for x in ((0, 0, 0), (5, 17, 11)):
        fref = so3.ifftSO3R_backward(coeffs_at_point(F, B, N, x), real=False)
        w = x[0] + N * x[1] + N * N * x[2]
        n3 = (2 * B) ** 3
        fx = f[w * n3:(w + 1) * n3].view(2 * B, 2 * B, 2 * B).permute(2, 1, 0).to(torch.complex128).cpu().numpy()
        assert rel(fx, fref) < TOLMIX, (x, rel(fx, fref))
    st.load_density(f.data_ptr())
    assert plan.tc_errors() == 0
    del f
    F2 = torch.empty_like(F)
    st.store(F2)
    F2.sub_(F)
    assert (torch.linalg.vector_norm(F2) / nF).item() < TOLMIX

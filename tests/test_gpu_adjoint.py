"""Reverse mode on the GPU: the adjoint derivative against the oracle's
term-by-term adjoint, the adjoint identity, trajectory gradients against the
oracle (FP64 reference gradient) and against central finite differences of
the library's own forward propagation (agreement 1e-5), and the
torch.autograd wrapper, including the 50-step B=12, 24^3 differentiation
workload with checkpoints every 10 steps.  The 50-step loss carries rounding
noise of ~1e-14 absolute, so the autograd checks take central differences with
a step relative to each parameter, h = 1e-4 |theta| (1e-4 for a zero entry):
at a fixed h = 1e-6 the noise/h term reaches 1e-8, the tolerance for gradients
below 1e-3, and a fixed 1e-4 is 0.5 % of J and shows its curvature."""
import importlib

import numpy as np
import pytest

from oracle import adjoint as adj
from oracle import pendulum as pd
from oracle import so3

pytestmark = pytest.mark.gpu


def rel(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return float(np.linalg.norm((a - b).ravel()) / np.linalg.norm(b.ravel()))


def rcoef(B, xs, rng, hermitian):
    lmax = B - 1
    F = np.zeros((2 * lmax + 1, 2 * lmax + 1, lmax + 1) + xs, np.complex128)
    for l in range(lmax + 1):
        s = slice(lmax - l, lmax + l + 1)
        F[s, s, l] = (rng.standard_normal((2 * l + 1, 2 * l + 1) + xs)
                      + 1j * rng.standard_normal((2 * l + 1, 2 * l + 1) + xs)) / (2 * l + 1)
    if hermitian:
        F = so3.fftSO3R_forward(so3.ifftSO3R_backward(F, real=True))
    return F


def gyro_of(P):
    J = np.diag(P.params['J'])
    return ((J[1] - J[2]) / J[0], (J[2] - J[0]) / J[1], (J[0] - J[1]) / J[2])


def model(kind):
    if kind == '3d':
        P = pd.pendulum_3d(4, 3, L=4.0)
        return P, gyro_of(P)
    return pd.pendulum_reduced(5, 2), (0.0, 0.0, 0.0)


def make_plan(hp, P, gyro, symmetry):
    plan = hp.Plan(P.B, P.Bx, P.ndim, hp.HP_FP64, symmetry)
    plan.set_model(P.L, P.b, P.G, P.MR, gyro)
    return plan


@pytest.mark.parametrize('kind', ['3d', '2d'])
def test_derivative_adjoint_vs_oracle(hp, kind):
    P, gyro = model(kind)
    rng = np.random.default_rng(1)
    xs = (2 * P.Bx,) * P.ndim
    lam = rcoef(P.B, xs, rng, True)
    ref = adj.derivative_adjoint(lam, P)
    out = make_plan(hp, P, gyro, hp.HP_REAL).derivative_adjoint(lam)
    assert rel(out, ref) < 1e-10
    # complex plans take any coefficients
    lamc = rcoef(P.B, xs, rng, False)
    outc = make_plan(hp, P, gyro, hp.HP_COMPLEX).derivative_adjoint(lamc)
    assert rel(outc, adj.derivative_adjoint(lamc, P)) < 1e-10


@pytest.mark.parametrize('kind', ['3d', '2d'])
def test_adjoint_identity_on_gpu(hp, kind):
    P, gyro = model(kind)
    rng = np.random.default_rng(2)
    xs = (2 * P.Bx,) * P.ndim
    plan = make_plan(hp, P, gyro, hp.HP_COMPLEX)
    x, lam = rcoef(P.B, xs, rng, False), rcoef(P.B, xs, rng, False)
    lhs = adj.dot(lam, plan.derivative(x))
    rhs = adj.dot(plan.derivative_adjoint(lam), x)
    assert abs(lhs - rhs) < 1e-11 * abs(lhs)


@pytest.mark.parametrize('kind', ['3d', '2d'])
@pytest.mark.parametrize('nsteps,ckpt', [(5, 2), (4, 10)])
def test_trajectory_adjoint_vs_oracle(hp, kind, nsteps, ckpt):
    P, gyro = model(kind)
    rng = np.random.default_rng(3)
    xs = (2 * P.Bx,) * P.ndim
    F0 = rcoef(P.B, xs, rng, True)
    C = rcoef(P.B, xs, rng, False)           # not real: the projection is part of the test
    dt = 0.01
    lam_ref, g_ref, _ = adj.euler_adjoint(F0, C, P, dt, nsteps)
    plan = make_plan(hp, P, gyro, hp.HP_REAL)
    lam0, g = plan.adjoint(F0, C, nsteps, dt, ckpt)
    assert rel(lam0, lam_ref) < 1e-10
    nd = P.ndim
    for i in range(nd):
        assert abs(g['b'][i] - g_ref[('b', i)]) < 1e-9 * abs(g_ref[('b', i)]) + 1e-14
        assert abs(g['gscale'][i] - g_ref[('gscale', i)]) < 1e-9 * abs(g_ref[('gscale', i)]) + 1e-14
        for j in range(i, nd):
            assert abs(g['G'][i, j] - g_ref[('G', i, j)]) < 1e-9 * abs(g_ref[('G', i, j)]) + 1e-14
    if nd == 3:
        for i in range(3):
            assert abs(g['gyro'][i] - g_ref[('gyro', i)]) < 1e-9 * abs(g_ref[('gyro', i)]) + 1e-14


def test_gradients_vs_finite_differences(hp):
    P, gyro = model('3d')
    rng = np.random.default_rng(4)
    xs = (2 * P.Bx,) * 3
    F0 = rcoef(P.B, xs, rng, True)
    C = rcoef(P.B, xs, rng, True)
    dt, n, h = 0.01, 6, 1e-6
    plan = make_plan(hp, P, gyro, hp.HP_REAL)
    lam0, g = plan.adjoint(F0, C, n, dt, 4)

    def loss(b=P.b, G=P.G, MR=P.MR, gy=gyro, F=F0):
        pl = hp.Plan(P.B, P.Bx, 3, hp.HP_FP64, hp.HP_REAL)
        pl.set_model(P.L, b, G, MR, gy)
        st = hp.State(pl)
        st.load(F)
        st.step(dt, 'euler', n)
        return adj.dot(C, st.store())

    def check(fd, val):
        assert abs(fd - val) < 1e-5 * max(abs(fd), 1e-6), (fd, val)

    for i in range(3):
        e = np.eye(3)[i] * h
        check((loss(b=P.b + e) - loss(b=P.b - e)) / (2 * h), g['b'][i])
        gp, gm = np.array(gyro, float), np.array(gyro, float)
        gp[i] += h
        gm[i] -= h
        check((loss(gy=tuple(gp)) - loss(gy=tuple(gm))) / (2 * h), g['gyro'][i])
        MRp, MRm = P.MR.copy(), P.MR.copy()
        MRp[..., i] *= 1 + h
        MRm[..., i] *= 1 - h
        check((loss(MR=MRp) - loss(MR=MRm)) / (2 * h), g['gscale'][i])
    E = np.zeros((3, 3))
    E[0, 1] = h
    check((loss(G=P.G + E) - loss(G=P.G - E)) / (2 * h), g['G'][0, 1])
    V = rcoef(P.B, xs, rng, True)
    check((loss(F=F0 + h * V) - loss(F=F0 - h * V)) / (2 * h), adj.dot(lam0, V))


def _autograd_case(hp, B, Bx, nsteps, ckpt, device):
    import torch
    ag = importlib.import_module('hybridpendulum-up_b200.autograd')
    P = pd.pendulum_3d(B, Bx, L=8.0)
    J_ref = np.array(np.diag(P.params['J']))
    plan = hp.Plan(B, Bx, 3, hp.HP_FP64, hp.HP_REAL)
    f0, _ = pd.seeded_density(B, Bx, 3, P.L, seed=21)
    F0 = ag.to_torch(plan.forward(f0), device)
    # the measurement density: matrix-Fisher with the initial density's seeded
    # parameters, omega spread 0.3 (so that the band-limited overlap is positive)
    pm, _ = pd.seeded_density(B, Bx, 3, P.L, seed=21, sigma=0.3)
    Pw = ag.measurement_weights(plan, pm, P.L).to(device)
    dt = 1e-3

    def loss_of(F, b, J, H):
        bb, gy, G, gs = ag.pendulum_params(b, J, H, J_ref)
        FT = ag.propagate(F, bb, gy, G, gs, plan=plan, MR=P.MR, L=P.L, dt=dt, nsteps=nsteps,
                          checkpoint_every=ckpt)
        return -torch.log(torch.real(torch.sum(torch.conj(Pw) * FT)))

    b = torch.tensor(P.b, dtype=torch.float64, requires_grad=True)
    J = torch.tensor(J_ref, dtype=torch.float64, requires_grad=True)
    H = torch.tensor(np.eye(3) * 0.2, dtype=torch.float64, requires_grad=True)
    F0g = F0.clone().requires_grad_(True)
    L0 = loss_of(F0g, b, J, H)
    assert torch.isfinite(L0)
    L0.backward()

    def fd(name, idx):
        args = dict(b=b.detach().clone(), J=J.detach().clone(), H=H.detach().clone())
        a = args[name].view(-1)
        h = 1e-4 * (abs(a[idx].item()) or 1.0)
        a[idx] += h
        lp = loss_of(F0, **args).item()
        a[idx] -= 2 * h
        lm = loss_of(F0, **args).item()
        return (lp - lm) / (2 * h)

    for name, t in (('b', b), ('J', J), ('H', H)):
        for idx in range(t.numel()):
            ref = fd(name, idx)
            val = t.grad.view(-1)[idx].item()
            assert abs(val - ref) < 1e-5 * max(abs(ref), 1e-3), (name, idx, val, ref)
    # initial coefficients along a real-density direction
    v, _ = pd.seeded_density(B, Bx, 3, P.L, seed=23)
    V = ag.to_torch(plan.forward(v), device)
    h = 1e-4
    with torch.no_grad():
        lp = loss_of(F0 + h * V, b, J, H).item()
        lm = loss_of(F0 - h * V, b, J, H).item()
    ref = (lp - lm) / (2 * h)
    val = torch.real(torch.sum(torch.conj(F0g.grad) * V)).item()
    assert abs(val - ref) < 1e-5 * max(abs(ref), 1e-3), (val, ref)


def test_autograd_small(hp):
    _autograd_case(hp, 4, 3, 6, 4, 'cpu')


def test_autograd_b12_omega24_50_steps(hp):
    """The differentiation workload: B=12, omega 24^3, 50 steps, checkpoints every 10."""
    _autograd_case(hp, 12, 12, 50, 10, 'cuda')

"""Host F inputs in page-locked, mapped memory are read in place (only the
entries the plan keeps) instead of being copied whole: the results must be
bit-identical to those of the same call on a pageable (numpy) buffer, which
takes the copy path, and the copy path must still match the FP64 oracle.
"""
import numpy as np
import pytest

from oracle import pendulum as pd
from oracle import so3

pytestmark = pytest.mark.gpu

torch = pytest.importorskip('torch')


def gyro_of(P):
    J = np.diag(P.params['J'])
    return ((J[1] - J[2]) / J[0], (J[2] - J[0]) / J[1], (J[0] - J[1]) / J[2])


def pinned(a, offset=0):
    """A page-locked host tensor holding `a` in MATLAB (column-major) order,
    starting `offset` elements into its allocation."""
    flat = np.asfortranarray(a).ravel(order='K')
    t = torch.empty(flat.size + offset, dtype=torch.from_numpy(flat[:1]).dtype, pin_memory=True)
    v = t[offset:]
    v.copy_(torch.from_numpy(flat))
    return v


def test_read_in_place_flags(hp):
    a = np.zeros(64, np.complex128)
    assert not hp.host_read_in_place(a)
    assert not hp.host_read_in_place(torch.zeros(64, dtype=torch.complex128))
    assert hp.host_read_in_place(pinned(a))
    assert hp.host_read_in_place(pinned(a, offset=3))
    # 8-byte aligned: copied whole (the in-place reads are 16-byte loads)
    t = torch.zeros(2 * 64 + 1, dtype=torch.float64, pin_memory=True)
    assert hp.host_read_in_place(t[:128])
    assert not hp.host_read_in_place(t[1:])


@pytest.mark.parametrize('ndim,symmetry', [(3, 0), (3, 1), (2, 0)])
@pytest.mark.parametrize('precision', [0, 1])
def test_backward_in_place_matches_copy(hp, ndim, symmetry, precision):
    B, Bx = 5, 3
    P = pd.pendulum_3d(B, Bx) if ndim == 3 else None
    xs = (2 * Bx,) * ndim
    if ndim == 3:
        f, _ = pd.seeded_density(B, Bx, 3, P.L, seed=21)
    else:
        rng = np.random.default_rng(22)
        f = rng.random((2 * B,) * 3 + xs) + 0.5
    F = so3.fftSO3R_forward(f)
    plan = hp.get_plan(B, Bx, ndim, precision, symmetry)
    ref = plan.backward(F)                           # pageable: copied whole
    Ft = pinned(F, offset=1)
    assert hp.host_read_in_place(Ft)
    fdt = torch.complex128 if symmetry == 1 else torch.float64
    out = torch.zeros(int(np.prod(plan.f_shape)), dtype=fdt, pin_memory=True)
    plan.backward(Ft, out=out)
    got = out.numpy().reshape(plan.f_shape, order='F')
    assert np.array_equal(got, ref)
    want = so3.ifftSO3R_backward(F, real=(symmetry == 0))
    tol = 1e-10 if precision == 0 else 1e-6
    assert np.linalg.norm((ref - want).ravel()) <= tol * np.linalg.norm(want.ravel())


@pytest.mark.parametrize('precision', [0, 1])
@pytest.mark.parametrize('method', ['euler', 'rk4'])
def test_propagate_in_place_matches_copy(hp, precision, method):
    P = pd.pendulum_3d(4, 2)
    f, _ = pd.seeded_density(4, 2, 3, P.L, seed=23)
    F = so3.fftSO3R_forward(f)
    plan = hp.get_plan(P.B, P.Bx, 3, precision, hp.HP_REAL)
    plan.set_model(P.L, P.b, P.G, P.MR, gyro_of(P))
    ref = plan.propagate(F, 1e-3, method)
    Ft = pinned(F)
    out = torch.zeros(F.size, dtype=torch.complex128, pin_memory=True)
    plan.propagate(Ft, 1e-3, method, out=out)
    assert np.array_equal(out.numpy().reshape(F.shape, order='F'), ref)
    # in place: input and output are the same pinned buffer
    plan.propagate(Ft, 1e-3, method, out=Ft)
    assert np.array_equal(Ft.numpy().reshape(F.shape, order='F'), ref)
    dF = plan.derivative(F)
    dFt = torch.zeros(F.size, dtype=torch.complex128, pin_memory=True)
    plan.derivative(pinned(F), out=dFt)
    assert np.array_equal(dFt.numpy().reshape(F.shape, order='F'), dF)


def test_state_load_in_place_matches_copy(hp):
    P = pd.pendulum_3d(4, 2)
    f, _ = pd.seeded_density(4, 2, 3, P.L, seed=24)
    F = so3.fftSO3R_forward(f)
    plan = hp.get_plan(P.B, P.Bx, 3, 0, hp.HP_REAL)
    plan.set_model(P.L, P.b, P.G, P.MR, gyro_of(P))
    a, b = hp.State(plan), hp.State(plan)
    a.load(F)
    b.load(pinned(F, offset=5))
    a.step(1e-3, 'euler', 3)
    b.step(1e-3, 'euler', 3)
    assert np.array_equal(a.store(), b.store())

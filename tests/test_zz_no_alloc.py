"""hp_pendulum_derivative_noalloc: the derivative for callers that cannot
allocate device memory while they run (all scratch in one static device array).

Collected last on purpose: a failure here leaves every other test already run.
Compared with the allocating entry point hp_pendulum_derivative on the same
inputs, through the C ABI, on two calls in a row (the second with different
inputs, so stale scratch contents would show), and with the FP64 oracle's
derivative.
"""
import ctypes

import numpy as np
import pytest

from oracle import pendulum as pd
from oracle import so3

pytestmark = pytest.mark.gpu

TOL = {0: 1e-10, 1: 1e-6}


def _fn(hp):
    fn = hp._lib.hp_pendulum_derivative_noalloc
    fn.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
    fn.restype = ctypes.c_int
    return fn


def _rel(a, b):
    import torch
    return float(torch.linalg.vector_norm(a - b) / torch.linalg.vector_norm(b))


def _setup(hp, ndim, precision):
    if ndim == 3:
        P = pd.pendulum_3d(4, 2)
        J = np.diag(P.params['J'])
        gyro = ((J[1] - J[2]) / J[0], (J[2] - J[0]) / J[1], (J[0] - J[1]) / J[2])
    else:
        P = pd.pendulum_reduced(4, 3)
        gyro = (0.0, 0.0, 0.0)
    plan = hp.Plan(P.B, P.Bx, ndim, precision, hp.HP_REAL)
    plan.set_model(P.L, P.b, P.G, P.MR, gyro)
    return P, plan


def _coeffs(P, seed):
    f, _ = pd.seeded_density(P.B, P.Bx, P.ndim, P.L, seed=seed)
    return so3.fftSO3R_forward(f)


@pytest.mark.parametrize('ndim', [3, 2])
@pytest.mark.parametrize('precision', [0, 1])
def test_noalloc_matches_allocating_derivative(hp, ndim, precision):
    import torch
    P, plan = _setup(hp, ndim, precision)
    fn = _fn(hp)
    for call, seed in enumerate((1, 2)):
        Fh = _coeffs(P, seed)
        F = torch.from_numpy(np.asfortranarray(Fh).ravel(order='F')).cuda()
        ref = plan.derivative(F)
        out = torch.full_like(F, complex(float('nan'), float('nan')))
        rc = fn(plan.handle, F.data_ptr(), out.data_ptr())
        assert rc == hp.HP_OK, hp._lib.hp_last_error().decode()
        torch.cuda.synchronize()
        assert torch.isfinite(torch.view_as_real(out)).all(), f'call {call}: output not fully written'
        assert _rel(out, ref) < TOL[precision], f'call {call}'
        oracle = pd.derivative_fast(Fh, P)
        got = out.cpu().numpy().reshape(Fh.shape, order='F')
        assert np.linalg.norm(got - oracle) / np.linalg.norm(oracle) < TOL[precision], f'call {call}'


def test_noalloc_rejects_grids_above_32_points(hp):
    """The plane tiles of the allocation-free path hold at most 32 points per
    axis; a 40-point grid is refused (the allocating path takes it)."""
    import torch
    P = pd.pendulum_reduced(2, 20)
    plan = hp.Plan(2, 20, 2, hp.HP_FP64, hp.HP_REAL)
    plan.set_model(P.L, P.b, P.G, P.MR)
    buf = torch.zeros(16, dtype=torch.complex128, device='cuda')
    assert _fn(hp)(plan.handle, buf.data_ptr(), buf.data_ptr()) == hp.HP_ERR_UNSUPPORTED


def test_noalloc_rejects_oversized_problem(hp):
    import torch
    P = pd.pendulum_reduced(10, 16)       # 715 rows x 1024 points x 64 B > 32 MiB
    plan = hp.Plan(10, 16, 2, hp.HP_FP64, hp.HP_REAL)
    plan.set_model(P.L, P.b, P.G, P.MR)
    buf = torch.zeros(16, dtype=torch.complex128, device='cuda')
    rc = _fn(hp)(plan.handle, buf.data_ptr(), buf.data_ptr())
    assert rc == hp.HP_ERR_SHAPE
    assert 'scratch' in hp._lib.hp_last_error().decode()

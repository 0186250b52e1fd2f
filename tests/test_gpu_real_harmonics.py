"""Real-harmonic transforms on the GPU (hp_fftSO3_real_forward/backward) against
the oracle restatement of fftSO3.m / ifftSO3.m (isreal).  FP64: <= 1e-12
relative (max norm)."""
import numpy as np
import pytest

from oracle import real_harmonics as rh
from oracle import so3

pytestmark = pytest.mark.gpu


def band_limited(B, seed):
    lmax = B - 1
    rng = np.random.default_rng(seed)
    F = np.zeros((2 * lmax + 1, 2 * lmax + 1, lmax + 1), complex)
    for l in range(lmax + 1):
        s = slice(lmax - l, lmax + l + 1)
        F[s, s, l] = rng.standard_normal((2 * l + 1, 2 * l + 1)) + 1j * rng.standard_normal((2 * l + 1, 2 * l + 1))
    return so3.ifftSO3R_backward(F, real=True)


def rmax(a, b):
    return float(np.abs(np.asarray(a) - np.asarray(b)).max() / np.abs(np.asarray(b)).max())


@pytest.mark.parametrize('B', [2, 3, 5, 8, 10])
def test_forward_backward_vs_oracle(hp, B):
    f = band_limited(B, B + 1)
    F = rh.forward(f)
    plan = hp.get_plan(B, 2, 2)
    assert rmax(plan.real_forward(f), F) < 1e-12
    assert rmax(plan.real_backward(F), rh.backward(F)) < 1e-12
    # module-level drop-ins
    assert rmax(hp.fftSO3_real(f), F) < 1e-12
    assert rmax(hp.ifftSO3_real(F), f) < 1e-12


def test_batched_and_device_memory(hp):
    import torch
    B, nb = 6, 3
    fs = np.stack([band_limited(B, 40 + k) for k in range(nb)], -1)
    plan = hp.get_plan(B, 2, 2)
    Fb = plan.real_forward(fs)
    assert Fb.shape == (2 * B - 1, 2 * B - 1, B, nb)
    for k in range(nb):
        assert rmax(Fb[..., k], rh.forward(fs[..., k])) < 1e-12
    ft = torch.from_numpy(np.asfortranarray(fs).ravel(order='F')).cuda()
    Ft = plan.real_forward(ft)
    assert np.abs(Ft.cpu().numpy() - Fb.ravel(order='F')).max() == 0.0
    fb = plan.real_backward(Ft)
    assert rmax(fb.cpu().numpy(), fs.ravel(order='F')) < 1e-12


def test_bandlimit_16_round_trip(hp):
    B = 16
    rng = np.random.default_rng(3)
    D = 2 * B - 1
    F = np.zeros((D, D, B))
    for l in range(B):
        s = slice(B - 1 - l, B + l)
        F[s, s, l] = rng.standard_normal((2 * l + 1, 2 * l + 1)) / (2 * l + 1)
    plan = hp.get_plan(B, 2, 2)
    f = plan.real_backward(F)
    assert rmax(plan.real_forward(f), F) < 1e-12


def test_real_transform_errors(hp):
    plan = hp.get_plan(3, 2, 2)
    with pytest.raises(hp.HPError):
        plan.real_forward(np.zeros((5, 6, 6)))
    with pytest.raises(hp.HPError):
        plan.real_backward(np.zeros((5, 5, 2)))


@pytest.mark.parametrize('B', [3, 5, 8])
def test_real_product_vs_oracle(hp, B):
    f, g = band_limited(B, 7), band_limited(B, 8)
    F, G = rh.forward(f), rh.forward(g)
    ref = rh.prod_literal(F, G)
    out = hp.fftSO3_prod_real(F, G)
    assert rmax(out, ref) < 1e-11
    # batched
    FG2 = hp.get_plan(B, 2, 2).real_prod(np.stack([F, G], -1), np.stack([G, F], -1))
    assert rmax(FG2[..., 0], ref) < 1e-11 and rmax(FG2[..., 1], ref) < 1e-11

"""Forward transform with its beta contraction on the tensor cores (tcgen05,
three TF32 products per FP32 product, or six BF16 products of BF16x3 split
operands) against the CUDA-core FP32 contraction and the FP64 oracle: every
padded node count (2B -> 8, 24, 32, 40, 48, 64),
real and complex plans, partial and multiple omega tiles (64 points each).
Tolerances: tensor vs FP64 oracle <= 1e-6 relative L2 (the mixed-precision
bar); tensor vs CUDA-core FP32 <= 1e-6."""
import numpy as np
import pytest

from oracle import so3

pytestmark = pytest.mark.gpu


def rel(a, b):
    return float(np.linalg.norm((np.asarray(a) - np.asarray(b)).ravel()) / np.linalg.norm(np.asarray(b).ravel()))


def coeffs(B, xs, seed, hermitian):
    rng = np.random.default_rng(seed)
    lmax = B - 1
    F = np.zeros((2 * lmax + 1, 2 * lmax + 1, lmax + 1) + xs, np.complex128)
    for l in range(lmax + 1):
        s = slice(lmax - l, lmax + l + 1)
        F[s, s, l] = (rng.standard_normal((2 * l + 1, 2 * l + 1) + xs)
                      + 1j * rng.standard_normal((2 * l + 1, 2 * l + 1) + xs)) / (2 * l + 1)
    if hermitian:
        F = so3.fftSO3R_forward(so3.ifftSO3R_backward(F, real=True))
    return F


ENGINES = {'tf32x3': ('HP_BETA_TENSOR', 'tf.anal.beta.tc'), 'bf16x3': ('HP_BETA_TENSOR_BF16', 'tf.anal.beta.tc16')}


def forward_both(hp, B, Bx, ndim, sym, f, engine='tf32x3'):
    plan = hp.Plan(B, Bx, ndim, hp.HP_MIXED, sym)
    plan.set_beta_engine(hp.HP_BETA_SIMT)
    F_simt = plan.forward(f)
    code, fam_name = ENGINES[engine]
    plan.set_beta_engine(getattr(hp, code))
    plan.profile(True)
    F_tc = plan.forward(f)
    fam = plan.profile_read()
    assert fam_name in fam and 'tf.anal.beta' not in fam, fam
    assert plan.tc_errors() == 0
    return F_simt, F_tc


@pytest.mark.parametrize('engine', ['tf32x3', 'bf16x3'])
@pytest.mark.parametrize('B', [4, 10, 15, 20, 24, 30, 32])
@pytest.mark.parametrize('real', [True, False])
def test_tc_beta_vs_oracle(hp, B, real, engine):
    Bx = 2
    F = coeffs(B, (4, 4), 10 + B, real)
    f = so3.ifftSO3R_backward(F, real=real)
    sym = hp.HP_REAL if real else hp.HP_COMPLEX
    F_simt, F_tc = forward_both(hp, B, Bx, 2, sym, f, engine)
    assert rel(F_tc, F) < 1e-6
    assert rel(F_tc, F_simt) < 1e-6


@pytest.mark.parametrize('engine', ['tf32x3', 'bf16x3'])
@pytest.mark.parametrize('B,Bx,ndim', [(15, 6, 2), (30, 6, 2), (8, 4, 3)])
def test_tc_beta_many_tiles(hp, B, Bx, ndim, engine):
    # 144 and 512 omega points: full 64-point tiles plus a partial one
    # a real band-limited density and its coefficients from the FP64 CUDA
    # transforms (parity-tested against the oracle elsewhere)
    Fc = coeffs(B, (2 * Bx,) * ndim, 7, False)
    f = np.asfortranarray(np.real(hp.Plan(B, Bx, ndim, hp.HP_FP64, hp.HP_COMPLEX).backward(Fc)))
    F = hp.Plan(B, Bx, ndim, hp.HP_FP64, hp.HP_REAL).forward(f)
    F_simt, F_tc = forward_both(hp, B, Bx, ndim, hp.HP_REAL, f, engine)
    assert rel(F_tc, F) < 1e-6
    assert rel(F_tc, F_simt) < 1e-6


def test_tc_beta_default_engine(hp):
    # HP_MIXED plans with B >= 15 take the tensor-core contraction unless told otherwise
    B, Bx = 15, 2
    F = coeffs(B, (4, 4), 3, True)
    plan = hp.Plan(B, Bx, 2, hp.HP_MIXED, hp.HP_REAL)
    plan.profile(True)
    out = plan.forward(so3.ifftSO3R_backward(F, real=True))
    assert 'tf.anal.beta.tc' in plan.profile_read()
    assert rel(out, F) < 1e-6

"""Precision of the tensor-core forward beta contraction, emulated on the CPU.

The tcgen05 kernel (tc_beta.cu) contracts, per (m, n) pair,
F^l_mn[w] = sum_b W[l][b] Q_b[w] with W = w_b d^l_mn(beta_b)
(fftSO3R.m:89-106), using three TF32 products per FP32 product: each operand
x = hi + lo with hi = x rounded to TF32 (low 13 mantissa bits cleared) and
lo = x - hi in FP32 (W's split from the FP64 table), D = A_hi W_hi + A_hi W_lo +
A_lo W_hi accumulated in FP32, and the tensor core reading only the TF32 part of
each operand (lo's low 13 bits dropped).  This test restates that arithmetic in
numpy for the pairs of B = 15 and B = 30 (w_b d from the oracle) and checks it
against the FP64 contraction of the same FP32 inputs: within the 1e-6 relative
L2 bar of the mixed-precision path, while one TF32 product per FP32 product is
not, which is why the split is there.

The second form, BF16x3 (kind::f16 with BF16 operands), splits each operand
three ways, x = b0 + b1 + b2 (b_i = bf16 round-to-nearest of the remainder,
each remainder exact in FP32; W's split from FP64), and sums the six products
of order <= 2 in FP32; every BF16 x BF16 product is exact in FP32.
"""
import numpy as np
import pytest

from oracle import so3


def tf32_rn(x):
    u = np.asarray(x, np.float32).view(np.uint32)
    return ((u + np.uint32(0x1000)) & np.uint32(0xFFFFE000)).view(np.float32)


def tf32_trunc(x):
    return (np.asarray(x, np.float32).view(np.uint32) & np.uint32(0xFFFFE000)).view(np.float32)


def pair_tables(B, ms):
    lmax = B - 1
    d = so3.wigner_d_table(B)            # [m+lmax, n+lmax, l, b]
    w = so3.quad_weights(B)
    for m in ms:
        for n in range(-lmax, lmax + 1):
            l0 = max(abs(m), abs(n))
            yield w[None, :] * d[m + lmax, n + lmax, l0:, :]     # W64[l - l0][b]


@pytest.mark.parametrize('B', [15, 30])
def test_three_tf32_products_meet_the_fp32_bar(B):
    rng = np.random.default_rng(B)
    nw = 128                              # real rows: 64 complex omega points
    err3 = err1 = err32 = ref = 0.0
    for W64 in pair_tables(B, ms=(0, 1, B // 2, B - 1)):
        Q32 = rng.standard_normal((2 * B, nw)).astype(np.float32)   # the kernel's FP32 input
        D64 = W64 @ Q32.astype(np.float64)
        # three TF32 products, FP32 accumulation
        Ah = tf32_rn(Q32)
        Al = tf32_trunc(Q32 - Ah)
        Wh = tf32_rn(W64.astype(np.float32))
        Wl = tf32_trunc((W64 - Wh.astype(np.float64)).astype(np.float32))
        D3 = (Wh @ Ah) + (Wl @ Ah) + (Wh @ Al)
        # one TF32 product, and plain FP32 FMAs (the CUDA-core kernel), for scale
        D1 = tf32_rn(W64.astype(np.float32)) @ tf32_rn(Q32)
        D32 = W64.astype(np.float32) @ Q32
        err3 += float(np.sum((D3 - D64) ** 2))
        err1 += float(np.sum((D1 - D64) ** 2))
        err32 += float(np.sum((D32 - D64) ** 2))
        ref += float(np.sum(D64 ** 2))
    r3, r1, r32 = (np.sqrt(e / ref) for e in (err3, err1, err32))
    assert r3 < 1e-6, r3
    assert r3 < 5 * r32 + 1e-7, (r3, r32)   # on par with plain FP32 arithmetic
    assert r1 > 1e-5, r1                    # a single TF32 product misses the bar


def bf16_rn(x):
    """Round FP32 to BF16 (nearest, ties to even) and back to FP32."""
    u = np.asarray(x, np.float32).view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000).astype(np.uint32)
    return r.view(np.float32)


def bf16x3(x64_or_32):
    x = np.asarray(x64_or_32, np.float64)
    b0 = bf16_rn(x.astype(np.float32))
    r1 = x - b0.astype(np.float64)
    b1 = bf16_rn(r1.astype(np.float32))
    r2 = r1 - b1.astype(np.float64)
    b2 = bf16_rn(r2.astype(np.float32))
    return b0, b1, b2


@pytest.mark.parametrize('B', [15, 30, 32])
def test_bf16x3_products_meet_the_fp32_bar(B):
    rng = np.random.default_rng(100 + B)
    nw = 128
    err = err1 = ref = 0.0
    for W64 in pair_tables(B, ms=(0, 1, B // 2, B - 1)):
        Q32 = rng.standard_normal((2 * B, nw)).astype(np.float32)
        D64 = W64 @ Q32.astype(np.float64)
        a0, a1, a2 = bf16x3(Q32)
        w0, w1, w2 = bf16x3(W64)
        f32 = np.float32
        D = (w0 @ a0).astype(f32) + (w1 @ a0).astype(f32) + (w0 @ a1).astype(f32) \
            + (w2 @ a0).astype(f32) + (w0 @ a2).astype(f32) + (w1 @ a1).astype(f32)
        D1 = bf16_rn(W64.astype(np.float32)) @ bf16_rn(Q32)
        err += float(np.sum((D.astype(np.float64) - D64) ** 2))
        err1 += float(np.sum((D1 - D64) ** 2))
        ref += float(np.sum(D64 ** 2))
    r, r1 = np.sqrt(err / ref), np.sqrt(err1 / ref)
    assert r < 1e-6, r
    assert r1 > 1e-4, r1                    # one BF16 product is far from the bar

"""The split-BF16 tensor-core product (tcgen05.mma kind::f16, TMA-staged, FP32 accumulation in
tensor memory) through dvr3d_b200_split_gemm.

Reference: the same product formed in FP64 from the BF16 slices themselves (hi = bf16(x),
lo = bf16(x - hi), round to nearest even at 8 significant bits), so that the only difference
left is the FP32 accumulation; and the plain FP64 product, against which the BF16x3 form must
be about 2^-16 accurate and clearly better than one BF16 product.
"""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def bf16(x: np.ndarray) -> np.ndarray:
    """Round float64 values to the nearest BF16 value (ties to even), as __double2bfloat16."""
    m, e = np.frexp(x)                      # x = m * 2**e, 0.5 <= |m| < 1
    return np.ldexp(np.rint(m * 256.0) / 256.0, e)


def split(x: np.ndarray):
    hi = bf16(x)
    return hi, bf16(x - hi)


SHAPES = [(1, 1, 1), (37, 5, 70), (128, 64, 64), (129, 65, 130), (300, 48, 1000), (1000, 200, 333),
          (257, 300, 2049)]


@pytest.mark.parametrize("m,n,k", SHAPES)
@pytest.mark.parametrize("nslice", [1, 2])
def test_split_gemm_matches_slice_products(ctx, m, n, k, nslice):
    rng = np.random.default_rng(1000 * m + 10 * n + k + nslice)
    a = rng.standard_normal((k, m))
    b = rng.standard_normal((k, n)) * np.exp(rng.uniform(-3, 3, size=(1, n)))
    got = ctx.split_gemm(a, b, nslice)
    ah, al = split(a)
    bh, bl = split(b)
    want = ah.T @ bh if nslice == 1 else ah.T @ bh + ah.T @ bl + al.T @ bh
    scale = np.abs(a).T @ np.abs(b)
    # FP32 accumulation of exactly representable slice products: the classical bound k u32
    bound = max(k, 16) * 2.0 ** -24
    assert np.all(np.abs(got - want) <= bound * scale + 1e-300), np.max(np.abs(got - want) / scale)
    err64 = np.max(np.abs(got - a.T @ b) / scale)
    assert err64 <= (2.0 ** -7 if nslice == 1 else 2.0 ** -14)


def test_bf16x3_is_far_more_accurate_than_one_product(ctx):
    rng = np.random.default_rng(7)
    a = rng.standard_normal((512, 300))
    b = rng.standard_normal((512, 96))
    exact = a.T @ b
    scale = np.abs(a).T @ np.abs(b)
    e1 = np.max(np.abs(ctx.split_gemm(a, b, 1) - exact) / scale)
    e3 = np.max(np.abs(ctx.split_gemm(a, b, 2) - exact) / scale)
    assert e3 < e1 / 50.0, (e1, e3)


def test_split_gemm_rejects_bad_arguments(ctx):
    import dvr3d_b200

    with pytest.raises(dvr3d_b200.DVR3DError):
        ctx.split_gemm(np.ones((4, 3)), np.ones((4, 2)), 3)

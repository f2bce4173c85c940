"""The arithmetic of the tensor-core trailing update, restated on the CPU.

k_dense_lu_tc and k_dlu_update_tc multiply FP32 operands on TF32 tensor cores by splitting each
value x into hi = x rounded to TF32 (cvt.rna.tf32.f32: 10 explicit mantissa bits, ties away
from zero) and lo = x - hi (exact in FP32), and computing hi_a hi_b + hi_a lo_b + lo_a hi_b with
FP32 accumulation.  The MMA reads lo as TF32 too, dropping its low 13 mantissa bits.  This test
emulates that arithmetic with numpy and checks:

* the split is exact (hi + lo == x) and |lo| <= 2^-11 |x|;
* a 128 x 128 tile with K = 32 (one panel of the dense LU) agrees with the FP64 product to well
  within FP32-level error (1e-6 of the largest entry), while a single TF32 product
  (hi_a hi_b only) does not."""

import numpy as np


def rna_tf32(x):
    """Round FP32 values to TF32 (ties away from zero), as cvt.rna.tf32.f32."""
    u = np.asarray(x, np.float32).view(np.uint32).astype(np.uint64)
    r = (u + 0x1000) & 0xFFFFE000  # add half an ulp of the 10-bit mantissa, then truncate
    return r.astype(np.uint32).view(np.float32)


def trunc_tf32(x):
    """The low 13 mantissa bits dropped, as the MMA reads an FP32 operand of kind::tf32."""
    u = np.asarray(x, np.float32).view(np.uint32) & np.uint32(0xFFFFE000)
    return u.view(np.float32)


def split(x):
    x = np.asarray(x, np.float32)
    hi = rna_tf32(x)
    lo = (x - hi).astype(np.float32)
    return hi, lo


def test_split_is_exact_and_small():
    rng = np.random.default_rng(0)
    x = np.concatenate([
        rng.standard_normal(100_000).astype(np.float32),
        (rng.standard_normal(10_000) * 1e30).astype(np.float32),
        (rng.standard_normal(10_000) * 1e-30).astype(np.float32),
        np.array([1.0, -1.0, 1.0 + 2.0 ** -11, 1.0 + 3 * 2.0 ** -12, 0.0], np.float32)])
    hi, lo = split(x)
    assert np.array_equal((hi.astype(np.float64) + lo.astype(np.float64)).astype(np.float32), x)
    assert np.array_equal(hi + lo, x)
    assert np.all(np.abs(lo) <= np.abs(x) * 2.0 ** -11 * (1 + 1e-7))
    # hi carries at most 10 explicit mantissa bits
    assert np.all(hi.view(np.uint32) & np.uint32(0x1FFF) == 0)


def test_three_product_tile_is_fp32_accurate():
    rng = np.random.default_rng(1)
    M, N, K = 128, 128, 32
    a = rng.uniform(-1, 1, (M, K)).astype(np.float32)   # L21 rows
    b = rng.uniform(-1, 1, (K, N)).astype(np.float32)   # U12 columns
    ref = a.astype(np.float64) @ b.astype(np.float64)
    ah, al = split(a)
    bh, bl = split(b)
    # operands as the MMA reads them (hi is already TF32; lo loses its low 13 bits); products
    # of TF32 values are exact in FP64, the sum is accumulated in FP32 over K
    terms = (trunc_tf32(ah).astype(np.float64)[:, :, None] * trunc_tf32(bh).astype(np.float64)[None]
             + trunc_tf32(ah).astype(np.float64)[:, :, None] * trunc_tf32(bl).astype(np.float64)[None]
             + trunc_tf32(al).astype(np.float64)[:, :, None] * trunc_tf32(bh).astype(np.float64)[None])
    acc = np.zeros((M, N), np.float32)
    for k in range(K):
        acc = (acc + terms[:, k, :].astype(np.float32)).astype(np.float32)
    scale = np.max(np.abs(ref))
    err3 = np.max(np.abs(acc - ref)) / scale
    one = np.zeros((M, N), np.float32)
    for k in range(K):
        one = (one + (ah[:, k, None].astype(np.float64) * bh[None, k, :]).astype(np.float32))
    err1 = np.max(np.abs(one - ref)) / scale
    print(f"3xTF32 {err3:.2e}, 1xTF32 {err1:.2e} of the largest entry")
    assert err3 < 1e-6
    assert err1 > 10 * err3

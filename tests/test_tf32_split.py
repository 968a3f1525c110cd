"""The TF32 operand splits of the tensor-core kernels, restated in numpy.

The kernels round to TF32 with integer bit arithmetic (``rn_tf32`` in
``csrc/tc_gemm.cu``: add half of the dropped 13-bit field to the bit pattern,
clear the field) and split a value as x_hi + x_lo.  Two splits are in use:

* round-to-nearest: x_hi = rn(x), x_lo = rn(x - x_hi) (C, U and the Gram
  operands);
* the half transform's streamed B tile: the tensor core takes the TF32
  truncation of the FP32 value as x_hi, and the kernel writes
  x_lo = rn(x - trunc(x)) (the residual is exact in FP32).

Both represent x to within 2^-22 relative, and the truncation split is as
unbiased as the round-to-nearest one because the residual carries the
truncated bits.
"""

import numpy as np


def rn_tf32(x: np.ndarray) -> np.ndarray:
    b = x.astype(np.float32).view(np.uint32)
    return ((b + np.uint32(0x1000)) & np.uint32(0xFFFFE000)).view(np.float32)


def trunc_tf32(x: np.ndarray) -> np.ndarray:
    return (x.astype(np.float32).view(np.uint32) & np.uint32(0xFFFFE000)).view(np.float32)


def _samples(n=200_000, seed=3):
    rng = np.random.default_rng(seed)
    x = (rng.standard_normal(n) * np.exp(rng.uniform(-20, 20, n))).astype(np.float32)
    return x[x != 0]


def test_rn_tf32_matches_round_to_nearest_on_10_mantissa_bits():
    x = _samples()
    h = rn_tf32(x).astype(np.float64)
    # representable: low 13 bits clear; error at most half a TF32 ulp (2^-11 relative)
    assert (rn_tf32(x).view(np.uint32) & 0x1FFF == 0).all()
    assert (np.abs(h - x) <= 2.0**-11 * np.abs(x.astype(np.float64))).all()


def test_both_splits_represent_x_to_2_pow_minus_22():
    x = _samples()
    x64 = x.astype(np.float64)
    hi_rn = rn_tf32(x)
    lo_rn = rn_tf32(x - hi_rn)
    hi_tr = trunc_tf32(x)
    resid = x - hi_tr
    # the truncation residual is exact in FP32
    assert (resid.astype(np.float64) == x64 - hi_tr.astype(np.float64)).all()
    lo_tr = rn_tf32(resid)
    for hi, lo in ((hi_rn, lo_rn), (hi_tr, lo_tr)):
        assert (lo.view(np.uint32) & 0x1FFF == 0).all()
        err = np.abs(hi.astype(np.float64) + lo.astype(np.float64) - x64)
        assert (err <= 2.0**-22 * np.abs(x64)).all()


def test_truncation_split_is_unbiased():
    """Mean signed error of hi + lo relative to |x|: ~0 for both splits, unlike
    truncation alone (which is always toward zero)."""
    x = _samples(400_000, seed=5)
    x64 = x.astype(np.float64)
    hi_tr = trunc_tf32(x)
    lo_tr = rn_tf32(x - hi_tr)
    rel = (hi_tr.astype(np.float64) + lo_tr.astype(np.float64) - x64) / np.abs(x64)
    alone = (hi_tr.astype(np.float64) - x64) / x64  # truncation toward zero: always <= 0
    assert (alone <= 0).all() and alone.mean() < -1e-4
    assert abs(rel.mean()) < 1e-9

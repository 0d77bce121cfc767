"""Log-likelihood error of reduced-precision pruning arithmetics against FP64
(oracle/precision.py), on the CPU.

The FP64 restatement in oracle/precision.py must equal the oracle; then the
FP32 form in the engine's summation order and the split hi + lo TF32 form
must stay far inside the 1e-3 |delta lnL| budget, while the split hi + lo BF16
form loses more than an order of magnitude of accuracy to them, split FP16
loses more still, and plain BF16 misses the budget outright. (The engine's FP32 kernel is measured on the GPU against
FP64 by test_gpu_parity.py; this file pins the arithmetic comparison between
the tensor-core forms.)"""
import numpy as np
import pytest

import oracle
from oracle import precision


def test_bf16_rounding_is_round_to_nearest_even():
    x = np.array([1.0, 1.0 + 2.0 ** -8, 1.0 + 3 * 2.0 ** -8, 1.0 + 2.0 ** -9, -2.5e-3],
                 dtype=np.float32)
    got = precision.bf16_round(x)
    # 1 + 2^-8 is halfway between 1 and 1 + 2^-7: ties go to the even 1.
    np.testing.assert_array_equal(got[:4], np.array([1.0, 1.0, 1.0 + 2.0 ** -6, 1.0],
                                                    dtype=np.float32))
    assert abs(got[4] - x[4]) <= abs(x[4]) * 2.0 ** -8
    hi, lo = precision._split(np.array([0.1], np.float32))
    assert abs(float(hi[0]) + float(lo[0]) - float(np.float32(0.1))) <= 0.1 * 2.0 ** -16


def test_fp64_restatement_equals_oracle():
    r = precision.study(10, 300, 3, seed=5)
    assert r["lnl_fp64"] == pytest.approx(r["lnl_oracle"], rel=1e-12)


def test_precision_forms_order():
    r = precision.study(24, 2000, 6, seed=11)
    assert r["fp32"] < 1e-4
    assert r["tf32x3"] < 1e-4
    assert r["bf16x3"] > 10 * max(r["fp32"], r["tf32x3"])
    assert r["bf16"] > 1e-2
    # Reading the raw FP32 operand as the hi part truncates both parts toward
    # zero: a one-signed error that ends up worse than split BF16.
    assert r["tf32x3raw"] > r["bf16x3"]
    # Split FP16 (the kind::f16 form) has TF32's significand but a 5-bit
    # exponent: small partial entries and the lo remainders fall into FP16's
    # subnormals or to zero, and the split ends up worse than split BF16.
    assert r["fp16x3"] > r["bf16x3"]
    assert r["fp16x3"] > 1e-3


def test_fp16_rounding_keeps_subnormals_and_flushes_below():
    x = np.array([1.0, 1.0 + 2.0 ** -11, 1e-5, 2.0 ** -25, 2.0 ** -26], dtype=np.float32)
    got = precision.fp16_round(x)
    assert got[0] == 1.0 and got[1] == 1.0           # tie to even
    assert abs(got[2] - x[2]) <= 2.0 ** -25           # a subnormal: absolute spacing 2^-24
    assert got[3] == 0.0 and got[4] == 0.0            # half the smallest subnormal and below: zero

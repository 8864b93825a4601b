"""The FP64 near field's own exp and rsqrt (bit_b200/csrc/fp64math.cuh) against CUDA's on the
device, over 4M seeded arguments each: exp on [-707, 0] (and its small-argument form on
(-8, 0]), rsqrt on [1e-12, 1e6]."""
import pytest


@pytest.mark.gpu
def test_fp64_exp_and_rsqrt_agree_with_cuda(ctx):
    err = ctx.fp64_math_error(1 << 22)
    # each is within about an ulp of the exact value, as CUDA's are
    assert err["exp"] <= 2.0, err
    assert err["rsqrt"] <= 2.0, err

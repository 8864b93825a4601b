"""Device math and the device-side failure path.  The FP64 near field's own exp and rsqrt
(bit_b200/csrc/fp64math.cuh) against CUDA's on the device, over 4M seeded arguments each:
exp on [-707, 0] (and its small-argument form on (-8, 0]), rsqrt on [1e-12, 1e6].  The
bounded wait's give-up path, with a barrier that nothing completes."""
import numpy as np
import pytest


@pytest.mark.gpu
def test_fp64_exp_and_rsqrt_agree_with_cuda(ctx):
    err = ctx.fp64_math_error(1 << 22)
    # each is within about an ulp of the exact value, as CUDA's are
    assert err["exp"] <= 2.0, err
    assert err["rsqrt"] <= 2.0, err


@pytest.mark.gpu
def test_bounded_wait_gives_up_with_a_status_and_the_context_stays_usable(ctx):
    """The give-up path of the kernels' bounded waits, made to run out on purpose: a CTA
    waits on an mbarrier that nothing completes (no copy in flight, no fault, no hang).
    The call returns BIT_ERR_CUDA with the context's message, the device flag is cleared,
    and the same context then evaluates the golden case to the reference's values."""
    import bit_b200 as B
    from conftest import load_golden
    assert ctx.wait_check(1000) == 2  # BIT_ERR_CUDA
    msg = B.lib().bit_ctx_last_error(ctx.h).decode()
    assert "gave up" in msg and "16" in msg, msg
    g = load_golden("box2000")
    t = ctx.treemake(g["x"], g["y"], g["z"], int(g["maxmemb"]))
    t.treemoments(g["q"], int(g["nterms"]), w=g["w"])
    pot = t.treepotential(float(g["acc"]), float(g["del_"]), mode=B.REFERENCE)
    ref = g["coulomb"]
    assert np.linalg.norm(pot - ref) / np.linalg.norm(ref) < 1e-12
    t.treeempty()

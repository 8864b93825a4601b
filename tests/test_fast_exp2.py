"""exp2_fma (bit_b200/csrc/near.cu), the screened near field's FMA-pipe exponential,
emulated step for step in float32 on the CPU: its relative error stays within the bound
of the MUFU ex2.approx.f32 it stands in for (about 2^-22) on the range the near field
uses (x = -kappa r log2(e) <= 0), and the coefficients are those remez_exp2.py derives."""
import importlib.util
import os

import numpy as np

from conftest import ROOT

C = [float.fromhex(h) for h in ("0x1.000002p+0", "0x1.62e428p-1", "0x1.ebf918p-3",
                                "0x1.c6b6e4p-5", "0x1.3d0c52p-7", "0x1.5c08e6p-10")]
BIG = np.float32(12582912.0)


def f32(a):
    return np.asarray(a, dtype=np.float64).astype(np.float32)


def exp2_fma(x):
    x = np.maximum(f32(x), np.float32(-125.0))
    t = f32(x.astype(np.float64) + float(BIG))
    n = f32(t.astype(np.float64) - float(BIG))
    f = f32(x.astype(np.float64) - n.astype(np.float64))
    p = np.full(x.shape, np.float32(C[5]))
    for c in (C[4], C[3], C[2], C[1], C[0]):  # fmaf: one rounding of p * f + c
        p = f32(p.astype(np.float64) * f.astype(np.float64) + c)
    e = t.view(np.int32).astype(np.int64) - int(BIG.view(np.int32))
    return (p.view(np.int32).astype(np.int64) + (e << 23)).astype(np.int32).view(np.float32)


def test_relative_error_within_ex2_approx_bound():
    rng = np.random.default_rng(1)
    xs = np.concatenate([np.linspace(-125.0, 0.0, 2_000_001), -rng.exponential(3.0, 1_000_000),
                         -rng.uniform(0.0, 1e-3, 100_000)]).astype(np.float32)
    xs = xs[xs >= -125.0]
    got = exp2_fma(xs).astype(np.float64)
    want = np.exp2(xs.astype(np.float64))
    assert np.max(np.abs(got / want - 1.0)) < 2.0 ** -21.9


def test_integer_arguments_are_exact_powers():
    xs = -np.arange(0, 126, dtype=np.float32)
    got = exp2_fma(xs).astype(np.float64)
    assert np.max(np.abs(got / np.exp2(xs.astype(np.float64)) - 1.0)) < 2.0 ** -22


def test_coefficients_match_the_remez_derivation():
    spec = importlib.util.spec_from_file_location(
        "remez_exp2", os.path.join(ROOT, "bit_b200", "csrc", "remez_exp2.py"))
    m = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(m)
    c, _ = m.remez(5)
    assert [float(np.float32(float(v))) for v in c] == C

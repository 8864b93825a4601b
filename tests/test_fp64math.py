"""CPU checks of the constants of the FP64 near field's own exp (bit_b200/csrc/fp64math.cuh):
the 2^(j/64) table (leading double and trailing correction), the reduction constants and the
Taylor coefficients, each recomputed here to 80 digits."""
import math
import os
import re
from decimal import Decimal, getcontext

HDR = os.path.join(os.path.dirname(__file__), "..", "bit_b200", "csrc", "fp64math.cuh")


def _src():
    return open(HDR).read()


def test_exp_table_is_lead_and_trail_of_2_to_the_j_over_64():
    getcontext().prec = 80
    body = re.search(r"kExp2Tab64\[64\] = \{(.*?)\n\};", _src(), re.S).group(1)
    pairs = re.findall(r"\{([^{}]+)\}", body)
    assert len(pairs) == 64
    for j, p in enumerate(pairs):
        hi, lo = (float.fromhex(v.strip()) for v in p.split(","))
        exact = Decimal(2) ** (Decimal(j) / 64)
        assert hi == float(exact), j
        assert lo == float(exact - Decimal(hi)), j


def test_reduction_constants():
    getcontext().prec = 80
    s = _src()
    get = lambda name: float.fromhex(re.search(name + r" = ([0-9a-fx.p+-]+);", s).group(1))
    ln2 = Decimal(2).ln()
    assert get("kExpInvL") == float(64 / ln2)
    hi = get("kExpLhi")
    assert hi == float(ln2 / 64)
    assert get("kExpLlo") == float(ln2 / 64 - Decimal(hi))
    assert get("kRoundShift") == 1.5 * 2.0 ** 52


def test_taylor_coefficients():
    s = _src()
    body = s[s.index("e^r - 1 = r"):s.index("p *= r;")]
    coef = [float.fromhex(c) for c in re.findall(r"0x1\.[0-9a-f]+p-\d+", body)]
    assert coef == [1 / math.factorial(5), 1 / math.factorial(4), 1 / math.factorial(3)]
    # truncation of the degree-5 polynomial at |r| <= ln2 / 128, relative to e^r
    r = math.log(2) / 128
    assert r ** 6 / math.factorial(6) < 4e-17

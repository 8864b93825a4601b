"""bench.py's host-side helpers: the far-field flops per pair come from the generator, the
rooflines divide them by measured peaks, and the matched-accuracy parameters name valid
expansion orders.  No GPU."""
import importlib.util
import os

from conftest import ROOT


def bench():
    spec = importlib.util.spec_from_file_location("bench", os.path.join(ROOT, "bench.py"))
    b = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(b)
    return b


def test_far_flops_per_pair():
    b = bench()
    f = b.far_flops_per_pair(9)
    assert f["coulomb"] == 1459 and f["screened"] == 2414


def test_roofline_entries():
    b = bench()
    st = {"far_pairs": 1000, "t_far": 1e-3, "near_pairs": 5000, "t_near": 2e-3}
    r = b.roofline_far("fp64", "screened", st, 2414, 36.0)
    assert abs(r["achieved"] - 2414 * 1000 / 1e-3 / 1e12) < 1e-12
    assert abs(r["frac"] - r["achieved"] / 36.0) < 1e-12
    assert r["kernel"] == "k_far<9, SCREENED, double>" and "measured" in r["peak_source"]
    n = 1000
    r = b.roofline_near("mixed", "coulomb", st, n, 72.0)
    assert abs(r["achieved"] - 11 * (5000 - n) / 2e-3 / 1e12) < 1e-12
    assert r["bound"] == "fp32+mufu"


def test_matched_parameters():
    b = bench()
    for d in (b.MATCHED_C2, b.MATCHED_BIE):
        assert 1 <= d["nterms"] <= 10 and 0 < d["acc"] < 1 and d["maxmemb"] > 0
    assert sorted(b.MATCHED_BATCH_ACC) == [5, 7, 9]

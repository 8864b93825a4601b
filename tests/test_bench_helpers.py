"""bench.py's host-side helpers: the per-launch DRAM traffic it reports as
roofline.traffic comes from the committed launch-list profile, the far-field flops per
pair from the generator, and the FP32 peak from the sampled clock.  No GPU."""
import importlib.util
import os

from conftest import ROOT


def bench():
    spec = importlib.util.spec_from_file_location("bench", os.path.join(ROOT, "bench.py"))
    b = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(b)
    return b


def test_profiled_traffic_lines_parse():
    b = bench()
    for key in ("k_far_screened_f32", "k_near_screened_f32"):
        v = b.profiled_traffic(key)
        assert isinstance(v, int) and 10 ** 7 < v < 10 ** 10, (key, v)


def test_far_flops_and_peak():
    b = bench()
    f = b.far_flops_per_pair(9)
    assert f["coulomb"] == 1459 and f["screened"] == 2414
    p = b.fp32_peak_from_clock({"sm_mhz": 1965.0})
    assert abs(p["tflops"] - 148 * 128 * 2 * 1.965e9 / 1e12) < 1e-9
    assert abs(p["mufu_ops"] - 148 * 16 * 1.965e9) < 1.0

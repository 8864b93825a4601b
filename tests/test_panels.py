"""Box boundary panels (bit_panels_box) against the reference's setboundaries, from the
golden fixture made by running the reference build (tests/golden/make_golden.py).  Host
code only: no GPU."""
import numpy as np

from conftest import load_golden


def test_panels_match_setboundaries_bit_for_bit():
    import bit_b200 as B
    g = load_golden("panels_box")
    pan = B.panels_box(int(g["xp"]), int(g["yp"]), int(g["zp"]), float(g["dl"]), float(g["dh"]),
                       float(g["dd"]))
    got = B.panels_as_array(pan)
    assert got.shape == g["panels"].shape
    np.testing.assert_array_equal(got, g["panels"])
    # the 4 < z < 5 ring carries the reference's 0 reference potential
    assert (got[:, 10] == 0.0).any() and (got[:, 10] == -50.0).any()


def test_panel_count_query():
    import ctypes as C
    import bit_b200 as B
    n = C.c_int()
    assert B.lib().bit_panels_box(3, 4, 5, 1.0, 1.0, 1.0, None, C.byref(n)) == 0
    assert n.value == 2 * (3 * 4 + 5 * 4 + 3 * 5)
    assert B.lib().bit_panels_box(0, 4, 5, 1.0, 1.0, 1.0, None, C.byref(n)) == 1

"""panelconstantsreal on the device and the revived panel solve on the treecode GMRES."""
import numpy as np
import pytest

from conftest import load_golden

pytestmark = pytest.mark.gpu


def golden_panels(B):
    g = load_golden("panels_box")
    pan = B.panels_box(int(g["xp"]), int(g["yp"]), int(g["zp"]), float(g["dl"]), float(g["dh"]),
                       float(g["dd"]))
    return g, pan


def test_panel_matrix_matches_panelconstantsreal_bit_for_bit(ctx):
    import bit_b200 as B
    g, pan = golden_panels(B)
    A = ctx.panel_matrix(pan, float(g["del_"]))
    np.testing.assert_array_equal(A, g["A"])


def test_panel_solve_matches_the_dense_solve(ctx):
    """b = refpot + 0.5 sum q / r over particles inside the box; A sigma = b solved densely
    with the reference's matrix, against the treecode GMRES solve."""
    import bit_b200 as B
    g, pan = golden_panels(B)
    rng = np.random.default_rng(31)
    npart = 300
    x = rng.uniform(-0.8, 0.8, npart); y = rng.uniform(-1.2, 1.2, npart)
    z = rng.uniform(-5.0, 5.0, npart); q = rng.uniform(-1.0, 1.0, npart)
    P = B.panels_as_array(pan)
    mid = P[:, 11:14]
    r = np.sqrt(((mid[:, None, :] - np.stack([x, y, z], 1)[None, :, :]) ** 2).sum(-1))
    b = P[:, 10] + (0.5 / r * q[None, :]).sum(1)
    sigma_dense = np.linalg.solve(g["A"], b)
    sigma, info, st = ctx.panel_solve(pan, x, y, z, q, float(g["del_"]), nterms=10, acc=0.05,
                                      maxmemb=16, tol=1e-12)
    assert st == 0, info
    assert np.linalg.norm(sigma - sigma_dense) / np.linalg.norm(sigma_dense) < 1e-6
    assert np.allclose([p.str for p in pan], sigma)

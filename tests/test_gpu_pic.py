"""Device-resident time stepping (bit_pic_steps) against the reference's particle loop
restated on the CPU: per step treemake, treemoments, treeforce with
F = field * charge_constant * q (freespace_particles_tree, src/tree3d.cpp:2268-2335),
then vel_update and loc_update (:4842-4888)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

CC, INVMASS = 1.0, 1.0   # the nondimensional constants (src/constants.h:29-30)


def cpu_steps(orc, x, y, z, u, v, w, q, steps, dt, nterms, maxmemb, del_, acc):
    x, y, z, u, v, w = (a.copy() for a in (x, y, z, u, v, w))
    F = None
    for _ in range(steps):
        T = orc.Tree(x, y, z, maxmemb)
        T.compute_moments(q, nterms)
        fx, fy, fz = T.evaluate_force(del_, acc)
        F = [f * CC * q for f in (fx, fy, fz)]
        u = u + dt * F[0] * INVMASS
        v = v + dt * F[1] * INVMASS
        w = w + dt * F[2] * INVMASS
        x = x + dt * u
        y = y + dt * v
        z = z + dt * w
    return (x, y, z, u, v, w), F


def gpu_steps(ctx, x, y, z, u, v, w, q, steps, dt, nterms, maxmemb, del_, acc, prec):
    import torch
    import bit_b200 as B
    dev = torch.device("cuda", 0)
    arrs = [torch.tensor(a, dtype=torch.float64, device=dev) for a in (x, y, z, u, v, w)]
    qd = torch.tensor(q, dtype=torch.float64, device=dev)
    F = [torch.zeros(len(x), dtype=torch.float64, device=dev) for _ in range(3)]
    opts = B.PicOpts(steps, nterms, maxmemb, dt, del_, acc, CC, INVMASS, prec)
    torch.cuda.synchronize()
    ctx.pic_steps_device(len(x), [a.data_ptr() for a in arrs], qd.data_ptr(), opts,
                         [f.data_ptr() for f in F])
    return [a.cpu().numpy() for a in arrs], [f.cpu().numpy() for f in F]


def rel(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


@pytest.mark.parametrize("prec_name,tol", [("FP64", 1e-12), ("MIXED", 1e-6)])
def test_pic_steps_match_the_reference_loop(ctx, orc, prec_name, tol):
    import bit_b200 as B
    from bit_b200 import workloads
    x, y, z, q = workloads.uniform_cube(6000, seed=21)
    q = q * 1e-3
    rng = np.random.default_rng(22)
    u, v, w = (rng.uniform(-0.1, 0.1, 6000) for _ in range(3))
    args = (x, y, z, u, v, w, q, 3, 1e-2, 5, 100, 1e-4, 0.5)
    ref, Fref = cpu_steps(orc, *args)
    got, F = gpu_steps(ctx, *args, getattr(B, prec_name))
    # the particles moved, and the GPU followed the reference loop
    assert rel(ref[0], x) > 1e-4
    for a, b in zip(got, ref):
        assert rel(a, b) < tol
    for a, b in zip(F, Fref):
        assert rel(a, b) < (tol if prec_name == "FP64" else 1e-5)


def test_pic_zero_steps_leave_particles_alone(ctx):
    import bit_b200 as B
    from bit_b200 import workloads
    x, y, z, q = workloads.uniform_cube(500, seed=3)
    zero = np.zeros(500)
    got, _ = gpu_steps(ctx, x, y, z, zero, zero, zero, q, 0, 0.1, 4, 50, 1e-4, 0.5, B.FP64)
    np.testing.assert_array_equal(got[0], x)

"""FP64 direct sums on the device (bit_direct_potential) against the oracle's direct sums
(shielded_pot_particle_ds, src/tree3d.cpp:1966-2016, and the Coulomb / regularised forms)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = 1e-12  # relative L2: same FP64 formula, different summation order and libm


@pytest.mark.parametrize("kernel", ["COULOMB", "SCREENED", "SCREENED_REG"])
@pytest.mark.parametrize("n,m", [(5000, 300), (40000, 257), (1, 1)])
def test_direct_matches_oracle(ctx, orc, kernel, n, m):
    import bit_b200 as B
    from bit_b200 import workloads
    x, y, z, q = workloads.clustered_blobs(n, seed=n + m)
    tg = workloads.sample_targets(n, min(m, n), seed=3)
    p = B.params(getattr(B, kernel), B.CONSISTENT, B.FP64, del_=1e-4, kappa=1.5)
    got = ctx.direct(x, y, z, q, p, tg)
    po = orc.params(getattr(orc, kernel), orc.MODE_CONSISTENT, del_=1e-4, kappa=1.5)
    ref = orc.direct(x, y, z, q, po, tg)
    if n == 1:
        np.testing.assert_array_equal(got, 0.0)
        return
    assert np.linalg.norm(got - ref) / np.linalg.norm(ref) < TOL


def test_direct_coincident_particles(ctx, orc):
    """Coincident sources: the regularised sums skip r^2 + del <= 1e-14 like the oracle."""
    import bit_b200 as B
    x = np.array([0.0, 0.0, 1.0, 1.0, 0.5]); y = np.zeros(5); z = np.zeros(5)
    q = np.array([1.0, 2.0, -1.0, 0.5, 3.0])
    tg = np.arange(5, dtype=np.int32)
    for k in ("COULOMB", "SCREENED_REG"):
        p = B.params(getattr(B, k), B.CONSISTENT, B.FP64, del_=0.0, kappa=1.0)
        got = ctx.direct(x, y, z, q, p, tg)
        ref = orc.direct(x, y, z, q, orc.params(getattr(orc, k), orc.MODE_CONSISTENT, kappa=1.0), tg)
        np.testing.assert_allclose(got, ref, rtol=1e-14)


def test_direct_rejects_bad_target(ctx):
    import bit_b200 as B
    x = np.zeros(4)
    with pytest.raises(B.BitError):
        ctx.direct(x, x, x, x, B.params(), [0, 4])


def test_streamed_writer_from_device_matches_host_writer(tmp_path, ctx):
    """bit_write_potential_device (chunked, overlapped copies) writes the same bytes."""
    import torch
    import bit_b200 as B
    rng = np.random.default_rng(5)
    n = 150_000  # more than two streamed chunks
    x, y, z, pot = (rng.standard_normal(n) for _ in range(4))
    B.write_potential(str(tmp_path / "host.txt"), x, y, z, pot)
    d = [torch.tensor(a, dtype=torch.float64, device="cuda") for a in (x, y, z, pot)]
    torch.cuda.synchronize()
    ctx.write_potential_device(str(tmp_path / "dev.txt"), n, *[a.data_ptr() for a in d])
    assert (tmp_path / "dev.txt").read_bytes() == (tmp_path / "host.txt").read_bytes()

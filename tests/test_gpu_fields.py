"""Fields and direct sums on the GPU against the reference build (oracle/_ref):
treeforce with KERNEL_ORDER > 0 (src/tree3d.cpp:456-810, 73-97), the screened 2-D field of
shielded_treeforce (:3268-3408, 2745-2973), and the field direct sums
force_particle_ds_reg / force_particle_ds_noreg (:298-330, 182-213)."""
import numpy as np
import pytest

import bit_b200 as B
from bit_b200 import workloads

pytestmark = pytest.mark.gpu

TOL = 1e-12  # relative L2 / max-norm against the reference's FP64 results


def close(a, b, tol=TOL):
    a, b = np.asarray(a), np.asarray(b)
    scale = np.max(np.abs(b))
    return np.linalg.norm(a - b) / np.linalg.norm(b) < tol and np.max(np.abs(a - b)) < tol * scale


def ref_or_skip(del_=0.01, korder=0):
    from oracle import ref
    if not ref.available(del_, korder):
        pytest.skip("reference build not present")
    return ref


@pytest.mark.parametrize("korder", [1, 2])
@pytest.mark.parametrize("nterms", [3, 6, 9])
def test_kernel_order_force_matches_reference(ctx, korder, nterms):
    ref = ref_or_skip(0.01, korder)
    x, y, z, q = workloads.clustered_blobs(3000, seed=21)
    R = ref.RefTree(x, y, z, q, nterms, 100, del_=0.01, korder=korder)
    R.moments()
    gx, gy, gz = R.force(0.5)
    R.close()
    t = ctx.treemake(x, y, z, 100)
    t.treemoments(q, nterms)
    fx, fy, fz = t.field(B.FIELD_COULOMB, acc=0.5, del_=0.01, kernel_order=korder)
    t.treeempty()
    for a, b in ((fx, gx), (fy, gy), (fz, gz)):
        assert close(a, b), (korder, nterms)


def test_kernel_order_changes_the_field(ctx):
    """KERNEL_ORDER 1 is not the order-0 field (the correction is really applied)."""
    x, y, z, q = workloads.uniform_cube(2000, seed=2)
    t = ctx.treemake(x, y, z, 100)
    t.treemoments(q, 5)
    f0 = t.field(B.FIELD_COULOMB, acc=0.5, del_=0.01, kernel_order=0)[0]
    f1 = t.field(B.FIELD_COULOMB, acc=0.5, del_=0.01, kernel_order=1)[0]
    t.treeempty()
    assert np.linalg.norm(f1 - f0) / np.linalg.norm(f0) > 1e-4


@pytest.mark.parametrize("nterms", [2, 5, 9])
@pytest.mark.parametrize("kappa", [0.5, 2.0])
def test_screened_field_matches_reference(ctx, nterms, kappa):
    ref = ref_or_skip()
    x, y, z, q = workloads.clustered_blobs(3000, seed=22)
    R = ref.RefTree(x, y, z, q, nterms, 100, del_=0.01)
    R.moments()
    gx, gy, gz = R.screened_field(kappa, 0.5)
    R.close()
    t = ctx.treemake(x, y, z, 100)
    t.treemoments(q, nterms)
    fx, fy, fz = t.field(B.FIELD_SCREENED, acc=0.5, kappa=kappa, mac_del=0.01)
    t.treeempty()
    assert close(fx, gx) and close(fy, gy)
    assert not fz.any() and not gz.any()


def test_screened_field_is_fp64_only(ctx):
    x, y, z, q = workloads.uniform_cube(500, seed=3)
    t = ctx.treemake(x, y, z, 100)
    t.treemoments(q, 4)
    with pytest.raises(B.BitError):
        t.field(B.FIELD_SCREENED, acc=0.5, kappa=1.0, precision=B.MIXED)
    with pytest.raises(B.BitError):
        t.field(B.FIELD_COULOMB, acc=0.5, del_=0.01, kernel_order=1, precision=B.MIXED)
    t.treeempty()


@pytest.mark.parametrize("korder", [0, 1, 2])
def test_direct_field_reg_matches_reference(ctx, korder):
    ref = ref_or_skip(0.01, korder)
    x, y, z, q = workloads.clustered_blobs(20000, seed=23)
    tg = workloads.sample_targets(len(x), 300, seed=1)
    g = ref.ds_force_reg(x, y, z, q, tg, del_=0.01, korder=korder)
    f = ctx.direct_field(x, y, z, q, tg, del_=0.01, regularised=True, kernel_order=korder)
    for a, b in zip(f, g):
        assert close(a, b)


def test_direct_field_noreg_matches_reference(ctx):
    ref = ref_or_skip()
    x, y, z, q = workloads.uniform_cube(20000, seed=24)
    tg = workloads.sample_targets(len(x), 300, seed=2)
    g = ref.ds_force_noreg(x, y, z, q, tg)
    f = ctx.direct_field(x, y, z, q, tg, regularised=False)
    for a, b in zip(f, g):
        assert close(a, b)

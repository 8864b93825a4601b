"""Forests: many independent systems in one tree (bit_forest_*).

Every system's subtree must be the tree the reference's treemake builds for that system
alone (walked in parallel from both roots, bit for bit), and every system's potential
must equal both the oracle's single-system evaluation (FP64 within 1e-12, mixed within
1e-6) and a separate single-system GPU evaluation of it, bit for bit (the same result
alone and in the mix).
"""
import numpy as np
import pytest

from test_gpu_tree import assert_same_bits

pytestmark = pytest.mark.gpu


def make_systems(sizes, seed):
    from bit_b200 import workloads
    rng = np.random.default_rng(seed)
    xs, ys, zs, qs = [], [], [], []
    for i, n in enumerate(sizes):
        gen = workloads.clustered_blobs if i % 2 else workloads.uniform_cube
        x, y, z, q = gen(n, seed=seed * 100 + i)
        shift = rng.uniform(-3, 3, 3)  # systems overlap in space: they must not interact
        xs.append(x + shift[0]); ys.append(y + shift[1]); zs.append(z + shift[2]); qs.append(q)
    return xs, ys, zs, qs


def walk_pairs(ch_a, root_a, ch_b, root_b):
    """Node pairs of two trees walked together in children-slot order."""
    out, stk = [], [(root_a, root_b)]
    while stk:
        a, b = stk.pop()
        out.append((a, b))
        ca, cb = ch_a[a], ch_b[b]
        np.testing.assert_array_equal(ca == -1, cb == -1)
        for k in range(7, -1, -1):
            if ca[k] != -1:
                stk.append((ca[k], cb[k]))
    return out


SIZES = [3000, 500, 7000, 2, 1200, 40]
MAXMEMB = [50, 20, 100, 10, 30, 40]


def test_forest_subtrees_match_treemake(ctx, orc):
    xs, ys, zs, _ = make_systems(SIZES, 1)
    F = ctx.forest(np.concatenate(xs), np.concatenate(ys), np.concatenate(zs), SIZES, MAXMEMB)
    nm, ch, f, mem = F.export()
    off = np.concatenate([[0], np.cumsum(nm)])
    nodes = 0
    for s in range(len(SIZES)):
        T = orc.Tree(xs[s], ys[s], zs[s], MAXMEMB[s])
        pairs = walk_pairs(ch, s, T.children, 0)
        assert len(pairs) == T.numtree
        nodes += len(pairs)
        for a, b in pairs:
            assert nm[a] == T.nummemb[b]
            assert_same_bits(f[a], T.fields[b])
            np.testing.assert_array_equal(mem[off[a]:off[a + 1]] - F.offsets[s], T.members(b))
    assert nodes == F.numtree


def system_params(B, s, prec):
    kinds = [
        B.params(B.COULOMB, B.CONSISTENT, prec, del_=1e-4, acc=0.5),
        B.params(B.SCREENED, B.REFERENCE, prec, kappa=1.0, mac_del=1e-3, acc=0.6),
        B.params(B.SCREENED_REG, B.CONSISTENT, prec, del_=1e-3, kappa=2.0, acc=0.4),
        B.params(B.COULOMB, B.REFERENCE, prec, del_=1e-2, acc=0.7),
        B.params(B.SCREENED, B.CONSISTENT, prec, kappa=0.5, acc=0.5),
        B.params(B.COULOMB, B.CONSISTENT, prec, del_=0.0, acc=0.3),
    ]
    return kinds[s % len(kinds)]


def oracle_params(orc, p):
    return orc.params(p.kernel, p.mode, del_=p.del_, mac_del=p.mac_del, kappa=p.kappa,
                      acc=p.acc, intg=p.intg)


NTERMS = [6, 9, 4, 3, 8, 5]


@pytest.mark.parametrize("prec_name,tol", [("FP64", 1e-12), ("MIXED", 1e-6)])
def test_forest_potentials_match_oracle_and_alone(ctx, orc, prec_name, tol):
    import bit_b200 as B
    prec = getattr(B, prec_name)
    xs, ys, zs, qs = make_systems(SIZES, 2)
    F = ctx.forest(np.concatenate(xs), np.concatenate(ys), np.concatenate(zs), SIZES, MAXMEMB)
    F.set_charges(np.concatenate(qs))
    F.moments(NTERMS)
    prm = [system_params(B, s, prec) for s in range(len(SIZES))]
    got = F.evaluate(prm)
    st = F.stats()
    # several (nterms, kernel) classes, each field run as one work-queue launch
    assert st["far_launches"] == 1 and st["near_launches"] == 1
    for s in range(len(SIZES)):
        mine = F.system(s, got)
        T = orc.Tree(xs[s], ys[s], zs[s], MAXMEMB[s])
        T.compute_moments(qs[s], NTERMS[s])
        ref = T.evaluate(oracle_params(orc, prm[s]))
        scale = max(np.linalg.norm(ref), 1e-300)
        assert np.linalg.norm(mine - ref) / scale < tol, (s, np.linalg.norm(mine - ref) / scale)
        alone = ctx.treemake(xs[s], ys[s], zs[s], MAXMEMB[s])
        alone.treemoments(qs[s], NTERMS[s])
        np.testing.assert_array_equal(mine, alone.evaluate(prm[s]))
        alone.treeempty()


@pytest.mark.parametrize("prec_name", ["FP64", "MIXED"])
def test_work_queue_equals_class_launches(prec_name):
    """The persistent work-queue kernels (one launch per field over all groups) give the
    results of one launch per (nterms, kernel) class bit for bit."""
    import bit_b200 as B
    prec = getattr(B, prec_name)
    xs, ys, zs, qs = make_systems(SIZES, 5)
    c = B.Context()
    try:
        F = c.forest(np.concatenate(xs), np.concatenate(ys), np.concatenate(zs), SIZES, MAXMEMB)
        F.set_charges(np.concatenate(qs))
        F.moments(NTERMS)
        prm = [system_params(B, s, prec) for s in range(len(SIZES))]
        c.set_work_queue(True)
        q = F.evaluate(prm)
        assert F.stats()["far_launches"] == 1
        c.set_work_queue(False)
        k = F.evaluate(prm)
        st = F.stats()
        assert st["far_launches"] >= 2 and st["near_launches"] >= 2
        np.testing.assert_array_equal(q, k)
    finally:
        c.close()


def test_forest_one_parameter_set_for_all(ctx):
    """One EvalParams broadcast to every system equals passing it per system."""
    import bit_b200 as B
    xs, ys, zs, qs = make_systems([800, 1500, 300], 3)
    F = ctx.forest(np.concatenate(xs), np.concatenate(ys), np.concatenate(zs), [800, 1500, 300], 60)
    F.set_charges(np.concatenate(qs))
    F.moments(7)
    p = B.params(B.COULOMB, B.CONSISTENT, B.MIXED, del_=1e-4, acc=0.5)
    a = F.evaluate(p)
    b = F.evaluate([p, p, p])
    np.testing.assert_array_equal(a, b)
    st = F.stats()
    assert st["far_launches"] == 1 and st["near_launches"] == 1


def test_forest_rejects_bad_input(ctx):
    import bit_b200 as B
    x = np.zeros(10)
    with pytest.raises(B.BitError):
        ctx.forest(x, x, x, [5, 0, 5], 10)
    xs, ys, zs, qs = make_systems([100, 100], 4)
    F = ctx.forest(np.concatenate(xs), np.concatenate(ys), np.concatenate(zs), [100, 100], 10)
    F.set_charges(np.concatenate(qs))
    with pytest.raises(B.BitError):
        F.moments([4, 11])
    F.moments([4, 5])
    with pytest.raises(B.BitError):  # mixed precisions in one call
        F.evaluate([B.params(precision=B.FP64), B.params(precision=B.MIXED)])


@pytest.mark.parametrize("group", [256, 1024])
def test_packed_leaf_groups_match_oracle(orc, group):
    """Packing consecutive small leaves into one group changes only the grouping of work:
    FP64 stays within 1e-12 of the oracle, every target keeps its own interaction lists,
    and a forest still gives each system its single-system result."""
    import bit_b200 as B
    ctx = B.Context()
    try:
        ctx.set_group_size(group)
        xs, ys, zs, qs = make_systems(SIZES, 5)
        F = ctx.forest(np.concatenate(xs), np.concatenate(ys), np.concatenate(zs), SIZES, MAXMEMB)
        F.set_charges(np.concatenate(qs))
        F.moments(NTERMS)
        prm = [system_params(B, s, B.FP64) for s in range(len(SIZES))]
        got = F.evaluate(prm)
        for s in range(len(SIZES)):
            T = orc.Tree(xs[s], ys[s], zs[s], MAXMEMB[s])
            T.compute_moments(qs[s], NTERMS[s])
            ref = T.evaluate(oracle_params(orc, prm[s]))
            scale = max(np.linalg.norm(ref), 1e-300)
            assert np.linalg.norm(F.system(s, got) - ref) / scale < 1e-12, s
        # per-target lists of a packed single-system tree equal the reference traversal
        x, y, z, q = xs[0], ys[0], zs[0], qs[0]
        t = ctx.treemake(x, y, z, 50)
        t.treemoments(q, 5)
        p = B.params(B.COULOMB, B.CONSISTENT, B.FP64, del_=1e-4, acc=0.5)
        t.evaluate(p)
        T = orc.Tree(x, y, z, 50)
        T.compute_moments(q, 5)
        po = orc.params(orc.COULOMB, orc.MODE_CONSISTENT, del_=1e-4, acc=0.5)
        for i in (0, 17, 1234, len(x) - 1):
            node, kind = t.target_lists(p, i)
            rn, rk = T.target_lists(po, i)
            np.testing.assert_array_equal(node, rn)
            np.testing.assert_array_equal(kind, rk)
        mixed = t.evaluate(B.params(B.COULOMB, B.CONSISTENT, B.MIXED, del_=1e-4, acc=0.5))
        ref = T.evaluate(po)
        assert np.linalg.norm(mixed - ref) / np.linalg.norm(ref) < 1e-6
    finally:
        ctx.close()


def test_group_size_is_validated(ctx):
    import bit_b200 as B
    with pytest.raises(B.BitError):
        ctx.set_group_size(5000)
    with pytest.raises(B.BitError):
        ctx.set_group_size(10)

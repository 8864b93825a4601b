"""GPU tree build (bit_tree_build) against the reference's treemake: bit for bit."""
import numpy as np
import pytest

from conftest import GOLDEN_CASES, load_golden

pytestmark = pytest.mark.gpu


def bits(a):
    return np.ascontiguousarray(a, dtype=np.float64).view(np.int64)


def assert_same_bits(a, b):
    """Bit-for-bit equal, except that any NaN equals any NaN: 0/0 aspect ratios of
    zero-extent boxes are NaN on both sides, but x86 and the GPU write different NaN
    payloads; every comparison on them is false either way, so the tree is the same."""
    a = np.ascontiguousarray(a, dtype=np.float64)
    b = np.ascontiguousarray(b, dtype=np.float64)
    both_nan = np.isnan(a) & np.isnan(b)
    np.testing.assert_array_equal(np.where(both_nan, 0, bits(a)), np.where(both_nan, 0, bits(b)))


def assert_same_tree(tree, nm, ch, f, mem):
    gnm, gch, gf, gmem = tree.export()
    assert tree.numtree == len(nm)
    np.testing.assert_array_equal(gnm, nm)
    np.testing.assert_array_equal(gch, ch)
    assert_same_bits(gf, f)
    np.testing.assert_array_equal(gmem, mem)


@pytest.mark.parametrize("name", GOLDEN_CASES)
def test_tree_matches_reference_golden(ctx, name):
    g = load_golden(name)
    t = ctx.treemake(g["x"], g["y"], g["z"], int(g["maxmemb"]))
    assert_same_tree(t, g["nummemb"], g["children"], g["fields"], g["members"])


@pytest.mark.parametrize("dist,n,maxmemb", [("uniform", 20000, 500), ("clustered", 60000, 300),
                                            ("clustered", 200000, 1000), ("uniform", 5000, 7)])
def test_tree_matches_oracle(ctx, orc, dist, n, maxmemb):
    from bit_b200 import workloads
    gen = workloads.uniform_cube if dist == "uniform" else workloads.clustered_blobs
    x, y, z, _ = gen(n, seed=n)
    t = ctx.treemake(x, y, z, maxmemb)
    T = orc.Tree(x, y, z, maxmemb)
    mem = np.concatenate([T.members(i) for i in range(T.numtree)])
    assert_same_tree(t, T.nummemb, T.children, T.fields, mem)


def test_tree_anisotropic_shapes(ctx, orc):
    """Slabs and needles drive the y-only, z-only and sibling z-split branches."""
    rng = np.random.default_rng(0)
    for sx, sy, sz in [(1, 1, 0.05), (1, 0.05, 1), (0.05, 1, 1), (1, 0.1, 0.01), (0.01, 0.1, 1)]:
        n = 8000
        x = rng.uniform(-sx, sx, n); y = rng.uniform(-sy, sy, n); z = rng.uniform(-sz, sz, n)
        t = ctx.treemake(x, y, z, 40)
        T = orc.Tree(x, y, z, 40)
        mem = np.concatenate([T.members(i) for i in range(T.numtree)])
        assert_same_tree(t, T.nummemb, T.children, T.fields, mem)


def test_tree_small_cases(ctx, orc):
    for n, mm in [(1, 1), (2, 1), (3, 1), (7, 3), (33, 2), (100, 100), (101, 100)]:
        rng = np.random.default_rng(n)
        x, y, z = rng.uniform(-1, 1, (3, n))
        t = ctx.treemake(x, y, z, mm)
        T = orc.Tree(x, y, z, mm)
        mem = np.concatenate([T.members(i) for i in range(T.numtree)])
        assert_same_tree(t, T.nummemb, T.children, T.fields, mem)


def test_tree_degenerate_and_invalid(ctx):
    import bit_b200
    with pytest.raises(bit_b200.BitError) as e:
        ctx.treemake(np.zeros(10), np.zeros(10), np.zeros(10), 3)
    assert e.value.status == 5
    x = np.array([0.0, np.nan, 1.0])
    with pytest.raises(bit_b200.BitError) as e:
        ctx.treemake(x, x, x, 1)
    assert e.value.status == 1
    # the context stays usable after an error
    t = ctx.treemake(np.arange(5.0), np.arange(5.0) ** 2, np.ones(5), 2)
    assert t.numtree >= 3


def test_duplicates_below_leaf_size(ctx, orc):
    """Coincident particles are fine while a leaf can hold them."""
    rng = np.random.default_rng(1)
    base = rng.uniform(-1, 1, (500, 3))
    p = np.concatenate([base, base[:50], base[:50]])
    t = ctx.treemake(p[:, 0], p[:, 1], p[:, 2], 20)
    T = orc.Tree(p[:, 0], p[:, 1], p[:, 2], 20)
    mem = np.concatenate([T.members(i) for i in range(T.numtree)])
    assert_same_tree(t, T.nummemb, T.children, T.fields, mem)

"""GPU evaluation (moments, lists, far and near field) against the oracle.

Bars: the plain FP64 GPU path matches the FP64 CPU treecode to 1e-12 relative (L2 and
max-norm relative to max |value|); the interaction lists match exactly; the mixed path
stays within 1e-6 relative L2 of the FP64 path at the same lists.
"""
import numpy as np
import pytest

from conftest import GOLDEN_CASES, load_golden

pytestmark = pytest.mark.gpu

TOL64 = 1e-12
TOL_MIXED = 1e-6


def rel(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return max(np.linalg.norm(a - b) / np.linalg.norm(b), np.abs(a - b).max() / np.abs(b).max())


def both(ctx, orc, x, y, z, q, nterms, maxmemb, w=None):
    t = ctx.treemake(x, y, z, maxmemb)
    t.treemoments(q, nterms, w=w)
    T = orc.Tree(x, y, z, maxmemb)
    T.compute_moments(q, nterms, w=w)
    return t, T


def gp(bit_b200, **kw):
    return bit_b200.params(**kw)


@pytest.mark.parametrize("name", GOLDEN_CASES)
def test_reference_mode_matches_golden(ctx, name):
    """Reference-mode potentials / force on the reference's own outputs."""
    import bit_b200 as B
    g = load_golden(name)
    t = ctx.treemake(g["x"], g["y"], g["z"], int(g["maxmemb"]))
    t.treemoments(g["q"], int(g["nterms"]), w=g["w"])
    d, acc, kappa = float(g["del_"]), float(g["acc"]), float(g["kappa"])
    np.testing.assert_allclose(t.export_moments(), g["moments"], rtol=1e-12,
                               atol=1e-13 * np.abs(g["moments"]).max())
    assert rel(t.treepotential(acc, d, mode=B.REFERENCE), g["coulomb"]) < TOL64
    assert rel(t.shielded_treepot(kappa, acc, mode=B.REFERENCE, mac_del=d), g["screened"]) < TOL64
    assert rel(t.treepotential(acc, d, mode=B.REFERENCE, points=g["points"]),
               g["coulomb_points"]) < TOL64
    assert rel(t.shielded_treepot(kappa, acc, mode=B.REFERENCE, mac_del=d, points=g["points"]),
               g["screened_points"]) < TOL64
    f = np.stack(t.treeforce(acc, d))
    assert rel(f, g["force"]) < TOL64


@pytest.mark.parametrize("nterms", range(1, 11))
def test_every_order_matches_oracle(ctx, orc, nterms):
    import bit_b200 as B
    from bit_b200 import workloads
    x, y, z, q = workloads.clustered_blobs(6000, seed=nterms)
    t, T = both(ctx, orc, x, y, z, q, nterms, 150)
    for kern, kw in [(B.COULOMB, dict(del_=1e-4)), (B.SCREENED, dict(kappa=1.5)),
                     (B.SCREENED_REG, dict(kappa=0.7, del_=1e-3))]:
        for mode in (B.REFERENCE, B.CONSISTENT):
            p = B.params(kern, mode, B.FP64, acc=0.6, **kw)
            po = orc.params(kern, mode, acc=0.6, **kw)
            assert rel(t.evaluate(p), T.evaluate(po)) < TOL64, (kern, mode)
    if nterms <= 10:
        f = np.stack(t.treeforce(0.6, 1e-4))
        fo = np.stack(T.evaluate_force(1e-4, 0.6))
        assert rel(f, fo) < TOL64


def test_lists_match_reference_traversal(ctx, orc):
    import bit_b200 as B
    from bit_b200 import workloads
    x, y, z, q = workloads.clustered_blobs(20000, seed=5)
    t, T = both(ctx, orc, x, y, z, q, 5, 200)
    for kern, po, p in [
        ("coulomb", orc.params(orc.COULOMB, acc=0.7, del_=2.5e-5),
         B.params(B.COULOMB, acc=0.7, del_=2.5e-5)),
        ("screened", orc.params(orc.SCREENED, acc=0.5, mac_del=0.01, kappa=1.0),
         B.params(B.SCREENED, acc=0.5, mac_del=0.01, kappa=1.0)),
    ]:
        for tg in workloads.sample_targets(20000, 40, seed=3):
            gn, gk = t.target_lists(p, int(tg))
            on, ok = T.target_lists(po, int(tg))
            np.testing.assert_array_equal(gn, on, err_msg=kern)
            np.testing.assert_array_equal(gk, ok, err_msg=kern)
    # interaction counts agree with the oracle's traversal
    t.evaluate(B.params(B.COULOMB, acc=0.7, del_=2.5e-5))
    st = t.stats()
    nf, nn, nl = T.count(orc.params(orc.COULOMB, acc=0.7, del_=2.5e-5))
    assert st["far_pairs"] == nf
    assert st["near_pairs"] - 20000 == nn  # the GPU count includes each target's self pair


@pytest.mark.parametrize("kern", ["coulomb", "screened"])
def test_mixed_precision_close_to_fp64(ctx, kern):
    import bit_b200 as B
    from bit_b200 import workloads
    x, y, z, q = workloads.clustered_blobs(100000, seed=7)
    t = ctx.treemake(x, y, z, 1000)
    t.treemoments(q, 9)
    kw = dict(del_=2.5e-5) if kern == "coulomb" else dict(kappa=1.0)
    k = B.COULOMB if kern == "coulomb" else B.SCREENED
    p64 = t.evaluate(B.params(k, B.CONSISTENT, B.FP64, acc=0.7, **kw))
    p32 = t.evaluate(B.params(k, B.CONSISTENT, B.MIXED, acc=0.7, **kw))
    assert workloads.rel_l2(p32, p64) < TOL_MIXED


def test_mixed_force_close_to_fp64(ctx):
    import bit_b200 as B
    from bit_b200 import workloads
    x, y, z, q = workloads.uniform_cube(30000, seed=8)
    t = ctx.treemake(x, y, z, 300)
    t.treemoments(q, 7)
    f64 = np.stack(t.treeforce(0.5, 1e-4, B.FP64))
    f32 = np.stack(t.treeforce(0.5, 1e-4, B.MIXED))
    assert workloads.rel_l2(f32, f64) < 1e-5


def test_error_against_direct_sum_decreases(ctx, orc):
    """tests/treecode.cpp:84-127 on the GPU: error vs the direct sum shrinks with nterms."""
    import bit_b200 as B
    from bit_b200 import workloads
    x, y, z, q = workloads.uniform_cube(20000, seed=1)
    tg = workloads.sample_targets(20000, 500, seed=1)
    po = orc.params(orc.COULOMB, orc.MODE_CONSISTENT, del_=1e-4, acc=0.5)
    ds = orc.direct(x, y, z, q, po, tg)
    t = ctx.treemake(x, y, z, 500)
    errs = []
    for nterms in (2, 4, 7, 10):
        t.treemoments(q, nterms)
        pot = t.evaluate(B.params(B.COULOMB, B.CONSISTENT, B.FP64, del_=1e-4, acc=0.5))
        errs.append(workloads.rel_l2(pot[tg], ds))
    assert all(b <= a for a, b in zip(errs, errs[1:])), errs


def test_repeat_and_stats(ctx):
    """Same inputs give bit-identical results; stats report the phases."""
    import bit_b200 as B
    from bit_b200 import workloads
    x, y, z, q = workloads.uniform_cube(20000, seed=2)
    t = ctx.treemake(x, y, z, 500)
    t.treemoments(q, 7)
    p = B.params(B.COULOMB, B.CONSISTENT, B.MIXED, del_=1e-4, acc=0.5)
    a = t.evaluate(p)
    b = t.evaluate(p)
    np.testing.assert_array_equal(a, b)
    st = t.stats()
    assert st["numtree"] == t.numtree and st["far_pairs"] > 0 and st["t_far"] > 0


def test_evaluate_into_a_caller_buffer(ctx):
    """evaluate(out=...) writes the same bits into the caller's array and returns it, for
    particles and points; a wrong dtype or length is refused before anything runs."""
    import bit_b200 as B
    from bit_b200 import workloads
    x, y, z, q = workloads.uniform_cube(20000, seed=3)
    t = ctx.treemake(x, y, z, 500)
    t.treemoments(q, 7)
    p = B.params(B.SCREENED, B.CONSISTENT, B.MIXED, kappa=1.5, acc=0.5)
    buf = np.full(20000, 7.0)
    got = t.evaluate(p, out=buf)
    assert got is buf
    np.testing.assert_array_equal(buf, t.evaluate(p))
    pts = np.random.default_rng(4).uniform(0.0, 1.0, (300, 3))
    pbuf = np.empty(300)
    np.testing.assert_array_equal(t.evaluate(p, points=pts, out=pbuf), t.evaluate(p, points=pts))
    with pytest.raises(ValueError):
        t.evaluate(p, out=np.zeros(20000, dtype=np.float32))
    with pytest.raises(ValueError):
        t.evaluate(p, out=np.zeros(19999))


def test_whole_pipeline_host_buffers(ctx, orc):
    import bit_b200 as B
    from bit_b200 import workloads
    x, y, z, q = workloads.uniform_cube(20000, seed=1)
    p = B.params(B.COULOMB, B.REFERENCE, B.FP64, del_=1e-4, acc=0.5)
    pot = ctx.treecode_potential(x, y, z, q, 7, 500, p)
    T = orc.Tree(x, y, z, 500)
    T.compute_moments(q, 7)
    assert rel(pot, T.evaluate(orc.params(orc.COULOMB, orc.MODE_REFERENCE, del_=1e-4, acc=0.5))) < TOL64


def test_acc_zero_is_the_direct_sum_through_the_fallback_lists(ctx, orc):
    """acc = 0 accepts no cluster: every leaf is a near entry of every group, far more than
    the first build's estimated arrays hold, so the lists come from the count / scan / fill
    passes, and the potential is the FP64 direct sum."""
    import bit_b200 as B
    from bit_b200 import workloads
    x, y, z, q = workloads.uniform_cube(20000, seed=7)
    t = ctx.treemake(x, y, z, 8)
    t.treemoments(q, 3)
    got = t.evaluate(B.params(B.COULOMB, B.CONSISTENT, B.FP64, del_=1e-4, acc=0.0))
    assert t.stats()["list_fallback"] == 1
    assert t.stats()["far_pairs"] == 0
    tg = workloads.sample_targets(20000, 400, seed=2)
    ds = orc.direct(x, y, z, q, orc.params(orc.COULOMB, orc.MODE_CONSISTENT, del_=1e-4), tg)
    assert rel(got[tg], ds) < TOL64


def test_lists_past_the_estimated_arena_fall_back_exactly(ctx, orc):
    """Small leaves and a strict MAC give more near entries than the first build's
    per-group allowance: the in-place pass runs out of room and the build falls back; the
    result still matches the oracle, and the next build is sized from this one."""
    import bit_b200 as B
    from bit_b200 import workloads
    x, y, z, q = workloads.uniform_cube(20000, seed=8)
    t, T = both(ctx, orc, x, y, z, q, 4, 32)
    p = B.params(B.COULOMB, B.CONSISTENT, B.FP64, del_=1e-4, acc=0.1)
    got = t.evaluate(p)
    assert t.stats()["list_fallback"] == 1
    ref = T.evaluate(orc.params(orc.COULOMB, orc.MODE_CONSISTENT, del_=1e-4, acc=0.1))
    assert rel(got, ref) < TOL64
    # a different MAC rebuilds the lists, sized from the last totals: no fallback
    got2 = t.evaluate(B.params(B.COULOMB, B.CONSISTENT, B.FP64, del_=1e-4, acc=0.11))
    assert t.stats()["list_fallback"] == 0
    ref2 = T.evaluate(orc.params(orc.COULOMB, orc.MODE_CONSISTENT, del_=1e-4, acc=0.11))
    assert rel(got2, ref2) < TOL64


def planted_close_pairs(n, pairs, seed):
    """Uniform particles plus `pairs` partners placed 1e-6..1e-4 from existing ones."""
    rng = np.random.default_rng(seed)
    p = rng.uniform(0.0, 1.0, (n, 3))
    src = rng.choice(n, pairs, replace=False)
    d = rng.standard_normal((pairs, 3))
    d *= (10.0 ** rng.uniform(-6, -4, pairs) / np.linalg.norm(d, axis=1))[:, None]
    p = np.concatenate([p, p[src] + d])
    q = rng.uniform(-1.0, 1.0, len(p))
    return p[:, 0].copy(), p[:, 1].copy(), p[:, 2].copy(), q


@pytest.mark.parametrize("kern", ["screened", "coulomb"])
def test_mixed_close_pairs_within_tolerance(ctx, kern):
    """Near-coincident pairs: the FP32 difference of leaf-centred coordinates would lose
    ~1e-5 relative accuracy; such pairs are summed in FP64, so the mixed path stays within
    1e-6 of the FP64 path."""
    import bit_b200 as B
    from bit_b200 import workloads
    x, y, z, q = planted_close_pairs(20000, 300, seed=9)
    t = ctx.treemake(x, y, z, 256)
    t.treemoments(q, 7)
    kw = dict(kappa=2.5) if kern == "screened" else dict(del_=1e-14)
    k = B.SCREENED if kern == "screened" else B.COULOMB
    p64 = t.evaluate(B.params(k, B.CONSISTENT, B.FP64, acc=0.6, **kw))
    p32 = t.evaluate(B.params(k, B.CONSISTENT, B.MIXED, acc=0.6, **kw))
    assert workloads.rel_l2(p32, p64) < TOL_MIXED


def test_mixed_force_close_pairs_within_tolerance(ctx):
    import bit_b200 as B
    from bit_b200 import workloads
    x, y, z, q = planted_close_pairs(20000, 300, seed=10)
    t = ctx.treemake(x, y, z, 256)
    t.treemoments(q, 7)
    f64 = np.stack(t.treeforce(0.5, 1e-14, B.FP64))
    f32 = np.stack(t.treeforce(0.5, 1e-14, B.MIXED))
    assert workloads.rel_l2(f32, f64) < TOL_MIXED


@pytest.mark.parametrize("kern", ["screened", "coulomb"])
@pytest.mark.parametrize("blob,maxmemb", [(1500, 2000), (3000, 4000)])
def test_mixed_close_pairs_across_source_tiles(ctx, kern, blob, maxmemb):
    """A blob of radius 1e-6 at (0.3, 0.3, 0.3) inside 20,000 uniform points: its leaf
    holds 1,821 sources (N0 = 2000: 2 source tiles) or 3,661 (N0 = 4000: 4 tiles), and
    every blob pair is a close pair.  A blob target records each of those tiles for the
    FP64 pass: 2 fit the record slots, 4 overflow them, and the pass then scans all of the
    target's near entries instead.  Both must match the FP64 path."""
    import bit_b200 as B
    from bit_b200 import workloads
    rng = np.random.default_rng(13)
    p = np.concatenate([rng.uniform(0.0, 1.0, (20000, 3)),
                        [0.3, 0.3, 0.3] + 1e-6 * rng.standard_normal((blob, 3))])
    x, y, z = (np.ascontiguousarray(p[:, a]) for a in range(3))
    q = rng.uniform(-1.0, 1.0, len(p))
    t = ctx.treemake(x, y, z, maxmemb)
    t.treemoments(q, 5)
    kw = dict(kappa=2.0) if kern == "screened" else dict(del_=1e-14)
    k = B.SCREENED if kern == "screened" else B.COULOMB
    p64 = t.evaluate(B.params(k, B.CONSISTENT, B.FP64, acc=0.5, **kw))
    p32 = t.evaluate(B.params(k, B.CONSISTENT, B.MIXED, acc=0.5, **kw))
    assert np.all(np.isfinite(p32))
    assert workloads.rel_l2(p32, p64) < TOL_MIXED
    np.testing.assert_array_equal(p32, t.evaluate(B.params(k, B.CONSISTENT, B.MIXED, acc=0.5, **kw)))


def test_mixed_coincident_duplicates_follow_the_fp64_rules(ctx):
    """Exact duplicates: the Coulomb sum skips r^2 + del <= 1e-14 in both precisions."""
    import bit_b200 as B
    from bit_b200 import workloads
    x, y, z, q = workloads.uniform_cube(5000, seed=11)
    x = np.concatenate([x, x[:50]]); y = np.concatenate([y, y[:50]]); z = np.concatenate([z, z[:50]])
    q = np.concatenate([q, q[:50]])
    t = ctx.treemake(x, y, z, 64)
    t.treemoments(q, 5)
    p64 = t.evaluate(B.params(B.COULOMB, B.CONSISTENT, B.FP64, del_=0.0, acc=0.5))
    p32 = t.evaluate(B.params(B.COULOMB, B.CONSISTENT, B.MIXED, del_=0.0, acc=0.5))
    assert np.all(np.isfinite(p64)) and np.all(np.isfinite(p32))
    assert workloads.rel_l2(p32, p64) < TOL_MIXED


@pytest.mark.parametrize("kern", ["screened", "coulomb"])
def test_mixed_far_field_at_tiny_scales(ctx, kern):
    """Four tight clusters (sigma 1e-6, about 2e-5 apart) with small leaves: far-field
    clusters are accepted at r ~ 1e-6..1e-5, where coefficients of size r^-(n+1) exceed
    the FP32 range.  The FP32 far field works on moments normalised by the cluster size,
    with terms (h/r)^n / r, so the mixed path stays finite and within 1e-6 of FP64."""
    import bit_b200 as B
    from bit_b200 import workloads
    rng = np.random.default_rng(12)
    centres = np.array([[0.5, 0.5, 0.5], [0.5 + 2e-5, 0.5, 0.5], [0.5, 0.5 + 2e-5, 0.5],
                        [0.5, 0.5, 0.5 + 3e-5]])
    p = np.concatenate([c + 1e-6 * rng.standard_normal((4000, 3)) for c in centres])
    x, y, z = (np.ascontiguousarray(p[:, a]) for a in range(3))
    q = rng.uniform(-1.0, 1.0, len(p))
    t = ctx.treemake(x, y, z, 64)
    t.treemoments(q, 9)
    kw = dict(kappa=1.0) if kern == "screened" else dict(del_=0.0)
    k = B.SCREENED if kern == "screened" else B.COULOMB
    p64 = t.evaluate(B.params(k, B.CONSISTENT, B.FP64, acc=0.5, **kw))
    p32 = t.evaluate(B.params(k, B.CONSISTENT, B.MIXED, acc=0.5, **kw))
    assert t.stats()["far_pairs"] > 0
    assert np.all(np.isfinite(p64)) and np.all(np.isfinite(p32))
    assert workloads.rel_l2(p32, p64) < TOL_MIXED


def shared_steps(c, x, y, z, q, prec, ps, pc, steps=2):
    """The benchmark's step on a fresh tree each time: screened, then Coulomb."""
    import bit_b200 as B
    out = []
    for _ in range(steps):
        t = c.treemake(x, y, z, 1000)
        t.treemoments(q, 9)
        s_pot = t.evaluate(B.params(B.SCREENED, B.CONSISTENT, prec, **ps))
        c_pot = t.evaluate(B.params(B.COULOMB, B.CONSISTENT, prec, **pc))
        out.append((s_pot, c_pot, t.stats()))
        t.treeempty()
    return out


def own_lists(c, x, y, z, q, prm):
    t = c.treemake(x, y, z, 1000)
    t.treemoments(q, 9)
    pot = t.evaluate(prm)
    assert t.stats()["lists_shared"] == 0
    t.treeempty()
    return pot


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_lists_shared_between_kernels_match_their_own(orc, prec):
    """From the second tree on, the screened build also checks the Coulomb MAC (the
    context's previous one); every decision agrees, so the Coulomb evaluation reuses those
    lists. Its potential is bit-identical to a context that walks the tree for Coulomb
    itself, and the FP64 one matches the oracle."""
    import bit_b200 as B
    from bit_b200 import workloads
    pr = B.FP64 if prec == "fp64" else B.MIXED
    x, y, z, q = workloads.clustered_blobs(50000, seed=21)
    ps, pc = dict(kappa=1.0, acc=0.7), dict(del_=0.005, acc=0.7)
    a, b = B.Context(), B.Context()
    try:
        steps = shared_steps(a, x, y, z, q, pr, ps, pc)
        assert steps[0][2]["lists_shared"] == 0
        s_pot, c_pot, st = steps[1]
        assert st["lists_shared"] == 1 and st["t_lists"] == 0.0
        np.testing.assert_array_equal(c_pot, own_lists(b, x, y, z, q, B.params(B.COULOMB, B.CONSISTENT, pr, **pc)))
        np.testing.assert_array_equal(s_pot, own_lists(b, x, y, z, q, B.params(B.SCREENED, B.CONSISTENT, pr, **ps)))
        np.testing.assert_array_equal(c_pot, steps[0][1])
        if pr == B.FP64:
            T = orc.Tree(x, y, z, 1000)
            T.compute_moments(q, 9)
            ref = T.evaluate(orc.params(orc.COULOMB, orc.MODE_CONSISTENT, del_=0.005, acc=0.7))
            assert rel(c_pot, ref) < TOL64
    finally:
        a.close()
        b.close()


@pytest.mark.parametrize("ps", [dict(kappa=1.0, acc=0.5), dict(kappa=1.0, acc=0.7, mac_del=0.01)])
def test_lists_not_shared_when_the_macs_decide_differently(ps):
    """A different acc, or the screened MAC's r^2 - mac_del: some decision differs, so the
    Coulomb evaluation walks the tree itself and gets exactly its own lists."""
    import bit_b200 as B
    from bit_b200 import workloads
    x, y, z, q = workloads.clustered_blobs(50000, seed=22)
    pc = dict(del_=0.01, acc=0.7)
    a, b = B.Context(), B.Context()
    try:
        for s_pot, c_pot, st in shared_steps(a, x, y, z, q, B.FP64, ps, pc):
            assert st["lists_shared"] == 0 and st["t_lists"] > 0
        np.testing.assert_array_equal(c_pot, own_lists(b, x, y, z, q, B.params(B.COULOMB, B.CONSISTENT, B.FP64, **pc)))
        np.testing.assert_array_equal(s_pot, own_lists(b, x, y, z, q, B.params(B.SCREENED, B.CONSISTENT, B.FP64, **ps)))
    finally:
        a.close()
        b.close()


@pytest.mark.parametrize("tile,split", [(128, 0), (256, 4), (1024, 32), (2048, 1), (512, 8)])
def test_near_config_keeps_results(orc, tile, split):
    """The autotuner's near-field knobs (source tile, threads-per-target cap) change only
    the rounding order: FP64 stays within 1e-12 of the oracle, mixed within 1e-6 of FP64."""
    import bit_b200 as B
    from bit_b200 import workloads
    x, y, z, q = workloads.clustered_blobs(30000, seed=17)
    T = orc.Tree(x, y, z, 300)
    T.compute_moments(q, 7)
    c = B.Context()
    try:
        c.set_near_config(tile, split)
        t = c.treemake(x, y, z, 300)
        t.treemoments(q, 7)
        for kern, kw in [(B.COULOMB, dict(del_=1e-4)), (B.SCREENED, dict(kappa=2.0))]:
            p64 = t.evaluate(B.params(kern, B.CONSISTENT, B.FP64, acc=0.5, **kw))
            p32 = t.evaluate(B.params(kern, B.CONSISTENT, B.MIXED, acc=0.5, **kw))
            ref = T.evaluate(orc.params(kern, orc.MODE_CONSISTENT, acc=0.5, **kw))
            assert rel(p64, ref) < TOL64
            assert np.linalg.norm(p32 - p64) / np.linalg.norm(p64) < TOL_MIXED
        t.treeempty()
        for bad in [(100, 0), (4096, 0), (512, 3), (512, 64)]:
            with pytest.raises(B.BitError):
                c.set_near_config(*bad)
    finally:
        c.close()


def test_pinned_host_arrays_give_the_same_results(ctx):
    """Page-locked caller arrays take the direct DMA path (copies of 4 MB and more), pageable
    ones the staged path: the tree, its moments and the potentials are the same bit for bit,
    into a pinned or a pageable result array."""
    import torch
    import bit_b200 as B
    n = 600_000
    rng = np.random.default_rng(7)
    x, y, z, q = (rng.uniform(-1, 1, n) for _ in range(4))
    keep = []

    def pinned(a):
        t = torch.empty(n, dtype=torch.float64, pin_memory=True)
        keep.append(t)
        arr = t.numpy()
        arr[:] = a
        return arr
    p = B.params(B.SCREENED, B.CONSISTENT, B.FP64, kappa=1.0, acc=0.5)
    t1 = ctx.treemake(x, y, z, 1000)
    t1.treemoments(q, 5)
    r1 = t1.evaluate(p)
    t1.treeempty()
    t2 = ctx.treemake(pinned(x), pinned(y), pinned(z), 1000)
    t2.treemoments(pinned(q), 5)
    out = pinned(np.zeros(n))
    r2 = t2.evaluate(p, out=out)
    t2.treeempty()
    assert r2 is out
    assert np.array_equal(r1, r2)


def test_trim_gives_back_cached_blocks_and_the_context_keeps_working(ctx):
    """bit_ctx_trim frees the context's cached blocks (never live ones): an evaluation
    after it gives the same potentials as before."""
    import bit_b200 as B
    g = load_golden("uniform3000")
    p = B.params(B.SCREENED, B.CONSISTENT, B.FP64, kappa=1.0, acc=0.5)
    t = ctx.treemake(g["x"], g["y"], g["z"], int(g["maxmemb"]))
    t.treemoments(g["q"], int(g["nterms"]))
    before = t.evaluate(p)
    ctx.trim(0)  # the tree's live buffers stay
    again = t.evaluate(p)
    t.treeempty()
    ctx.trim(0)
    t = ctx.treemake(g["x"], g["y"], g["z"], int(g["maxmemb"]))
    t.treemoments(g["q"], int(g["nterms"]))
    after = t.evaluate(p)
    t.treeempty()
    assert np.array_equal(before, again) and np.array_equal(before, after)

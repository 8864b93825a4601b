"""The large clustered evaluation at its full size, against the reference build.

N = 2,000,000 particles (80% in 8 Gaussian blobs of sigma 0.1, 20% uniform in [-1,1]^3,
charges U[-1,1], the seed the benchmark uses), N0 = 1000, p = 8 (nterms 9), theta = 0.7:

- the tree (node numbering, children, the 13 FP64 fields of every node, member lists in
  order) equals the reference's treemake (src/tree3d.cpp:1345-1551) bit for bit;
- the FP64 moments equal treemoments (:2631-2711) to 1e-12 of each node's largest moment;
- FP64 potentials at 10,000 seeded targets equal the reference's own shielded_treepot
  (kappa = 1, :3448-3627) and treepotential (delta = 0.005, :4679-4778, moments padded so
  its degree-nterms read stays in bounds) to 1e-12 in reference mode, and the oracle's
  restatement to 1e-12 in consistent mode;
- the mixed path stays within 1e-6 of the FP64 path at every particle.
"""
import numpy as np
import pytest

import bit_b200 as B
from bit_b200 import workloads

pytestmark = pytest.mark.gpu

N, N0, NTERMS, ACC, KAPPA, DEL = 2_000_000, 1000, 9, 0.7, 1.0, 0.005 ** 2
SAMPLE = 10_000
TOL64, TOL_MIXED = 1e-12, 1e-6


def rel(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return max(np.linalg.norm(a - b) / np.linalg.norm(b), np.abs(a - b).max() / np.abs(b).max())


@pytest.fixture(scope="module")
def full():
    from oracle import ref
    if not ref.available(DEL):
        pytest.skip("reference build not present")
    x, y, z, q = workloads.clustered_blobs(N, seed=1)
    R = ref.RefTree(x, y, z, q, NTERMS, N0, del_=DEL)
    R.moments()
    tg = workloads.sample_targets(N, SAMPLE, seed=11)
    out = dict(x=x, y=y, z=z, q=q, R=R, tg=tg)
    yield out
    R.close()


def test_fullsize_tree_is_the_reference_tree(ctx, full):
    from test_gpu_tree import assert_same_tree
    t = ctx.treemake(full["x"], full["y"], full["z"], N0)
    nm, ch, f, mem = full["R"].export()
    assert_same_tree(t, nm, ch, f, mem)
    t.treeempty()


def test_fullsize_moments_match_reference(ctx, full):
    R = full["R"]
    t = ctx.treemake(full["x"], full["y"], full["z"], N0)
    t.treemoments(full["q"], NTERMS)
    m = t.export_moments()
    idx = [(i, j, k) for i in range(NTERMS) for j in range(NTERMS - i) for k in range(NTERMS - i - j)]
    ii, jj, kk = (np.array(v) for v in zip(*idx))
    worst = 0.0
    for node in range(t.numtree):
        want = R.node_moments(node)[ii, jj, kk]
        worst = max(worst, np.abs(m[node] - want).max() / max(np.abs(want).max(), 1e-300))
    t.treeempty()
    assert worst < TOL64, worst


def test_fullsize_fp64_potentials_match_reference(ctx, full):
    R, tg = full["R"], full["tg"]
    t = ctx.treemake(full["x"], full["y"], full["z"], N0)
    t.treemoments(full["q"], NTERMS)
    scr = t.shielded_treepot(KAPPA, ACC, mode=B.REFERENCE, mac_del=DEL)
    coul = t.treepotential(ACC, DEL, mode=B.REFERENCE)
    t.treeempty()
    assert rel(scr[tg], R.screened(KAPPA, ACC, tg)) < TOL64
    assert rel(coul[tg], R.potential(ACC, tg)) < TOL64


def test_fullsize_consistent_mode_and_mixed(ctx, orc, full):
    x, y, z, q, tg = full["x"], full["y"], full["z"], full["q"], full["tg"]
    t = ctx.treemake(x, y, z, N0)
    t.treemoments(q, NTERMS)
    T = orc.Tree(x, y, z, N0)
    T.compute_moments(q, NTERMS)
    for kern, kw in ((B.SCREENED, dict(kappa=KAPPA)), (B.COULOMB, dict(del_=DEL))):
        p64 = t.evaluate(B.params(kern, B.CONSISTENT, B.FP64, acc=ACC, **kw))
        p32 = t.evaluate(B.params(kern, B.CONSISTENT, B.MIXED, acc=ACC, **kw))
        want = T.evaluate(orc.params(kern, orc.MODE_CONSISTENT, acc=ACC, **kw), targets=tg)
        assert rel(p64[tg], want) < TOL64, kern
        assert np.linalg.norm(p32 - p64) / np.linalg.norm(p64) < TOL_MIXED, kern
    t.treeempty()

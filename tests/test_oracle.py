"""CPU tests of the oracle (the C restatement in oracle/bit_oracle.c).

The restatement is pinned bit for bit to golden outputs of the unmodified reference
(tests/golden/*.npz, made by tests/golden/make_golden.py), to the reference's own
known-answer comment (tests/kernel_convergence.cpp:50-51), and -- when the reference
libraries are built on this machine -- to the reference directly on larger inputs.
"""
import numpy as np
import pytest

from conftest import GOLDEN_CASES, load_golden


def bits(a):
    return np.ascontiguousarray(a, dtype=np.float64).view(np.int64)


def oracle_tree(orc, g):
    T = orc.Tree(g["x"], g["y"], g["z"], int(g["maxmemb"]))
    T.compute_moments(g["q"], int(g["nterms"]), w=g["w"])
    return T


@pytest.mark.parametrize("name", GOLDEN_CASES)
def test_tree_matches_reference_golden(orc, name):
    """treemake: node count, children order, every field bit for bit, member lists."""
    g = load_golden(name)
    T = oracle_tree(orc, g)
    assert T.numtree == len(g["nummemb"])
    np.testing.assert_array_equal(T.nummemb, g["nummemb"])
    np.testing.assert_array_equal(T.children, g["children"])
    np.testing.assert_array_equal(bits(T.fields), bits(g["fields"]))
    members = np.concatenate([T.members(i) for i in range(T.numtree)])
    np.testing.assert_array_equal(members, g["members"])


@pytest.mark.parametrize("name", GOLDEN_CASES)
def test_moments_match_reference_golden(orc, name):
    g = load_golden(name)
    T = oracle_tree(orc, g)
    np.testing.assert_array_equal(bits(T.mom), bits(g["moments"].reshape(-1)))


@pytest.mark.parametrize("name", GOLDEN_CASES)
def test_potentials_match_reference_golden(orc, name):
    """treepotential / shielded_treepot / treeforce, particle and point targets, bit for bit."""
    g = load_golden(name)
    T = oracle_tree(orc, g)
    d, acc, kappa = float(g["del_"]), float(g["acc"]), float(g["kappa"])
    pc = orc.params(orc.COULOMB, orc.MODE_REFERENCE, del_=d, acc=acc)
    ps = orc.params(orc.SCREENED, orc.MODE_REFERENCE, del_=d, mac_del=d, kappa=kappa, acc=acc)
    np.testing.assert_array_equal(bits(T.evaluate(pc)), bits(g["coulomb"]))
    np.testing.assert_array_equal(bits(T.evaluate(ps)), bits(g["screened"]))
    np.testing.assert_array_equal(bits(T.evaluate(pc, points=g["points"])), bits(g["coulomb_points"]))
    np.testing.assert_array_equal(bits(T.evaluate(ps, points=g["points"])), bits(g["screened_points"]))
    f = np.stack(T.evaluate_force(d, acc))
    np.testing.assert_array_equal(bits(f), bits(g["force"]))


def test_kernel_known_answer(orc):
    """|grad G_noreg - grad G_reg| at (0.1, 0.2, 0.3), DEL = 0.01, KERNEL_ORDER = 0:
    the reference's recorded answer (tests/kernel_convergence.cpp:50-51)."""
    dx, dy, dz = 0.1, 0.2, 0.3
    rs = dx * dx + dy * dy + dz * dz
    noreg = -np.array([dx, dy, dz]) / (rs * np.sqrt(rs))
    rs2 = rs + 0.01
    reg = -np.array([dx, dy, dz]) * (1.0 / (np.sqrt(rs2) * rs2))
    np.testing.assert_allclose(np.abs(reg - noreg),
                               [1.876829391553e-01, 3.753658783106e-01, 5.630488174659e-01],
                               rtol=1e-11)
    # the restatement's near-field force uses the same kernel: a 2-particle system
    x = np.array([0.0, dx]); y = np.array([0.0, dy]); z = np.array([0.0, dz])
    q = np.array([1.0, 1.0])
    fx, fy, fz = orc.direct_force(x, y, z, q, 0.01, np.array([0], np.int32))
    np.testing.assert_allclose([fx[0], fy[0], fz[0]], reg, rtol=1e-15)


def test_convergence_in_nterms(orc):
    """tests/treecode.cpp:84-127: max error of the treecode force against the direct sum
    is non-increasing for nterms = 1..4 (reference fixture shape, smaller N)."""
    g = load_golden("box2000")
    x, y, z, q = g["x"], g["y"], g["z"], g["q"]
    T = orc.Tree(x, y, z, 100)
    tg = np.arange(len(x), dtype=np.int32)
    ds = np.stack(orc.direct_force(x, y, z, q, 0.01, tg))
    prev = None
    for nterms in range(1, 5):
        T.compute_moments(q, nterms)
        f = np.stack(T.evaluate_force(0.01, 0.5))
        err = np.abs(f - ds).max(axis=1).sum()
        if prev is not None:
            assert err <= prev
        prev = err


def test_consistent_mode_matches_direct_sum(orc):
    """With one kernel in near and far field the treecode converges to the direct sum."""
    from bit_b200 import workloads
    x, y, z, q = workloads.uniform_cube(3000, seed=11)
    T = orc.Tree(x, y, z, 100)
    tg = workloads.sample_targets(3000, 200, seed=2)
    for kern, kw in [(orc.COULOMB, dict(del_=1e-4)), (orc.SCREENED, dict(kappa=1.0)),
                     (orc.SCREENED_REG, dict(kappa=1.0, del_=1e-3))]:
        errs = []
        for nterms in (3, 6, 9):
            T.compute_moments(q, nterms)
            p = orc.params(kern, orc.MODE_CONSISTENT, acc=0.3, **kw)
            errs.append(workloads.rel_l2(T.evaluate(p, tg), orc.direct(x, y, z, q, p, tg)))
        assert errs[2] < errs[0] and errs[2] < 1e-4, errs


def test_degenerate_input_reported(orc):
    """More than maxmemb coincident particles: the reference's treemake never ends; the
    restatement reports it."""
    x = np.zeros(10); y = np.zeros(10); z = np.zeros(10)
    with pytest.raises(RuntimeError, match="-2"):
        orc.Tree(x, y, z, 3)


def test_small_and_single_leaf_trees(orc):
    for n, mm in [(1, 1), (2, 1), (7, 3), (50, 100)]:
        rng = np.random.default_rng(n)
        x, y, z = rng.uniform(-1, 1, (3, n))
        T = orc.Tree(x, y, z, mm)
        assert T.nummemb[0] == n
        leaves = [i for i in range(T.numtree) if T.is_leaf(i)]
        assert sum(T.nummemb[i] for i in leaves) == n
        assert all(T.nummemb[i] <= mm for i in leaves)


def test_dense_gmres_restatement(orc):
    """solver::gmres restated (src/solver.h:157-310) solves a well-conditioned system."""
    rng = np.random.default_rng(3)
    n = 60
    A = np.eye(n) * 4 + rng.uniform(-0.5, 0.5, (n, n))
    b = rng.uniform(-1, 1, n)
    x, it = orc.gmres_dense_ref(A, b)
    assert it > 0
    np.testing.assert_allclose(A @ x, b, rtol=0, atol=1e-5 * np.abs(b).max() * 10)


def test_dense_gmres_restatement_matches_reference(orc):
    """The restatement of solver::gmres against the reference's own (oracle/_ref): the same
    Arnoldi step count and solution to 1e-12."""
    from oracle import ref
    if not ref.available(0.01):
        pytest.skip("reference build not present")
    rng = np.random.default_rng(9)
    n = 200
    A = np.eye(n) * 3 + rng.uniform(-0.5, 0.5, (n, n)) / np.sqrt(n)
    b = rng.uniform(-1, 1, n)
    x_ref, it_ref = ref.gmres_dense(A, b)
    x, it = orc.gmres_dense_ref(A, b)
    assert it == it_ref
    assert np.linalg.norm(x - x_ref) / np.linalg.norm(x_ref) < 1e-12


def test_restarted_gmres_treecode(orc):
    """GMRES(m) with the CPU treecode matvec reaches its residual target."""
    from bit_b200 import workloads
    cen, area, h = workloads.icosphere(2)
    f = workloads.sh_rhs(cen, lmax=4, seed=1)
    T = orc.Tree(cen[:, 0], cen[:, 1], cen[:, 2], 40)
    T.compute_moments(np.zeros(len(cen)), 5)
    p = orc.params(orc.SCREENED_REG, orc.MODE_CONSISTENT, del_=h * h, kappa=1.0, acc=0.5)
    s, it, rr, rc = orc.gmres_treecode(T, p, 0.5, area, f, restart=20, tol=1e-8, maxit=200)
    assert rc == 0 and rr <= 1e-7, (it, rr)


@pytest.mark.skipif("not __import__('oracle.ref', fromlist=['x']).available(1e-4)")
def test_restatement_against_reference_build():
    """Larger inputs straight against the reference build (when it exists here)."""
    from oracle import orc, ref
    from bit_b200 import workloads
    x, y, z, q = workloads.clustered_blobs(30000, seed=9)
    R = ref.RefTree(x, y, z, q, 8, 300, del_=1e-4)
    T = orc.Tree(x, y, z, 300)
    nm, ch, f, mem = R.export()
    np.testing.assert_array_equal(T.children, ch)
    np.testing.assert_array_equal(bits(T.fields), bits(f))
    R.moments()
    T.compute_moments(q, 8)
    tg = workloads.sample_targets(30000, 2000, seed=1)
    p = orc.params(orc.SCREENED, orc.MODE_REFERENCE, mac_del=1e-4, kappa=1.0, acc=0.7)
    np.testing.assert_array_equal(bits(T.evaluate(p, tg)), bits(R.screened(1.0, 0.7, tg)))
    p = orc.params(orc.COULOMB, orc.MODE_REFERENCE, del_=1e-4, acc=0.7)
    np.testing.assert_array_equal(bits(T.evaluate(p, tg)), bits(R.potential(0.7, tg)))
    R.close()

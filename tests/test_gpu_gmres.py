"""GMRES on the device: the dense solver::gmres drop-in and the treecode-matvec solver."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_dense_gmres_matches_restatement(ctx, orc):
    """solver::gmres (src/solver.h:157-310) on the device vs the CPU restatement."""
    rng = np.random.default_rng(4)
    n = 300
    A = np.eye(n) * 3 + rng.uniform(-0.5, 0.5, (n, n)) / np.sqrt(n)
    b = rng.uniform(-1, 1, n)
    x_gpu, it_gpu, st = ctx.gmres_dense(A, b)
    x_cpu, it_cpu = orc.gmres_dense_ref(A, b)
    assert st == 0
    assert abs(it_gpu - it_cpu) <= 2, (it_gpu, it_cpu)
    exact = np.linalg.solve(A, b)
    assert np.linalg.norm(x_gpu - exact) / np.linalg.norm(exact) < 1e-5
    assert np.linalg.norm(x_gpu - x_cpu) / np.linalg.norm(x_cpu) < 1e-6


@pytest.mark.parametrize("n,seed", [(64, 1), (300, 4), (700, 5)])
def test_dense_gmres_matches_reference_solver(ctx, n, seed):
    """The device solver against the reference's own solver::gmres (src/solver.h:157-310,
    built unmodified into oracle/_ref): the same number of Arnoldi steps and the same
    solution to 1e-10 relative (the algorithm and its stop test are the same; only the
    summation order of the device's dot products differs)."""
    from oracle import ref
    if not ref.available(0.01):
        pytest.skip("reference build not present")
    rng = np.random.default_rng(seed)
    A = np.eye(n) * 3 + rng.uniform(-0.5, 0.5, (n, n)) / np.sqrt(n)
    b = rng.uniform(-1, 1, n)
    x_ref, it_ref = ref.gmres_dense(A, b)
    x_gpu, it_gpu, st = ctx.gmres_dense(A, b)
    assert st == 0
    assert it_gpu == it_ref, (it_gpu, it_ref)
    assert np.linalg.norm(x_gpu - x_ref) / np.linalg.norm(x_ref) < 1e-10


def test_dense_gmres_zero_rhs(ctx):
    """b = 0: x = 0 after no step (the reference would divide by |b| = 0)."""
    A = np.eye(8) * 2.0
    x, it, st = ctx.gmres_dense(A, np.zeros(8))
    assert st == 0 and it == 0 and not x.any()


def test_dense_gmres_breakdown(ctx):
    """A Krylov space that closes at step 1 reports breakdown (src/solver.h:220-225)."""
    n = 16
    b = np.zeros(n)
    b[0] = 2.0
    x, it, st = ctx.gmres_dense(np.eye(n), b)
    assert st == 6
    np.testing.assert_allclose(x, b, rtol=1e-12)


def bie_problem(level=3):
    from bit_b200 import workloads
    cen, area, h = workloads.icosphere(level)
    f = workloads.sh_rhs(cen, lmax=8, seed=1)
    return cen, area, h, f


def test_bie_fp64_matches_cpu_gmres(ctx, orc):
    import bit_b200 as B
    cen, area, h, f = bie_problem(3)
    t = ctx.treemake(cen[:, 0], cen[:, 1], cen[:, 2], 100)
    p = B.params(B.SCREENED_REG, B.CONSISTENT, B.FP64, del_=h * h, kappa=1.0, acc=0.5)
    s, info, st = t.bie_solve(p, 7, 0.5, area, f, restart=50, tol=1e-8, precision=B.FP64)
    assert st == 0 and info["relres"] <= 1e-8, info
    T = orc.Tree(cen[:, 0], cen[:, 1], cen[:, 2], 100)
    T.compute_moments(np.zeros(len(cen)), 7)
    po = orc.params(orc.SCREENED_REG, orc.MODE_CONSISTENT, del_=h * h, kappa=1.0, acc=0.5)
    s_cpu, it, rr, rc = orc.gmres_treecode(T, po, 0.5, area, f, restart=50, tol=1e-8, maxit=500)
    assert rc == 0
    assert np.linalg.norm(s - s_cpu) / np.linalg.norm(s_cpu) < 1e-6


def test_bie_mixed_refinement_reaches_fp64_tolerance(ctx):
    import bit_b200 as B
    cen, area, h, f = bie_problem(4)
    t = ctx.treemake(cen[:, 0], cen[:, 1], cen[:, 2], 200)
    p = B.params(B.SCREENED_REG, B.CONSISTENT, B.FP64, del_=h * h, kappa=1.0, acc=0.5)
    s64, i64, st = t.bie_solve(p, 7, 0.5, area, f, restart=50, tol=1e-8, precision=B.FP64)
    assert st == 0
    s32, i32, st = t.bie_solve(p, 7, 0.5, area, f, restart=50, tol=1e-8, precision=B.MIXED)
    assert st == 0, i32
    assert i32["relres"] <= 1e-8
    assert i32["matvecs_fp64"] <= i32["refinements"] + 1
    assert np.linalg.norm(s32 - s64) / np.linalg.norm(s64) < 1e-6


def test_bie_solution_is_the_same_alone_and_after_other_work(ctx):
    """Device state left by other evaluations does not change a solve."""
    import bit_b200 as B
    from bit_b200 import workloads
    cen, area, h, f = bie_problem(3)
    p = B.params(B.SCREENED_REG, B.CONSISTENT, B.FP64, del_=h * h, kappa=1.0, acc=0.5)
    t = ctx.treemake(cen[:, 0], cen[:, 1], cen[:, 2], 100)
    a, _, _ = t.bie_solve(p, 7, 0.5, area, f, tol=1e-8)
    x, y, z, q = workloads.clustered_blobs(20000, seed=2)
    u = ctx.treemake(x, y, z, 300)
    u.treemoments(q, 5)
    u.evaluate(B.params(B.COULOMB, B.CONSISTENT, B.MIXED, del_=1e-4, acc=0.6))
    b, _, _ = t.bie_solve(p, 7, 0.5, area, f, tol=1e-8)
    np.testing.assert_array_equal(a, b)


@pytest.mark.parametrize("level,maxmemb", [(3, 100), (4, 200), (5, 500)])
def test_bie_operator_matches_oracle(ctx, orc, level, maxmemb):
    """The regularised-screened treecode on icosphere nodes (the BIE matvec) vs the oracle."""
    import bit_b200 as B
    cen, area, h, f = bie_problem(level)
    q = area * np.random.default_rng(level).standard_normal(len(area))
    t = ctx.treemake(cen[:, 0], cen[:, 1], cen[:, 2], maxmemb)
    t.treemoments(q, 7)
    T = orc.Tree(cen[:, 0], cen[:, 1], cen[:, 2], maxmemb)
    T.compute_moments(q, 7)
    for prec, tol in ((B.FP64, 1e-12), (B.MIXED, 1e-6)):
        got = t.evaluate(B.params(B.SCREENED_REG, B.CONSISTENT, prec, del_=h * h, kappa=1.0, acc=0.5))
        ref = T.evaluate(orc.params(orc.SCREENED_REG, orc.MODE_CONSISTENT, del_=h * h, kappa=1.0, acc=0.5))
        assert np.linalg.norm(got - ref) / np.linalg.norm(ref) < tol, prec

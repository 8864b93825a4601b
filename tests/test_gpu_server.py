"""The serving loop (bit_server_*): continuous batching of evaluate and solve requests.

Each result must be the same alone and in the mix: bit-identical to the same request run
alone on a one-slot server, and to the single-request API.  Admission must respect the
HBM budget, and requests must overlap on the device when slots and memory allow.
"""
import threading

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

MB = 1 << 20


def est_eval(n):
    """Admission estimate of an evaluate request (the server's formula)."""
    return 64 * MB + 448 * n


def eval_requests(B, count, seed):
    from bit_b200 import workloads
    rng = np.random.default_rng(seed)
    out = []
    for i in range(count):
        n = int(rng.integers(2000, 30000))
        x, y, z, q = workloads.clustered_blobs(n, seed=seed * 1000 + i)
        if i % 2:
            p = B.params(B.SCREENED, B.CONSISTENT, B.MIXED, kappa=float(rng.uniform(0.5, 4)), acc=0.6)
        else:
            p = B.params(B.COULOMB, B.CONSISTENT, B.MIXED, del_=1e-4, acc=0.6)
        out.append((x, y, z, q, int(rng.choice([5, 7, 9])), 256, p))
    return out


def solve_request(B, level, seed):
    from bit_b200 import workloads
    cen, area, h = workloads.icosphere(level)
    f = workloads.sh_rhs(cen, lmax=8, seed=seed)
    p = B.params(B.SCREENED_REG, B.CONSISTENT, B.FP64, del_=h * h, kappa=1.0, acc=0.5)
    return [np.ascontiguousarray(cen[:, a]) for a in range(3)] + [area, f, 7, 200, p, 0.5]


def test_results_are_the_same_alone_and_in_the_mix(ctx):
    import bit_b200 as B
    evals = eval_requests(B, 10, seed=1)
    solves = [solve_request(B, 3, 1), solve_request(B, 4, 2)]
    mixed = B.Server(slots=4)
    ids = []
    for i, r in enumerate(evals):
        ids.append(("e", i, mixed.submit_eval(*r)))
        if i in (3, 7):
            k = len([t for t in ids if t[0] == "s"])
            x, y, z, w, f, nt, mm, p, d = solves[k]
            ids.append(("s", k, mixed.submit_solve(x, y, z, w, f, nt, mm, p, d,
                                                   precision=B.MIXED)))
    got = {}
    for kind, i, rid in ids:
        res, info, st = mixed.wait(rid)
        assert st == 0, (kind, i, info)
        assert info["t_submit"] <= info["t_start"] <= info["t_done"]
        got[(kind, i)] = res
    stats = mixed.stats()
    mixed.close()
    assert stats["completed"] == len(ids)
    assert stats["max_running"] >= 2  # requests overlapped on the device
    alone = B.Server(slots=1)
    for kind, i, _ in ids:
        if kind == "e":
            rid = alone.submit_eval(*evals[i])
        else:
            x, y, z, w, f, nt, mm, p, d = solves[i]
            rid = alone.submit_solve(x, y, z, w, f, nt, mm, p, d, precision=B.MIXED)
        res, _, st = alone.wait(rid)
        assert st == 0
        np.testing.assert_array_equal(res, got[(kind, i)])
    alone.close()
    # and the single-request API gives the same evaluation
    x, y, z, q, nt, mm, p = evals[0]
    np.testing.assert_array_equal(ctx.treecode_potential(x, y, z, q, nt, mm, p), got[("e", 0)])


def test_admission_respects_the_hbm_budget():
    """A budget that holds one request at a time serialises them."""
    import bit_b200 as B
    evals = eval_requests(B, 6, seed=2)
    budget = max(est_eval(len(r[0])) for r in evals) + MB  # below two requests' worth
    srv = B.Server(slots=4, hbm_budget=budget)
    ids = [srv.submit_eval(*r) for r in evals]
    infos = [srv.wait(i)[1] for i in ids]
    stats = srv.stats()
    srv.close()
    assert stats["max_running"] == 1
    assert stats["max_reserved"] <= budget
    # FIFO: each request starts after the previous one finished
    for a, b in zip(infos, infos[1:]):
        assert b["t_start"] >= a["t_done"]


def test_request_larger_than_the_budget_is_refused():
    import bit_b200 as B
    evals = eval_requests(B, 1, seed=3)
    srv = B.Server(slots=2, hbm_budget=32 * MB)
    with pytest.raises(B.BitError) as e:
        srv.submit_eval(*evals[0])
    assert e.value.status == 9
    srv.close()


def test_submission_from_several_threads():
    import bit_b200 as B
    evals = eval_requests(B, 8, seed=4)
    srv = B.Server(slots=3)
    results = {}

    def client(k):
        for i in range(k, len(evals), 2):
            rid = srv.submit_eval(*evals[i])
            results[i] = srv.wait(rid)

    th = [threading.Thread(target=client, args=(k,)) for k in range(2)]
    for t in th:
        t.start()
    for t in th:
        t.join()
    srv.close()
    assert sorted(results) == list(range(len(evals)))
    assert all(st == 0 for _, _, st in results.values())


def test_memory_held_stays_within_the_budget():
    """Admission counts what every slot's context really holds (running reservations and
    idle slots' live and cached blocks), and a running request's context may not allocate
    beyond its reservation: every request's peak is at most its reservation, the total
    accounted never exceeds the budget, and no request fails."""
    import bit_b200 as B
    evals = eval_requests(B, 12, seed=7)
    budget = 3 * max(est_eval(len(r[0])) for r in evals)
    srv = B.Server(slots=4, hbm_budget=budget)
    ids = [srv.submit_eval(*r) for r in evals]
    sol = solve_request(B, 4, seed=3)
    ids.append(srv.submit_solve(*sol))
    infos = [srv.wait(i) for i in ids]
    stats = srv.stats()
    srv.close()
    for _, info, st in infos:
        assert st == 0
        assert info["peak_bytes"] <= info["bytes_reserved"], info
    assert stats["max_reserved"] <= budget

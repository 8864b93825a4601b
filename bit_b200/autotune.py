"""Autotuner for the treecode's leaf size N0 (maxmemb) and its leaf packing (group size).

N0 trades near-field work (larger leaves: more direct pairs) against far-field and list
work (smaller leaves: more clusters, more entries).  The best value depends on the
expansion order, the kernel and the system size, so it is measured: each candidate is
timed on the device on a seeded synthetic system of the requested size and distribution
(tree build, moments, lists, far and near field; device times from bit_tree_stats), and
the fastest is kept.  Results are cached per (nterms, kernel, precision, size bucket,
distribution) for the life of the process.

Leaf packing (bit_ctx_set_group_size) decides whether consecutive small leaves share one
group of targets.  It pays off for many small leaves (batched uneven systems: 35% faster)
and costs where near entries then cover too few targets (the icosphere solves: 70% slower),
so tune_group times it on the caller's own workload.
"""
import math

import numpy as np

CANDIDATES = (64, 128, 256, 512, 1024)
_cache = {}


def _bucket(n):
    return int(round(math.log2(max(n, 1)) * 2))  # half-octave buckets


def _system(n, dist, seed):
    from . import workloads
    if dist == "clustered":
        return workloads.clustered_blobs(n, seed=seed)
    rng = np.random.default_rng(seed)
    p = rng.uniform(0.0, 1.0, (n, 3))
    return p[:, 0].copy(), p[:, 1].copy(), p[:, 2].copy(), rng.uniform(-1.0, 1.0, n)


def step_seconds(ctx, x, y, z, q, maxmemb, nterms, prm, repeats=2):
    """Device seconds of one build + moments + evaluation (best of `repeats`)."""
    best = float("inf")
    for _ in range(repeats):
        t = ctx.treemake(x, y, z, maxmemb)
        t.treemoments(q, nterms)
        t.evaluate(prm)
        s = t.stats()
        t.treeempty()
        best = min(best, s["t_build"] + s["t_moments"] + s["t_lists"] + s["t_far"] + s["t_near"])
    return best


def tune_n0(ctx, nterms, kernel, n, acc, del_=0.0, kappa=1.0, precision=None, dist="uniform",
            candidates=CANDIDATES, seed=0):
    """The fastest leaf size for systems of about n particles: (n0, {candidate: seconds})."""
    import bit_b200 as B
    prec = B.MIXED if precision is None else precision
    key = (nterms, kernel, prec, _bucket(n), dist)
    if key in _cache:
        return _cache[key]
    x, y, z, q = _system(n, dist, seed)
    prm = B.params(kernel, B.CONSISTENT, prec, del_=del_, kappa=kappa, acc=acc)
    times = {}
    for c in candidates:
        if c > n:
            continue
        times[c] = step_seconds(ctx, x, y, z, q, c, nterms, prm)
    best = min(times, key=times.get) if times else min(candidates)
    _cache[key] = (best, times)
    return _cache[key]


GROUP_CANDIDATES = (0, 256, 512, 1024)


def tune_group(ctx, run, candidates=GROUP_CANDIDATES, repeats=2):
    """Pick the leaf packing (group size) for a workload: run(ctx) performs one
    representative step and returns its device seconds.  Leaves the context set to the
    fastest candidate and returns (group, {candidate: seconds})."""
    times = {}
    for g in candidates:
        ctx.set_group_size(g)
        times[g] = min(run(ctx) for _ in range(repeats))
    best = min(times, key=times.get)
    ctx.set_group_size(best)
    return best, times

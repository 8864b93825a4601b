"""Autotuner for the treecode's launch shape: the leaf size N0 (maxmemb), the leaf packing
(target-batch size), and the near field's source tile and threads per target.

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

The near field's source tile (records per TMA copy into shared memory) and the cap on the
threads that split one target's sources (bit_ctx_set_near_config) are tuned per
(nterms, kernel, N0, precision) by tune_near on the same seeded systems; tune() chains
N0 and the near-field knobs for one workload class.
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
    key = ("n0", nterms, kernel, prec, _bucket(n), dist, acc)
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


NEAR_TILES = {"mixed": (512, 1024, 2048), "fp64": (256, 512, 1024)}
NEAR_SPLITS = (0, 4, 8, 16, 32)


def tune_near(ctx, nterms, kernel, n, acc, n0, del_=0.0, kappa=1.0, precision=None,
              dist="uniform", seed=0, repeats=2):
    """The fastest near-field (tile, threads-per-target cap) for systems of about n
    particles with leaf size n0, timed on the near field's device time of a seeded system.
    Leaves the context set to it and returns ((tile, split), {(tile, split): seconds})."""
    import bit_b200 as B
    prec = B.MIXED if precision is None else precision
    key = ("near", nterms, kernel, prec, _bucket(n), dist, acc, n0)
    if key in _cache:
        best, times = _cache[key]
        ctx.set_near_config(*best)
        return best, times
    x, y, z, q = _system(n, dist, seed)
    prm = B.params(kernel, B.CONSISTENT, prec, del_=del_, kappa=kappa, acc=acc)
    t = ctx.treemake(x, y, z, n0)
    t.treemoments(q, nterms)
    times = {}
    for tile in NEAR_TILES["mixed" if prec == B.MIXED else "fp64"]:
        for split in NEAR_SPLITS:
            ctx.set_near_config(tile, split)
            best = float("inf")
            for _ in range(repeats):
                t.evaluate(prm)
                best = min(best, t.stats()["t_near"])
            times[(tile, split)] = best
    t.treeempty()
    best = min(times, key=times.get)
    ctx.set_near_config(*best)
    _cache[key] = (best, times)
    return best, times


def tune(ctx, nterms, kernel, n, acc, del_=0.0, kappa=1.0, precision=None, dist="uniform"):
    """N0, then the near-field tile and threads-per-target cap, for one (p, kernel) class
    of systems of about n particles.  Returns {"n0", "tile", "threads_per_target"} and
    leaves the context set to the near-field choice."""
    n0, _ = tune_n0(ctx, nterms, kernel, n, acc, del_=del_, kappa=kappa, precision=precision,
                    dist=dist)
    (tile, split), _ = tune_near(ctx, nterms, kernel, n, acc, n0, del_=del_, kappa=kappa,
                                 precision=precision, dist=dist)
    return {"n0": n0, "tile": tile, "threads_per_target": split}

"""Treecode benchmark on B200 (one JSON line on rank 0).

Workload (one "step"): the large clustered evaluation -- N = 2,000,000 particles, 80% in
8 Gaussian blobs (sigma 0.1), 20% uniform in [-1,1]^3, charges U[-1,1] (seeded); tree
build (N0 = 1000), FP64 moments for p = 8 (nterms 9), then the potential at every
particle twice: screened kernel exp(-kappa r)/r with kappa = 1, and regularised Coulomb
1/sqrt(r^2 + delta^2) with delta = 0.005, both with MAC theta = 0.7.  evals = 2 N per step.

value  -- evals/s of the plain FP64 GPU path (the reference's arithmetic) with the inputs
          resident in HBM
e2e    -- the same through the C ABI with host buffers (H2D inputs, D2H potentials inside
          the timed region)
mixed  -- the mixed-precision path on the same step (FP32 near/far field in cluster-centred
          coordinates with compensated accumulation; FP64 MAC and moments), its e2e and its
          speed-up over FP64
accuracy_matched -- the clustered step, the boundary-integral solve, the batched systems
          and the serving stream at (p, theta) where the FP64 treecode reaches 1e-6 against
          the FP64 direct sum: FP64 and mixed throughput, errors and ratios

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl bit|reference] [--n N]

Multi-GPU: one process per GPU (torchrun); every rank evaluates its own independent
system of the same size (replicas, weak scaling, no collective on the data path); the
time is the max over ranks.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

NTERMS = 9          # p = 8
MAXMEMB = 1000      # N0
ACC = 0.7           # theta
KAPPA = 1.0
DEL = 0.005 ** 2    # delta^2
FLOPS_NEAR = {"screened": 14, "coulomb": 11}     # per near pair (rsqrt, exp counted as 1)
# FP64 pipe operations the FP64 near kernel issues per pair (its own rsqrt and exp spelled
# out: 3 differences, 3 for r^2 + del, 4 for the Newton step, 11 for exp, the products):
# the instruction-level ceiling of that kernel is peak / 2 / ops pairs per second
FP64_OPS_NEAR = {"screened": 26, "coulomb": 13}
# Accuracy-matched parameters: (p, theta, N0) at which the plain FP64 treecode reaches 1e-6
# relative L2 against the FP64 direct sum on these workloads (measured; the run reports
# the errors it reaches)
MATCHED_C2 = dict(nterms=9, acc=0.15, maxmemb=1000)
MATCHED_BIE = dict(nterms=9, acc=0.15, maxmemb=500)
MATCHED_BATCH_ACC = {5: 0.015, 7: 0.05, 9: 0.1}   # theta by nterms (p = 4, 6, 8)
# DRAM bytes (read + write) per launch of the full-size kernels (clustered N = 2M, p = 8,
# theta = 0.7, N0 = 1000, the near field at its default tile), from an ncu launch list of
# one step taking dram__bytes_read.sum and dram__bytes_write.sum in one pass per launch.
# Captures of the 200k case give 13.5 MB (FP64 near) and 7.8 MB (FP64 far) per launch,
# i.e. 135 and 78 MB scaled by N; the full-size launches read more (sources re-read by
# groups of several waves once the 126 MB L2 no longer holds them).
TRAFFIC = {
    "k_near<SCREENED, F64>": 266.19e6, "k_near<COULOMB, F64>": 225.88e6,
    "k_far<9, SCREENED, double>": 102.06e6, "k_far<9, COULOMB, double>": 102.54e6,
    "k_near<SCREENED, F32>": 131.96e6, "k_near<COULOMB, F32>": 114.60e6,
    "k_far<9, SCREENED, float>": 98.32e6, "k_far<9, COULOMB, float>": 98.96e6,
}
TRAFFIC_SOURCE = ("ncu launch list of the full-size step (gpu__time_duration.sum, "
                  "dram__bytes_read.sum, dram__bytes_write.sum; one pass per launch), "
                  "kernels of this build, near field at its default tile")
METRIC = "treecode evals/s (clustered N=2M, p=8, theta=0.7, N0=1000, screened+Coulomb)"


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled during the timed region."""

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.out = []

    def __enter__(self):
        q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={q}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.out.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.out:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 7:
                continue
            try:
                sm.append(float(parts[0]))
                mx = max(mx, float(parts[1]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[3:7]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx or None,
                "reasons": sorted(reasons), "samples": len(sm)}


def workload(n, seed):
    from bit_b200 import workloads
    return workloads.clustered_blobs(n, seed=seed)


def run_bit(args):
    import torch
    import bit_b200 as B

    from bit_b200 import replicas
    rank, world, local = replicas.rank_info()
    torch.cuda.set_device(local)
    dist = replicas.init("nccl")
    n = args.n
    x, y, z, q = workload(n, seed=replicas.system_seed(rank))
    dev = torch.device("cuda", local)
    # One stream for the library's context and every CUDA event that times it: the events
    # must be recorded on the stream the kernels run on (torch's default stream would not
    # order against the context's work).
    stream = torch.cuda.Stream(dev)
    torch.cuda.set_stream(stream)
    X = torch.tensor(np.stack([x, y, z, q]), dtype=torch.float64, device=dev)
    out_s = torch.empty(n, dtype=torch.float64, device=dev)
    out_c = torch.empty(n, dtype=torch.float64, device=dev)
    ctx = B.Context(local, stream=stream.cuda_stream)
    # measured CUDA-core FMA peaks of this device: the roofline denominators
    peaks = {"fp64": ctx.fma_peak(B.FP64) / 1e12, "fp32": ctx.fma_peak(B.MIXED) / 1e12}
    # the autotuner's near-field (tile, threads-per-target cap) per (precision, kernel) of
    # this class (p = 8, N0 = 1000, clustered), measured on a seeded system of the step's
    # size (a 200k sample chose settings that were slower at 2M)
    near_cfg, tuned = {}, {}
    if args.tune:
        from bit_b200 import autotune
        for prec, pname in ((B.FP64, "fp64"), (B.MIXED, "mixed")):
            default = (1024 if prec == B.MIXED else 512, 0)
            for kern, kname, kw in ((B.SCREENED, "screened", dict(kappa=KAPPA)),
                                    (B.COULOMB, "coulomb", dict(del_=DEL))):
                best, times = autotune.tune_near(ctx, NTERMS, kern, n, ACC, MAXMEMB,
                                                 precision=prec, dist="clustered", **kw)
                near_cfg[(prec, kern)] = best
                tuned[f"{pname}_{kname}"] = {
                    "tile": best[0], "threads_per_target": best[1],
                    "near_speedup_vs_default": times[default] / times[best] if default in times else None}
        ctx.set_near_config(0, 0)

    def near(prec, kern):
        ctx.set_near_config(*near_cfg.get((prec, kern), (0, 0)))

    def step(prec, keep=False, nterms=NTERMS, maxmemb=MAXMEMB, acc=ACC):
        t = ctx.treemake_device(n, X[0].data_ptr(), X[1].data_ptr(), X[2].data_ptr(), maxmemb)
        t.set_charges_device(X[3].data_ptr())
        t.moments(nterms)
        near(prec, B.SCREENED)
        t.evaluate_device(B.params(B.SCREENED, B.CONSISTENT, prec, kappa=KAPPA, acc=acc),
                          out_s.data_ptr())
        st_s = t.stats() if keep else None
        near(prec, B.COULOMB)
        t.evaluate_device(B.params(B.COULOMB, B.CONSISTENT, prec, del_=DEL, acc=acc),
                          out_c.data_ptr())
        st_c = t.stats() if keep else None
        if keep:
            return t, st_s, st_c
        t.treeempty()
        return None

    launches = {}

    def timed(prec, steps, warmup, **kw):
        for _ in range(warmup):
            step(prec, **kw)
        torch.cuda.synchronize()
        replicas.barrier(dist)
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        l0 = B.kernel_launches()
        e0.record(stream)
        for _ in range(steps):
            step(prec, **kw)
        e1.record(stream)
        torch.cuda.synchronize()
        launches[prec] = (B.kernel_launches() - l0) // steps
        return replicas.max_over_ranks(e0.elapsed_time(e1) / steps, dist, dev)

    # plain FP64 (the headline: the reference's arithmetic), timed with clocks sampled
    with ClockSampler(local) as clk:
        ms64 = timed(B.FP64, args.steps, args.warmup)
    clocks = clk.summary()
    ms32 = timed(B.MIXED, args.steps, args.warmup)
    # per-kernel device times of one step (events on the library's stream)
    t, st64_s, st64_c = step(B.FP64, keep=True)
    res64_s = out_s.cpu().numpy()
    res64_c = out_c.cpu().numpy()
    t.treeempty()
    t, st_s, st_c = step(B.MIXED, keep=True)
    res_s = out_s.cpu().numpy()
    res_c = out_c.cpu().numpy()
    t.treeempty()

    # e2e through the C ABI with host buffers in pinned (page-locked) host memory, as a
    # caller streaming systems through the GPU keeps them: the inputs, and two result
    # arrays allocated once and reused every step.  The library copies page-locked arrays
    # by DMA directly (pageable ones through its own pinned staging).
    pinned_keep = []

    def pinned(a=None):
        tt = torch.empty(n, dtype=torch.float64, pin_memory=True)
        pinned_keep.append(tt)
        arr = tt.numpy()
        arr[:] = 0.0 if a is None else a
        return arr
    hx, hy, hz, hq = pinned(x), pinned(y), pinned(z), pinned(q)
    host_s, host_c = pinned(), pinned()

    def e2e_step(prec):
        t = ctx.treemake(hx, hy, hz, MAXMEMB)
        t.treemoments(hq, NTERMS)
        near(prec, B.SCREENED)
        a = t.evaluate(B.params(B.SCREENED, B.CONSISTENT, prec, kappa=KAPPA, acc=ACC), out=host_s)
        near(prec, B.COULOMB)
        b = t.evaluate(B.params(B.COULOMB, B.CONSISTENT, prec, del_=DEL, acc=ACC), out=host_c)
        t.treeempty()
        return a, b

    def e2e_timed(prec):
        for _ in range(max(1, args.warmup // 2)):
            e2e_step(prec)
        torch.cuda.synchronize()
        replicas.barrier(dist)
        t0 = time.perf_counter()
        steps = max(1, args.steps // 2)
        for _ in range(steps):
            e2e_step(prec)
        torch.cuda.synchronize()
        return replicas.max_over_ranks((time.perf_counter() - t0) * 1e3 / steps, dist, dev)
    e2e64_ms = e2e_timed(B.FP64)
    e2e32_ms = e2e_timed(B.MIXED)

    matched = run_matched_c2(step, timed, ctx, x, y, z, q, out_s, out_c, args) if args.matched else None

    if rank != 0:
        replicas.finish(dist)
        return

    evals = 2 * n * world
    e2e_in = 4 * n * 8
    e2e_out = 2 * n * 8
    line = {
        "metric": METRIC, "value": evals / (ms64 * 1e-3), "unit": "evals/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms64, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded clustered blobs)",
        "config": {"workload": "clustered evaluation N=2,000,000 (80% in 8 Gaussian blobs sigma 0.1, "
                               "20% uniform), p=8, theta=0.7, N0=1000, screened kappa=1 + Coulomb "
                               "delta=0.005, all particles as targets; plain FP64 GPU path",
                   "n": n, "nterms": NTERMS, "maxmemb": MAXMEMB, "acc": ACC,
                   "parallelism": f"replicas x{world}",
                   "l2": "inputs (128 MB coordinates+charges, 64 MB sorted FP64 sources) exceed the "
                         "126 MB L2; no flush"},
        "clocks": clocks,
        "e2e": {"value": evals / (e2e64_ms * 1e-3), "unit": "evals/s",
                "h2d_bytes_per_step": e2e_in, "d2h_bytes_per_step": e2e_out,
                "ms_per_step": e2e64_ms,
                "host_buffers": "pinned host arrays (inputs and reused result arrays), "
                                "copied by DMA inside each step"},
        "mixed": {"dtype": "f32 near/far field in cluster-centred coordinates with compensated "
                           "accumulation, f64 MAC+moments",
                  "value": evals / (ms32 * 1e-3), "ms_per_step": ms32,
                  "speedup_vs_fp64": ms64 / ms32,
                  "e2e": {"value": evals / (e2e32_ms * 1e-3), "unit": "evals/s",
                          "h2d_bytes_per_step": e2e_in, "d2h_bytes_per_step": e2e_out,
                          "ms_per_step": e2e32_ms},
                  "e2e_speedup_vs_fp64": e2e64_ms / e2e32_ms,
                  "gpu_launches_per_step": launches[B.MIXED]},
        "fma_peaks_tflops": peaks,
        "autotune": {"near_config": tuned,
                     "note": "near-field source tile and threads-per-target cap chosen per "
                             "(precision, kernel) on a seeded clustered system of the step's size, N0=1000, "
                             "p=8, theta=0.7; applied to every step"} if tuned else None,
    }
    # per-phase device times and interaction counts (screened + Coulomb)
    phases = {}
    for prec, (ss, sc) in (("fp64", (st64_s, st64_c)), ("mixed", (st_s, st_c))):
        ph = {}
        for name, st in (("screened", ss), ("coulomb", sc)):
            ph[name] = {k: st[k] for k in ("t_far", "t_near", "t_lists", "far_pairs", "near_pairs",
                                           "far_entries", "near_entries", "batches",
                                           "lists_shared")}
        ph["build_s"] = ss["t_build"]
        ph["moments_s"] = ss["t_moments"]
        ph["numtree"] = ss["numtree"]
        phases[prec] = ph
    line["phases"] = phases
    # interactions per step: near (target, source) and far (target, cluster) pairs of both
    # kernels, counted from the lists (the same for both precisions and for the reference)
    inter = sum(st[k] for st in (st64_s, st64_c) for k in ("far_pairs", "near_pairs")) * world
    line["interactions"] = {
        "per_step": inter, "fp64_per_s": inter / (ms64 * 1e-3), "mixed_per_s": inter / (ms32 * 1e-3),
        "e2e_fp64_per_s": inter / (e2e64_ms * 1e-3), "e2e_mixed_per_s": inter / (e2e32_ms * 1e-3),
        "counted": "near (target, source) pairs plus far (target, cluster) pairs, screened and "
                   "Coulomb, all ranks"}
    # rooflines: the dominant kernel of the FP64 step first, then the others
    fpp = far_flops_per_pair(NTERMS)
    roofs = []
    for prec, st, pk in (("fp64", st64_s, peaks["fp64"]), ("fp64", st64_c, peaks["fp64"]),
                         ("mixed", st_s, peaks["fp32"]), ("mixed", st_c, peaks["fp32"])):
        kname = "screened" if st is st64_s or st is st_s else "coulomb"
        roofs.append(roofline_far(prec, kname, st, fpp[kname], pk))
        roofs.append(roofline_near(prec, kname, st, n, pk))
    fp64_roofs = sorted((r for r in roofs if r["precision"] == "fp64"), key=lambda r: -r["seconds"])
    line["roofline"] = fp64_roofs[0]
    line["roofline_others"] = [r for r in roofs if r is not fp64_roofs[0]]
    # accuracy of this step against the FP64 GPU path and the FP64 direct sum (sampled)
    line["accuracy"] = accuracy(ctx, x, y, z, q, res_s, res_c, res64_s, res64_c, args)
    if matched is not None:
        line["accuracy_matched"] = {"clustered_2M": matched}
    if args.bie:
        line["bie"] = run_bie(ctx, args)
        if args.matched:
            line["accuracy_matched"]["bie"] = run_bie(ctx, args, **MATCHED_BIE)
    if args.batched:
        line["batched"] = run_batched(ctx, args, dev)
        if args.matched:
            line["accuracy_matched"]["batched"] = run_batched(ctx, args, dev, acc_by_nterms=MATCHED_BATCH_ACC)
    if args.serve_requests:
        # the servers below get the device memory the batched runs left cached here
        ctx.trim(0)
        torch.cuda.empty_cache()
        line["serving"] = run_serving(ctx, args)
        if args.matched:
            line["accuracy_matched"]["serving"] = run_serving(ctx, args, matched=True)
    if args.cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(x, y, z, q, n, args)
        # the same lists, so the same interactions per eval
        line["cpu_baseline"]["interactions_per_s"] = line["cpu_baseline"]["value"] * inter / evals
    line["gpu_launches"] = launches[B.FP64] * args.steps
    line["gpu_launches_per_step"] = launches[B.FP64]
    print(json.dumps(line), flush=True)
    replicas.finish(dist)


def roofline_far(prec, kname, st, flops_pair, peak_tflops):
    """Far field (k_far): the reference recurrence's flops per (target, cluster) pair, as the
    generator counts them, times the pairs of the launch, over its device time."""
    ach = flops_pair * st["far_pairs"] / st["t_far"] / 1e12
    t = "double" if prec == "fp64" else "float"
    key = f"k_far<{NTERMS}, {kname.upper()}, {t}>"
    return {"bound": "fp64" if prec == "fp64" else "fp32", "kernel": key, "precision": prec,
            "achieved": ach, "peak": peak_tflops, "unit": "TFLOP/s", "frac": ach / peak_tflops,
            "peak_source": f"measured {'FP64 DFMA' if prec == 'fp64' else 'FP32 FFMA'} throughput of "
                           "this device (bit_device_fma_peak: FMA-chain kernel, CUDA events)",
            "traffic": TRAFFIC.get(key), "traffic_unit": "bytes per launch (dram read+write)",
            "traffic_source": TRAFFIC_SOURCE if TRAFFIC.get(key) else None,
            "seconds": st["t_far"],
            "algorithmic": f"{flops_pair} flops (the reference's {kname} recurrence to degree "
                           f"{NTERMS - 1} and the moment dot product) x {st['far_pairs']} "
                           "(target, cluster) pairs per launch"}


def roofline_near(prec, kname, st, n, peak_tflops):
    """Near field (k_near): the per-pair flops of the reference's leaf loop (rsqrt and exp
    counted as 1) times the (target, source) pairs of the launch, self pairs excluded."""
    pairs = st["near_pairs"] - n
    fl = FLOPS_NEAR[kname]
    ach = fl * pairs / st["t_near"] / 1e12
    t = "F64" if prec == "fp64" else "F32"
    key = f"k_near<{kname.upper()}, {t}>"
    out = {"bound": "fp64" if prec == "fp64" else "fp32+mufu", "kernel": key, "precision": prec,
           "achieved": ach, "peak": peak_tflops, "unit": "TFLOP/s", "frac": ach / peak_tflops,
           "peak_source": f"measured {'FP64 DFMA' if prec == 'fp64' else 'FP32 FFMA'} throughput of "
                          "this device (bit_device_fma_peak)",
           "traffic": TRAFFIC.get(key), "traffic_unit": "bytes per launch (dram read+write)",
           "traffic_source": TRAFFIC_SOURCE if TRAFFIC.get(key) else None,
           "seconds": st["t_near"],
           "algorithmic": f"{fl} flops x {pairs} near pairs per launch"}
    if prec == "fp64":
        ops = FP64_OPS_NEAR[kname]
        ceiling = fl / (2.0 * ops)
        out["fp64_ops_per_pair"] = ops
        out["frac_ceiling"] = ceiling
        out["frac_of_ceiling"] = out["frac"] / ceiling
    return out


def run_matched_c2(step, timed, ctx, x, y, z, q, out_s, out_c, args):
    """The clustered 2M step at (p, theta, N0) where the plain FP64 treecode reaches 1e-6
    relative L2 against the FP64 direct sum: FP64 and mixed evals/s and errors."""
    import bit_b200 as B
    from bit_b200 import workloads
    kw = dict(nterms=MATCHED_C2["nterms"], maxmemb=MATCHED_C2["maxmemb"], acc=MATCHED_C2["acc"])
    steps = max(2, args.steps // 4)
    ms64 = timed(B.FP64, steps, 1, **kw)
    step(B.FP64, **kw)
    r64 = (out_s.cpu().numpy(), out_c.cpu().numpy())
    ms32 = timed(B.MIXED, steps, 1, **kw)
    step(B.MIXED, **kw)
    r32 = (out_s.cpu().numpy(), out_c.cpu().numpy())
    tg = workloads.sample_targets(len(x), args.sample, seed=11)
    ds = (ctx.direct(x, y, z, q, B.params(B.SCREENED, B.CONSISTENT, B.FP64, kappa=KAPPA), tg),
          ctx.direct(x, y, z, q, B.params(B.COULOMB, B.CONSISTENT, B.FP64, del_=DEL), tg))
    evals = 2 * len(x)
    out = {"workload": f"clustered N={len(x)}, screened kappa=1 + Coulomb delta=0.005, "
                       f"p={kw['nterms'] - 1}, theta={kw['acc']}, N0={kw['maxmemb']}",
           "fp64": {"evals_per_s": evals / (ms64 * 1e-3), "ms_per_step": ms64},
           "mixed": {"evals_per_s": evals / (ms32 * 1e-3), "ms_per_step": ms32},
           "mixed_speedup": ms64 / ms32, "error_targets": int(len(tg))}
    for i, name in enumerate(("screened", "coulomb")):
        out[name] = {"fp64_vs_direct": workloads.rel_l2(r64[i][tg], ds[i]),
                     "mixed_vs_direct": workloads.rel_l2(r32[i][tg], ds[i]),
                     "mixed_vs_fp64": workloads.rel_l2(r32[i], r64[i])}
    errs = [out[k][m] for k in ("screened", "coulomb") for m in ("fp64_vs_direct", "mixed_vs_direct")]
    out["max_error_vs_direct"] = max(errs)
    out["at_most_1e-6"] = max(errs) <= 1e-6
    return out


def run_bie(ctx, args, nterms=7, acc=0.5, maxmemb=500):
    """Boundary-integral GMRES solve: icosphere level 6 (81,920 centroids, weights = areas),
    (I/2 + K) sigma = f, K the area-weighted screened kernel (kappa = 1) regularised with
    delta = mean edge length, f = real spherical harmonics of degree <= 8 with seeded
    N(0,1) coefficients; p = 6, theta = 0.5, N0 = 500 (or the given p, theta, N0),
    GMRES(50) to 1e-8.  Plain FP64 matvecs vs FP32 matvecs inside FP64 iterative
    refinement; device seconds per solve."""
    import bit_b200 as B
    from bit_b200 import workloads
    cen, area, h = workloads.icosphere(args.bie_level)
    f = workloads.sh_rhs(cen, lmax=8, seed=1)
    cx, cy, cz = [np.ascontiguousarray(cen[:, a]) for a in range(3)]
    p = B.params(B.SCREENED_REG, B.CONSISTENT, B.FP64, del_=h * h, kappa=1.0, acc=acc)
    t = ctx.treemake(cx, cy, cz, maxmemb)
    out = {"workload": f"icosphere level {args.bie_level} ({len(cen)} nodes), screened kappa=1 "
                       f"regularised with delta = mean edge ({h:.4g}), p={nterms - 1}, "
                       f"theta={acc}, N0={maxmemb}, GMRES(50) to 1e-8", "n": int(len(cen))}
    tg = workloads.sample_targets(len(cen), 2000, seed=4)
    for name, prec in (("fp64", B.FP64), ("mixed", B.MIXED)):
        t.bie_solve(p, nterms, 0.5, area, f, restart=50, tol=1e-8, precision=prec)  # warm-up
        secs, info, sol, st = [], None, None, None
        for _ in range(args.bie_solves):
            sol, info, st = t.bie_solve(p, nterms, 0.5, area, f, restart=50, tol=1e-8, precision=prec)
            secs.append(info["seconds"])
        # residual of the solution against the direct-sum operator on sampled rows
        Ks = ctx.direct(cx, cy, cz, area * sol, p, tg)
        res = workloads.rel_l2(0.5 * sol[tg] + Ks, f[tg])
        out[name] = {"solves_per_s": 1.0 / statistics.median(secs),
                     "s_per_solve": statistics.median(secs), "status": int(st),
                     "iterations": info["iterations"], "refinements": info["refinements"],
                     "matvecs_fp64": info["matvecs_fp64"], "matvecs_fp32": info["matvecs_fp32"],
                     "relres_treecode": info["relres"], "relres_direct_sum_2000_rows": res}
    out["mixed_speedup"] = out["fp64"]["s_per_solve"] / out["mixed"]["s_per_solve"]
    errs = [out[k]["relres_direct_sum_2000_rows"] for k in ("fp64", "mixed")]
    out["max_error_vs_direct"] = max(errs)
    out["at_most_1e-6"] = max(errs) <= 1e-6
    t.treeempty()
    return out


def run_batched(ctx, args, dev, acc_by_nterms=None):
    """Batched uneven systems in one pass: 2048 independent systems, N log-uniform in
    [1e3, 1e5], each uniform in its own unit cube; half regularised Coulomb (delta = 0.01),
    half screened (kappa ~ U[0.5, 4]); p from {4, 6, 8}; theta = 0.6; N0 per (p, kernel)
    from the autotuner.  Mixed precision as one forest (build, moments, far and near
    launches per class) vs a per-system loop of the plain FP64 path, and the plain FP64
    path as one forest (which separates the precision gain from the batching gain); error
    vs the FP64 direct sum on 1,000 sampled targets per system.  acc_by_nterms: theta per
    expansion order instead of 0.6 (the accuracy-matched run)."""
    import torch
    import bit_b200 as B
    from bit_b200 import autotune, workloads
    systems = workloads.batched_systems(args.batched, seed=3)
    sizes = np.array([len(s["x"]) for s in systems], dtype=np.int64)
    med = int(np.median(sizes))
    n0 = {}
    for s in systems:
        key = (s["nterms"], s["kernel"])
        if key not in n0:
            n0[key] = autotune.tune_n0(ctx, s["nterms"], s["kernel"], med,
                                       acc=0.6 if acc_by_nterms is None else acc_by_nterms[s["nterms"]],
                                       del_=1e-4 if s["kernel"] == B.COULOMB else 0.0,
                                       kappa=2.0)[0]
    mm = np.array([n0[(s["nterms"], s["kernel"])] for s in systems], dtype=np.int32)
    nt = np.array([s["nterms"] for s in systems], dtype=np.int32)
    total = int(sizes.sum())
    off = np.concatenate([[0], np.cumsum(sizes)])
    X = torch.tensor(np.stack([np.concatenate([s[k] for s in systems]) for k in "xyzq"]),
                     dtype=torch.float64, device=dev)
    out32 = torch.empty(total, dtype=torch.float64, device=dev)
    out64 = torch.empty(total, dtype=torch.float64, device=dev)
    outf64 = torch.empty(total, dtype=torch.float64, device=dev)

    def theta(s):
        return 0.6 if acc_by_nterms is None else acc_by_nterms[s["nterms"]]

    def prm(s, prec):
        return B.params(s["kernel"], B.CONSISTENT, prec, del_=s["del_"], kappa=s["kappa"], acc=theta(s))
    p32 = [prm(s, B.MIXED) for s in systems]
    p64 = [prm(s, B.FP64) for s in systems]
    ptr = [X[k].data_ptr() for k in range(4)]

    def forest_step(prec=B.MIXED):
        F = ctx.forest_device(sizes, mm, ptr[0], ptr[1], ptr[2])
        F.set_charges_device(ptr[3])
        F.moments(nt)
        if prec == B.MIXED:
            F.evaluate_device(p32, out32.data_ptr())
        else:
            F.evaluate_device(p64, outf64.data_ptr())
        st = F.stats()
        F.treeempty()
        return st

    def loop_step(prec, out):
        for i, s in enumerate(systems):
            o = int(off[i]) * 8
            t = ctx.treemake_device(int(sizes[i]), ptr[0] + o, ptr[1] + o, ptr[2] + o, int(mm[i]))
            t.set_charges_device(ptr[3] + o)
            t.moments(int(nt[i]))
            t.evaluate_device(prm(s, prec), out.data_ptr() + o)
            t.treeempty()

    def timed(fn, reps):
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        r = None
        for _ in range(reps):
            r = fn()
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / reps * 1e-3, r

    # leaf packing for the forest: timed on the whole batch, fastest kept
    group, gtimes = autotune.tune_group(ctx, lambda c: timed(forest_step, 1)[0])
    forest_step()  # warm-up
    t32, st = timed(forest_step, 2)
    forest_step(B.FP64)  # warm-up
    tf64, _ = timed(lambda: forest_step(B.FP64), 2)
    ctx.set_group_size(0)  # the plain FP64 path in its default configuration
    loop_step(B.FP64, out64)  # warm-up
    t64, _ = timed(lambda: loop_step(B.FP64, out64), 1)
    r32 = out32.cpu().numpy()
    r64 = out64.cpu().numpy()
    rf64 = outf64.cpu().numpy()
    e32, e64 = [], []
    for i, s in enumerate(systems):
        tg = workloads.sample_targets(int(sizes[i]), 1000, seed=i)
        ds = ctx.direct(s["x"], s["y"], s["z"], s["q"], p64[i], tg)
        e32.append(workloads.rel_l2(r32[off[i]:off[i + 1]][tg], ds))
        e64.append(workloads.rel_l2(r64[off[i]:off[i + 1]][tg], ds))
    mix_vs_64 = [workloads.rel_l2(r32[off[i]:off[i + 1]], r64[off[i]:off[i + 1]])
                 for i in range(len(systems))]
    forest_vs_loop = max(workloads.rel_l2(rf64[off[i]:off[i + 1]], r64[off[i]:off[i + 1]])
                         for i in range(len(systems)))
    th = ("theta=0.6" if acc_by_nterms is None else
          "theta by p: " + ", ".join(f"p={k - 1}: {v}" for k, v in sorted(acc_by_nterms.items())))
    err_all = e32 + e64
    return {"workload": f"{len(systems)} systems, N log-uniform in [1e3, 1e5] (total {total}), "
                        "half Coulomb delta=0.01, half screened kappa~U[0.5,4], p in {4,6,8}, "
                        f"{th}, N0 autotuned per (p, kernel), leaf packing autotuned for the batch",
            "systems": len(systems), "particles": total,
            "n0": {f"nterms{k[0]}_{'coulomb' if k[1] == 0 else 'screened'}": v
                   for k, v in sorted(n0.items())},
            "group_size": group, "group_size_times_s": {str(k): v for k, v in gtimes.items()},
            "mixed_forest": {"evals_per_s": total / t32, "s_per_step": t32,
                             "far_launches": st["far_launches"], "near_launches": st["near_launches"]},
            "fp64_per_system_loop": {"evals_per_s": total / t64, "s_per_step": t64},
            "fp64_forest": {"evals_per_s": total / tf64, "s_per_step": tf64,
                            "max_rel_diff_vs_loop": forest_vs_loop},
            "speedup": t64 / t32,
            "speedup_precision_only": tf64 / t32,
            "speedup_batching_only": t64 / tf64,
            "max_error_vs_direct": float(np.max(err_all)),
            "at_most_1e-6": bool(np.max(err_all) <= 1e-6),
            "error_vs_direct_1000_per_system": {
                "mixed_median": float(np.median(e32)), "mixed_max": float(np.max(e32)),
                "fp64_median": float(np.median(e64)), "fp64_max": float(np.max(e64)),
                "mixed_vs_fp64_max": float(np.max(mix_vs_64))}}


def serving_requests(count, seed, ctx, matched=False):
    """The request stream: 70% evaluate requests (N lognormal, median 20,000, clipped to
    [1e3, 1e6], Gaussian blobs; kernel and parameters as in the batched run) and 30%
    GMRES solves on icospheres of level 4..7 (system as in the boundary-integral solve).
    matched: theta per p of the accuracy-matched batched run, and the accuracy-matched
    boundary-integral parameters for the solves."""
    import bit_b200 as B
    from bit_b200 import autotune, workloads
    rng = np.random.default_rng(seed)
    spheres = {}
    reqs = []
    for i in range(count):
        if rng.uniform() < 0.7:
            n = int(np.clip(round(20000 * np.exp(rng.normal(0.0, 1.0))), 1000, 1_000_000))
            x, y, z, q = workloads.clustered_blobs(n, seed=seed * 100000 + i)
            coul = rng.uniform() < 0.5
            nterms = int(rng.choice([4, 6, 8])) + 1
            kappa = 0.0 if coul else float(rng.uniform(0.5, 4.0))
            kern = B.COULOMB if coul else B.SCREENED
            acc = MATCHED_BATCH_ACC[nterms] if matched else 0.6
            n0 = autotune.tune_n0(ctx, nterms, kern, 20000, acc=acc, del_=1e-4 if coul else 0.0,
                                  kappa=2.0, dist="clustered")[0]
            reqs.append(dict(kind="eval", n=n, data=(x, y, z, q), nterms=nterms, n0=n0,
                             kernel=kern, del_=1e-4 if coul else 0.0, kappa=kappa, acc=acc))
        else:
            level = int(rng.integers(4, 8))
            if level not in spheres:
                spheres[level] = workloads.icosphere(level)
            cen, area, h = spheres[level]
            f = workloads.sh_rhs(cen, lmax=8, seed=seed * 100000 + i)
            cx, cy, cz = [np.ascontiguousarray(cen[:, a]) for a in range(3)]
            sp = MATCHED_BIE if matched else dict(nterms=7, acc=0.5, maxmemb=500)
            reqs.append(dict(kind="solve", n=len(cen), data=(cx, cy, cz, area, f),
                             nterms=sp["nterms"], n0=sp["maxmemb"], acc=sp["acc"], del_=h * h,
                             level=level))
    return reqs


def serve(reqs, arrivals, prec, srv, slots):
    """Submit request i at arrivals[i] seconds (open loop) to the running server srv and
    collect every result."""
    import threading
    import bit_b200 as B
    ids = [None] * len(reqs)

    def producer():
        t0 = time.perf_counter()
        for i, r in enumerate(reqs):
            dt = arrivals[i] - (time.perf_counter() - t0)
            if dt > 0:
                time.sleep(dt)
            if r["kind"] == "eval":
                p = B.params(r["kernel"], B.CONSISTENT, prec, del_=r["del_"], kappa=r["kappa"], acc=r["acc"])
                ids[i] = srv.submit_eval(*r["data"], r["nterms"], r["n0"], p)
            else:
                p = B.params(B.SCREENED_REG, B.CONSISTENT, B.FP64, del_=r["del_"], kappa=1.0, acc=r["acc"])
                x, y, z, w, f = r["data"]
                ids[i] = srv.submit_solve(x, y, z, w, f, r["nterms"], r["n0"], p, 0.5, restart=50,
                                          tol=1e-8, precision=prec)
    th = threading.Thread(target=producer)
    th.start()
    th.join()
    out, infos = [], []
    for i in range(len(reqs)):
        res, info, st = srv.wait(ids[i])
        out.append(res)
        info["status"] = st
        infos.append(info)
    lat = np.array([i["t_done"] - i["t_submit"] for i in infos])
    span = max(i["t_done"] for i in infos) - min(i["t_submit"] for i in infos)
    # most requests running at once in this stream: +1 at each start, -1 at each finish
    ev = sorted([(i["t_start"], 1) for i in infos] + [(i["t_done"], -1) for i in infos])
    running = np.cumsum([d for _, d in ev])
    return out, {"requests_per_s": len(reqs) / span, "p50_latency_s": float(np.percentile(lat, 50)),
                 "p99_latency_s": float(np.percentile(lat, 99)), "mean_latency_s": float(lat.mean()),
                 "max_running": int(running.max()), "slots": slots,
                 "failed": int(sum(1 for i in infos if i["status"] not in (0,)))}


def run_serving(ctx, args, matched=False):
    """Serving stream: open-loop Poisson arrivals of the request mix at 80% of the warm mixed
    server's measured capacity, admitted by a 150 GB HBM budget into a continuous-batching
    server (mixed precision, several slots), next to the plain FP64 GPU path serving one
    request at a time on the same arrivals.  matched: the accuracy-matched parameters."""
    import bit_b200 as B
    from bit_b200 import workloads
    reqs = serving_requests(args.serve_requests, seed=5, ctx=ctx, matched=matched)
    budget = 150 * 10 ** 9
    # Each server is long-lived, as in deployment: it first serves the whole request set
    # once (every buffer grown, every plan made), then the timed streams.  Arrival rate:
    # 80% of the warm mixed server's capacity, measured closed-loop (every request queued
    # at t = 0).
    closed = [0.0] * len(reqs)
    load = 0.8
    srv = B.Server(slots=args.serve_slots, hbm_budget=budget)
    try:
        serve(reqs, closed, B.MIXED, srv, args.serve_slots)
        with ClockSampler(int(os.environ.get("LOCAL_RANK", 0))) as clk:
            _, cap = serve(reqs, closed, B.MIXED, srv, args.serve_slots)
        cap_clocks = clk.summary()
        rate = load * cap["requests_per_s"]
        rng = np.random.default_rng(6)
        arrivals = np.cumsum(rng.exponential(1.0 / rate, len(reqs)))
        res32, mixed = serve(reqs, arrivals, B.MIXED, srv, args.serve_slots)
    finally:
        srv.close()
    srv = B.Server(slots=1, hbm_budget=budget)
    try:
        serve(reqs, closed, B.FP64, srv, 1)
        _, cap64 = serve(reqs, closed, B.FP64, srv, 1)
        res64, plain = serve(reqs, arrivals, B.FP64, srv, 1)
    finally:
        srv.close()
    # accuracy: mixed vs plain FP64 per request; evaluate requests also vs the direct sum
    diff = [workloads.rel_l2(a, b) for a, b in zip(res32, res64)]
    derr, serr = [], []
    for i, r in enumerate(reqs):
        tg = workloads.sample_targets(r["n"], 200, seed=i)
        if r["kind"] == "eval":
            x, y, z, q = r["data"]
            p = B.params(r["kernel"], B.CONSISTENT, B.FP64, del_=r["del_"], kappa=r["kappa"])
            for res in (res32, res64):
                derr.append(workloads.rel_l2(res[i][tg], ctx.direct(x, y, z, q, p, tg)))
        else:
            x, y, z, w, f = r["data"]
            p = B.params(B.SCREENED_REG, B.CONSISTENT, B.FP64, del_=r["del_"], kappa=1.0)
            for res in (res32, res64):
                Ks = ctx.direct(x, y, z, w * res[i], p, tg)
                serr.append(workloads.rel_l2(0.5 * res[i][tg] + Ks, f[tg]))
    kinds = [r["kind"] for r in reqs]
    th = "theta by p " + str({k - 1: v for k, v in sorted(MATCHED_BATCH_ACC.items())}) if matched else "theta 0.6"
    sp = MATCHED_BIE if matched else dict(nterms=7, acc=0.5, maxmemb=500)
    return {"workload": f"{len(reqs)} requests, Poisson arrivals at {rate:.1f}/s "
                        f"({load:.0%} of the warm mixed server's closed-loop capacity, "
                        f"{cap['requests_per_s']:.1f}/s) "
                        f"({kinds.count('eval')} evaluate: N lognormal median 2e4 in [1e3, 1e6], "
                        f"blobs, p in {{4,6,8}}, {th}; {kinds.count('solve')} solves: "
                        f"icosphere level 4..7, p={sp['nterms'] - 1}, theta={sp['acc']}, "
                        f"N0={sp['maxmemb']}, GMRES(50) to 1e-8), 150 GB budget",
            "offered_load": load, "mixed_closed_loop_requests_per_s": cap["requests_per_s"],
            "mixed_closed_loop_clocks": cap_clocks,
            "fp64_closed_loop_requests_per_s": cap64["requests_per_s"],
            "capacity_ratio": cap["requests_per_s"] / cap64["requests_per_s"],
            "mixed_continuous_batching": mixed, "fp64_one_at_a_time": plain,
            "throughput_ratio": mixed["requests_per_s"] / plain["requests_per_s"],
            "p99_ratio": plain["p99_latency_s"] / mixed["p99_latency_s"],
            "mixed_vs_fp64_max": float(max(diff)),
            "eval_error_vs_direct_200_targets": {"median": float(np.median(derr)),
                                                 "max": float(np.max(derr))},
            "solve_residual_vs_direct_200_rows": {"median": float(np.median(serr)) if serr else None,
                                                  "max": float(np.max(serr)) if serr else None},
            "max_error_vs_direct": float(max(derr + serr)),
            "at_most_1e-6": bool(max(derr + serr) <= 1e-6)}


def far_flops_per_pair(nterms):
    """Flops per (target, cluster) pair of the generated far-field recurrences, counted from
    the generator (bit_b200/csrc/gen_farfield.py)."""
    import importlib.util
    spec = importlib.util.spec_from_file_location(
        "gen_farfield", os.path.join(ROOT, "bit_b200", "csrc", "gen_farfield.py"))
    g = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(g)
    return g.flops_per_pair(nterms)


def accuracy(ctx, x, y, z, q, s32, c32, s64, c64, args):
    """Relative L2 error against the FP64 direct sum on args.sample seeded targets.  The
    direct sum runs on the GPU (bit_direct_potential, FP64); it is itself checked against
    the CPU oracle's direct sum on the first args.oracle_sample of those targets."""
    import bit_b200 as B
    from bit_b200 import workloads
    from oracle import orc
    tg = workloads.sample_targets(len(x), args.sample, seed=11)
    ds_s = ctx.direct(x, y, z, q, B.params(B.SCREENED, B.CONSISTENT, B.FP64, kappa=KAPPA), tg)
    ds_c = ctx.direct(x, y, z, q, B.params(B.COULOMB, B.CONSISTENT, B.FP64, del_=DEL), tg)
    sub = tg[:args.oracle_sample]
    ps = orc.params(orc.SCREENED, orc.MODE_CONSISTENT, kappa=KAPPA, acc=ACC)
    pc = orc.params(orc.COULOMB, orc.MODE_CONSISTENT, del_=DEL, acc=ACC)
    pin_s = workloads.rel_l2(ds_s[:len(sub)], orc.direct(x, y, z, q, ps, sub))
    pin_c = workloads.rel_l2(ds_c[:len(sub)], orc.direct(x, y, z, q, pc, sub))
    return {
        "direct_sum_targets": int(len(tg)),
        "direct_sum": f"FP64 on the GPU; equals the CPU oracle's direct sum on {len(sub)} of "
                      f"the targets to {max(pin_s, pin_c):.1e} relative",
        "screened": {"mixed_vs_direct": workloads.rel_l2(s32[tg], ds_s),
                     "fp64_vs_direct": workloads.rel_l2(s64[tg], ds_s),
                     "mixed_vs_fp64": workloads.rel_l2(s32, s64)},
        "coulomb": {"mixed_vs_direct": workloads.rel_l2(c32[tg], ds_c),
                    "fp64_vs_direct": workloads.rel_l2(c64[tg], ds_c),
                    "mixed_vs_fp64": workloads.rel_l2(c32, c64)},
    }


def cpu_reference_time(x, y, z, q, n, sample, threads):
    """The reference's own treemake + treemoments + shielded_treepot / treepotential
    (oracle/_ref, OpenMP over targets like tests/treecode_mp.cpp:83-95) on all host cores;
    the evaluation is timed on `sample` seeded targets and scaled to all N."""
    from oracle import ref
    from bit_b200 import workloads
    if not ref.available(DEL):
        return None
    tg = workloads.sample_targets(n, sample, seed=5)
    t0 = time.perf_counter()
    R = ref.RefTree(x, y, z, q, NTERMS, MAXMEMB, del_=DEL)
    t1 = time.perf_counter()
    R.moments()
    t2 = time.perf_counter()
    R.screened(KAPPA, ACC, tg, nthreads=threads)
    t3 = time.perf_counter()
    R.potential(ACC, tg, nthreads=threads)
    t4 = time.perf_counter()
    R.close()
    per_target = (t4 - t2) / len(tg)  # both kernels
    total = (t1 - t0) + (t2 - t1) + per_target * n
    return {"build_s": t1 - t0, "moments_s": t2 - t1, "eval_sample_s": t4 - t2,
            "est_step_s": total, "evals_per_s": 2 * n / total}


def cpu_baseline(x, y, z, q, n, args):
    threads = os.cpu_count() or 1
    r = cpu_reference_time(x, y, z, q, n, args.cpu_sample, threads)
    if r is None:
        return {"value": None, "unit": "evals/s", "cores": threads, "kind": "reference",
                "sample": "reference build not present"}
    return {"value": r["evals_per_s"], "unit": "evals/s", "cores": threads, "kind": "reference",
            "sample": f"full treemake+treemoments ({r['build_s']:.2f}+{r['moments_s']:.2f} s) and "
                      f"screened+Coulomb evaluation of {args.cpu_sample} seeded targets "
                      f"({r['eval_sample_s']:.2f} s) scaled to all {n}; Coulomb uses the reference "
                      "with moment arrays padded to (nterms+1)^3 (its degree-nterms read is out of bounds)",
            "detail": r}


def run_reference(args):
    from bit_b200 import replicas
    rank, world, _ = replicas.rank_info()
    if rank != 0:
        return
    threads = os.cpu_count() or 1
    x, y, z, q = workload(args.n, seed=1)
    est, measured = [], []
    for i in range(args.warmup + args.steps):
        t0 = time.perf_counter()
        r = cpu_reference_time(x, y, z, q, args.n, args.ref_sample, threads)
        if r is None:
            print(json.dumps({"impl": "reference", "unavailable": "reference build (oracle/_ref) not present"}))
            return
        if i >= args.warmup:
            est.append(r["est_step_s"])
            measured.append(time.perf_counter() - t0)
    est_ms = 1e3 * statistics.mean(est)
    ms = 1e3 * statistics.mean(measured)
    v = 2 * args.n / (est_ms * 1e-3)
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": "evals/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded clustered blobs)",
            "config": {"workload": "clustered evaluation N=2,000,000 (80% in 8 Gaussian blobs sigma "
                                   "0.1, 20% uniform), p=8, theta=0.7, N0=1000, screened kappa=1 + "
                                   "Coulomb delta=0.005, all particles as targets",
                       "n": args.n, "nterms": NTERMS, "maxmemb": MAXMEMB, "acc": ACC},
            "value_basis": f"extrapolated: each step times the full treemake + treemoments and the "
                           f"evaluation of {args.ref_sample} seeded targets (both kernels), and the "
                           f"evaluation time is scaled to all {args.n} targets; ms_per_step is the "
                           "measured time of one such sampled step, extrapolated_ms_per_full_step "
                           "the estimate for all targets",
            "extrapolated_ms_per_full_step": est_ms,
            "cpu_baseline": {"value": v, "unit": "evals/s", "cores": threads, "kind": "reference",
                             "sample": f"per step: full tree build + moments, evaluation of "
                                       f"{args.ref_sample} seeded targets scaled to all N"},
            "e2e": {"value": v, "unit": "evals/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=4)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="bit", choices=["bit", "reference"])
    ap.add_argument("--n", type=int, default=2_000_000)
    ap.add_argument("--sample", type=int, default=10_000, help="direct-sum targets for the error")
    ap.add_argument("--oracle-sample", type=int, default=100,
                    help="of those, targets also summed by the CPU oracle")
    ap.add_argument("--cpu-sample", type=int, default=300_000,
                    help="targets of the CPU baseline's evaluation sample (about 10 s on 16 cores)")
    ap.add_argument("--ref-sample", type=int, default=100_000,
                    help="targets per step of the --impl reference arm")
    ap.add_argument("--no-cpu-baseline", dest="cpu_baseline", action="store_false")
    ap.add_argument("--bie-level", type=int, default=6, help="icosphere level of the GMRES solve")
    ap.add_argument("--bie-solves", type=int, default=2)
    ap.add_argument("--no-bie", dest="bie", action="store_false")
    ap.add_argument("--batched", type=int, default=2048, help="systems of the batched run (0: skip)")
    ap.add_argument("--serve-requests", type=int, default=120,
                    help="requests of the serving stream (0: skip)")
    ap.add_argument("--serve-slots", type=int, default=8)
    ap.add_argument("--no-matched", dest="matched", action="store_false",
                    help="skip the accuracy-matched (1e-6 vs direct sum) runs")
    ap.add_argument("--no-tune", dest="tune", action="store_false",
                    help="default near-field tile and threads per target instead of tuned ones")
    args = ap.parse_args()
    if args.impl == "reference":
        run_reference(args)
    else:
        run_bit(args)


if __name__ == "__main__":
    main()

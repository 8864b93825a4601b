"""Treecode benchmark on B200 (one JSON line on rank 0).

Workload (one "step"): the large clustered evaluation -- N = 2,000,000 particles, 80% in
8 Gaussian blobs (sigma 0.1), 20% uniform in [-1,1]^3, charges U[-1,1] (seeded); tree
build (N0 = 1000), FP64 moments for p = 8 (nterms 9), then the potential at every
particle twice: screened kernel exp(-kappa r)/r with kappa = 1, and regularised Coulomb
1/sqrt(r^2 + delta^2) with delta = 0.005, both with MAC theta = 0.7.  evals = 2 N per step.

value  -- evals/s with the inputs resident in HBM (mixed precision: FP32 near/far field in
          cluster-centred coordinates with compensated accumulation; FP64 MAC and moments)
e2e    -- the same through the C ABI with host buffers (H2D inputs, D2H potentials inside
          the timed region)
fp64   -- the plain FP64 GPU path on the same step, for the mixed-vs-FP64 speed-up

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
METRIC = "treecode evals/s (clustered N=2M, p=8, theta=0.7, N0=1000, screened+Coulomb)"


def rank_info():
    return (int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1)),
            int(os.environ.get("LOCAL_RANK", 0)))


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
    from bit_b200 import workloads

    rank, world, local = rank_info()
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import torch.distributed as dist
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    n = args.n
    x, y, z, q = workload(n, seed=1 + rank)
    dev = torch.device("cuda", local)
    X = torch.tensor(np.stack([x, y, z, q]), dtype=torch.float64, device=dev)
    out_s = torch.empty(n, dtype=torch.float64, device=dev)
    out_c = torch.empty(n, dtype=torch.float64, device=dev)
    stream = torch.cuda.current_stream(dev)
    ctx = B.Context(local, stream=stream.cuda_stream)

    def step(prec, keep=False):
        t = ctx.treemake_device(n, X[0].data_ptr(), X[1].data_ptr(), X[2].data_ptr(), MAXMEMB)
        t.set_charges_device(X[3].data_ptr())
        t.moments(NTERMS)
        t.evaluate_device(B.params(B.SCREENED, B.CONSISTENT, prec, kappa=KAPPA, acc=ACC),
                          out_s.data_ptr())
        st_s = t.stats() if keep else None
        t.evaluate_device(B.params(B.COULOMB, B.CONSISTENT, prec, del_=DEL, acc=ACC),
                          out_c.data_ptr())
        st_c = t.stats() if keep else None
        if keep:
            return t, st_s, st_c
        t.treeempty()
        return None

    launches = {}

    def timed(prec, steps, warmup):
        for _ in range(warmup):
            step(prec)
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        l0 = B.kernel_launches()
        e0.record(stream)
        for _ in range(steps):
            step(prec)
        e1.record(stream)
        torch.cuda.synchronize()
        launches[prec] = (B.kernel_launches() - l0) // steps
        ms = e0.elapsed_time(e1) / steps
        if dist:
            t = torch.tensor([ms], device=dev)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            ms = float(t.item())
        return ms

    # mixed precision (the product path): timed with clocks sampled
    with ClockSampler(local) as clk:
        ms = timed(B.MIXED, args.steps, args.warmup)
    clocks = clk.summary()
    ms64 = timed(B.FP64, max(1, args.steps // 2), 1)
    # per-kernel device times of one step (events on the library's stream)
    t, st_s, st_c = step(B.MIXED, keep=True)
    res_s = out_s.cpu().numpy()
    res_c = out_c.cpu().numpy()
    t.treeempty()
    _, st64_s, st64_c = step(B.FP64, keep=True)
    res64_s = out_s.cpu().numpy()
    res64_c = out_c.cpu().numpy()

    # e2e through the C ABI with host buffers
    def e2e_step():
        t = ctx.treemake(x, y, z, MAXMEMB)
        t.treemoments(q, NTERMS)
        a = t.evaluate(B.params(B.SCREENED, B.CONSISTENT, B.MIXED, kappa=KAPPA, acc=ACC))
        b = t.evaluate(B.params(B.COULOMB, B.CONSISTENT, B.MIXED, del_=DEL, acc=ACC))
        t.treeempty()
        return a, b
    for _ in range(max(1, args.warmup // 2)):
        e2e_step()
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    t0 = time.perf_counter()
    e2e_steps = max(1, args.steps // 2)
    for _ in range(e2e_steps):
        e2e_step()
    torch.cuda.synchronize()
    e2e_ms = (time.perf_counter() - t0) * 1e3 / e2e_steps
    if dist:
        tt = torch.tensor([e2e_ms], device=dev)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        e2e_ms = float(tt.item())

    if rank != 0:
        if dist:
            dist.barrier()
            dist.destroy_process_group()
        return

    evals = 2 * n * world
    line = {
        "metric": METRIC, "value": evals / (ms * 1e-3), "unit": "evals/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32 near/far field, f64 MAC+moments",
        "data": "synthetic (seeded clustered blobs)",
        "config": {"workload": "clustered evaluation N=2,000,000 (80% in 8 Gaussian blobs sigma 0.1, "
                               "20% uniform), p=8, theta=0.7, N0=1000, screened kappa=1 + Coulomb "
                               "delta=0.005, all particles as targets",
                   "n": n, "nterms": NTERMS, "maxmemb": MAXMEMB, "acc": ACC,
                   "parallelism": f"replicas x{world}",
                   "l2": "inputs (128 MB coordinates+charges, 64 MB sorted FP64 sources) exceed the "
                         "126 MB L2; no flush"},
        "clocks": clocks,
        "fp64": {"value": evals / (ms64 * 1e-3), "ms_per_step": ms64,
                 "mixed_speedup": ms64 / ms},
    }
    e2e_in = 4 * n * 8
    e2e_out = 2 * n * 8
    line["e2e"] = {"value": 2 * n * world / (e2e_ms * 1e-3), "unit": "evals/s",
                   "h2d_bytes_per_step": e2e_in, "d2h_bytes_per_step": e2e_out,
                   "ms_per_step": e2e_ms}
    # per-phase device times and interaction counts (mixed, screened + Coulomb)
    phases = {}
    for name, st in (("screened", st_s), ("coulomb", st_c)):
        phases[name] = {k: st[k] for k in ("t_far", "t_near", "t_lists", "far_pairs", "near_pairs",
                                           "far_entries", "near_entries", "batches")}
    phases["build_s"] = st_s["t_build"]
    phases["moments_s"] = st_s["t_moments"]
    phases["numtree"] = st_s["numtree"]
    phases["fp64"] = {name: {"t_far": s["t_far"], "t_near": s["t_near"]}
                      for name, s in (("screened", st64_s), ("coulomb", st64_c))}
    line["phases"] = phases
    # dominant kernel roofline: the screened near field
    pairs = st_s["near_pairs"] - n
    flops = FLOPS_NEAR["screened"] * pairs
    t_near = st_s["t_near"]
    achieved = flops / t_near / 1e12
    peak = fp32_peak_from_clock(clocks)
    line["roofline"] = {"bound": "fp32", "kernel": "k_near32<SCREENED>",
                        "achieved": achieved, "peak": peak["tflops"], "unit": "TFLOP/s",
                        "frac": achieved / peak["tflops"], "peak_source": peak["source"],
                        "traffic": None,
                        "algorithmic": f"{FLOPS_NEAR['screened']} flops x {pairs} near pairs per launch",
                        "mufu_bound_frac": (2 * pairs / t_near) / peak["mufu_ops"]}
    # accuracy of this step against the FP64 GPU path and the FP64 direct sum (sampled)
    line["accuracy"] = accuracy(x, y, z, q, res_s, res_c, res64_s, res64_c, args)
    if args.cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(x, y, z, q, n, args)
    line["gpu_launches"] = launches[B.MIXED] * args.steps
    line["gpu_launches_per_step"] = launches[B.MIXED]
    print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()


def fp32_peak_from_clock(clocks):
    """Nominal B200 CUDA-core FP32 peak at the sampled SM clock: 148 SMs x 128 FFMA/clk x 2
    flops; MUFU (rsqrt / ex2) peak 148 x 16 ops/clk."""
    mhz = clocks.get("sm_mhz") or 1965.0
    return {"tflops": 148 * 128 * 2 * mhz * 1e6 / 1e12, "mufu_ops": 148 * 16 * mhz * 1e6,
            "source": f"nominal 148x128 FFMA/clk at the sampled median SM clock ({mhz:.0f} MHz); "
                      "MEASURED_PEAKS.json has no CUDA-core FP32 figure"}


def accuracy(x, y, z, q, s32, c32, s64, c64, args):
    from bit_b200 import workloads
    from oracle import orc
    tg = workloads.sample_targets(len(x), args.sample, seed=11)
    ps = orc.params(orc.SCREENED, orc.MODE_CONSISTENT, kappa=KAPPA, acc=ACC)
    pc = orc.params(orc.COULOMB, orc.MODE_CONSISTENT, del_=DEL, acc=ACC)
    ds_s = orc.direct(x, y, z, q, ps, tg)
    ds_c = orc.direct(x, y, z, q, pc, tg)
    return {
        "direct_sum_targets": int(len(tg)),
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
    rank, world, _ = rank_info()
    if rank != 0:
        return
    threads = os.cpu_count() or 1
    x, y, z, q = workload(args.n, seed=1)
    times = []
    for i in range(args.warmup + args.steps):
        r = cpu_reference_time(x, y, z, q, args.n, args.cpu_sample, threads)
        if r is None:
            print(json.dumps({"impl": "reference", "unavailable": "reference build (oracle/_ref) not present"}))
            return
        if i >= args.warmup:
            times.append(r["est_step_s"])
    ms = 1e3 * statistics.mean(times)
    v = 2 * args.n / (ms * 1e-3)
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": "evals/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded clustered blobs)",
            "config": {"workload": "clustered evaluation N=2,000,000, p=8, theta=0.7, N0=1000, "
                                   "screened kappa=1 + Coulomb delta=0.005", "n": args.n},
            "cpu_baseline": {"value": v, "unit": "evals/s", "cores": threads, "kind": "reference",
                             "sample": f"per step: full tree build + moments, evaluation of "
                                       f"{args.cpu_sample} seeded targets scaled to all N"},
            "e2e": {"value": v, "unit": "evals/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=4)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="bit", choices=["bit", "reference"])
    ap.add_argument("--n", type=int, default=2_000_000)
    ap.add_argument("--sample", type=int, default=400, help="direct-sum targets for the error")
    ap.add_argument("--cpu-sample", type=int, default=2000)
    ap.add_argument("--no-cpu-baseline", dest="cpu_baseline", action="store_false")
    args = ap.parse_args()
    if args.impl == "reference":
        run_reference(args)
    else:
        run_bit(args)


if __name__ == "__main__":
    main()

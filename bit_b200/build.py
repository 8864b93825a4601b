"""Build libbit_b200.so (sm_100a) in-tree: bit_b200/lib/libbit_b200.so.

    python -m bit_b200.build [--force] [--verbose]

Generates the unrolled far-field recurrences (csrc/gen_farfield.py), compiles every
csrc/*.cu for sm_100a with nvcc, and links one shared library exporting the C ABI of
include/bit_b200.h.  Objects are rebuilt only when a source or header is newer.
"""
import argparse
import concurrent.futures as cf
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
GEN = os.path.join(CSRC, "generated")
OBJ = os.path.join(HERE, "lib", "obj")
LIB = os.path.join(HERE, "lib", "libbit_b200.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-O2",
         "--expt-relaxed-constexpr", "-I", os.path.join(ROOT, "include"), "-I", CSRC]
HOST_CXX = "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else "g++"


def _newer(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def sources():
    return sorted(f for f in os.listdir(CSRC) if f.endswith(".cu"))


def headers():
    hs = [os.path.join(ROOT, "include", h) for h in os.listdir(os.path.join(ROOT, "include"))]
    hs += [os.path.join(CSRC, h) for h in os.listdir(CSRC) if h.endswith((".cuh", ".h"))]
    if os.path.isdir(GEN):
        hs += [os.path.join(GEN, h) for h in os.listdir(GEN)]
    return hs


def build(force=False, verbose=False, extra=()):
    os.makedirs(GEN, exist_ok=True)
    os.makedirs(OBJ, exist_ok=True)
    gen_out = os.path.join(GEN, "farfield_gen.cuh")
    gen_src = os.path.join(CSRC, "gen_farfield.py")
    if force or _newer(gen_out, [gen_src]):
        subprocess.run([sys.executable, gen_src, gen_out], check=True)
    deps = headers()
    jobs = []
    for s in sources():
        src = os.path.join(CSRC, s)
        obj = os.path.join(OBJ, s[:-3] + ".o")
        if force or _newer(obj, [src] + deps):
            cmd = [NVCC, "-ccbin", HOST_CXX] + ARCH + FLAGS + list(extra) + ["-c", src, "-o", obj]
            jobs.append((s, cmd))
    def run(job):
        name, cmd = job
        if verbose:
            print(" ".join(cmd), flush=True)
        r = subprocess.run(cmd, capture_output=True, text=True)
        return name, r
    failed = []
    with cf.ThreadPoolExecutor(max_workers=max(1, min(8, os.cpu_count() or 1))) as ex:
        for name, r in ex.map(run, jobs):
            if r.returncode != 0:
                failed.append(name)
                sys.stderr.write(f"--- {name}\n{r.stdout}{r.stderr}")
            elif verbose and (r.stdout or r.stderr):
                sys.stderr.write(r.stdout + r.stderr)
    if failed:
        raise RuntimeError("nvcc failed for: " + ", ".join(failed))
    objs = [os.path.join(OBJ, s[:-3] + ".o") for s in sources()]
    if force or jobs or _newer(LIB, objs):
        cmd = [NVCC, "-ccbin", HOST_CXX] + ARCH + ["-shared", "-o", LIB] + objs
        subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--verbose", action="store_true")
    ap.add_argument("--ptxas-v", action="store_true", help="print register / spill usage")
    a = ap.parse_args()
    print(build(a.force, a.verbose or a.ptxas_v, ["-Xptxas", "-v"] if a.ptxas_v else []))

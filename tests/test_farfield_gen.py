"""The generated far-field recurrences (bit_b200/csrc/gen_farfield.py), run in FP64 on the
CPU: the scaled forms the kernels use (coefficients times R^(|v|+1), moments
normalised by h^|v|, shells folded in with (h/R)^n / R) are the same function as the
literal form of the reference's recurrence, so the two agree to rounding for every
nterms and both kernels.  Also pins the per-pair flop counts behind the bench's roofline.
No GPU."""
import importlib.util
import math
import os
import re

import numpy as np
import pytest

from conftest import ROOT

# FP64 agreement of the two forms: measured at most 1.2e-13 over 2,400 random cases; a
# change of 7e-8 in one generated constant already moves the result by 1.3e-12
TOL = 5e-13


def gen():
    spec = importlib.util.spec_from_file_location(
        "gen_farfield", os.path.join(ROOT, "bit_b200", "csrc", "gen_farfield.py"))
    g = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(g)
    return g


def compile_lines(lines, args):
    """The generator's C++ statements as a Python function of `args` (FP64)."""
    body = []
    for ln in lines:
        ln = ln.strip().rstrip(";")
        if ln.startswith("return "):
            body.append(ln)
            continue
        ln = re.sub(r"^(const\s+)?(V4<T>|T)\s+", "", ln)
        ln = re.sub(r"T\(([^()]*)\)", r"(\1)", ln)
        ln = re.sub(r"ld4\(M, (\d+)\)", r"M[4 * \1:4 * \1 + 4]", ln)
        ln = re.sub(r"(mv\d+)\.([xyzw])", lambda m: f"{m.group(1)}[{'xyzw'.index(m.group(2))}]", ln)
        for part in re.split(r", (?=\w+(?: = |$))", ln):
            if "=" in part:
                body.append(part)
    src = f"def f({', '.join(args)}):\n" + "\n".join("    " + b for b in body)
    env = {"fma_t": lambda a, b, c: a * b + c, "rsqrt_t": lambda x: 1.0 / math.sqrt(x),
           "sqrt_t": math.sqrt, "exp_t": math.exp}
    exec(src, env)
    return env["f"]


def shell_degrees(g, nt):
    return np.array([sum(v) for v in g.shells(nt - 1)])


@pytest.mark.parametrize("nt", [2, 3, 5, 7, 9, 10])
def test_scaled_recurrences_equal_the_literal_ones(nt):
    g = gen()
    lit_c = compile_lines(g.gen_coulomb(nt), ["dx", "dy", "dz", "rs", "M"])
    sc_c = compile_lines(g.gen_coulomb_scaled(nt), ["dx", "dy", "dz", "rs", "h", "M"])
    sp_c = compile_lines(g.gen_coulomb_scaled(nt, hoisted=False), ["dx", "dy", "dz", "rs", "h", "M"])
    lit_s = compile_lines(g.gen_screened(nt), ["dx", "dy", "dz", "dist2", "kappa", "M"])
    sc_s = compile_lines(g.gen_screened_scaled(nt), ["dx", "dy", "dz", "dist2", "kappa", "h", "M"])
    sp_s = compile_lines(g.gen_screened_scaled_plain(nt), ["dx", "dy", "dz", "dist2", "kappa", "h", "M"])
    deg = shell_degrees(g, nt)
    rng = np.random.default_rng(nt)
    for _ in range(20):
        d = rng.uniform(-1.0, 1.0, 3)
        r2 = float(d @ d)
        h = 2.0 ** int(rng.integers(-6, 0))  # a power of two above the cluster radius
        # moments in shell order of a cluster of radius < h, and their normalised copy
        M = rng.uniform(-1.0, 1.0, len(deg)) * (0.9 * h) ** deg
        Mn = M / h ** deg
        pad = lambda a: np.concatenate([a, np.zeros((-len(a)) % 4)])
        M, Mn = pad(M), pad(Mn)
        for reg in (0.0, 1e-4):
            a, b = lit_c(*d, r2 + reg, M), sc_c(*d, r2 + reg, h, Mn)
            assert abs(a - b) <= TOL * max(abs(a), 1e-300), (nt, a, b)
            b = sp_c(*d, r2 + reg, h, Mn)
            assert abs(a - b) <= TOL * max(abs(a), 1e-300), (nt, a, b)
        for kappa in (0.5, 3.0):
            a, b = lit_s(*d, r2, kappa, M), sc_s(*d, r2, kappa, h, Mn)
            assert abs(a - b) <= TOL * max(abs(a), 1e-300), (nt, kappa, a, b)
            b = sp_s(*d, r2, kappa, h, Mn)
            assert abs(a - b) <= TOL * max(abs(a), 1e-300), (nt, kappa, a, b)


def test_flop_counts_behind_the_roofline():
    """bench.py's roofline counts the reference recurrence's flops per (target, cluster)
    pair at p = 8 (nterms 9); the scaled forms do fewer."""
    g = gen()
    assert g.flops_per_pair(9)["coulomb"] == 1459
    assert g.flops_per_pair(9)["screened"] == 2414
    assert g.count_flops(g.gen_coulomb_scaled(9)) < g.count_flops(g.gen_coulomb_scaled(9, False)) < 1459
    assert g.count_flops(g.gen_screened_scaled(9)) < g.count_flops(g.gen_screened_scaled_plain(9)) < 2414


def test_shell_positions_of_the_tma_moment_blocks():
    """The moment reduction writes each node's moments into a shell-order block by the
    closed form of moments.cu's canon_shell_pos: degree d, then i and j descending, i.e.
    C(d + 2, 3) + (d - i)(d - i + 1) / 2 + (d - i - j).  It must be the inverse of the
    generator's shell order (what the far-field kernels consume), for every nterms, and
    the blocks are padded to a multiple of 4 (16-byte TMA copies of FP32 moments)."""
    g = gen()

    def pos(t, nt):
        i = j = 0
        while t >= (nt - i) * (nt - i + 1) // 2:
            t -= (nt - i) * (nt - i + 1) // 2
            i += 1
        while t >= nt - i - j:
            t -= nt - i - j
            j += 1
        d = i + j + t
        return d * (d + 1) * (d + 2) // 6 + (d - i) * (d - i + 1) // 2 + (d - i - j)

    for nt in range(1, 11):
        canon = g.moment_index(nt)
        for k, v in enumerate(g.shells(nt - 1)):
            assert pos(canon[v], nt) == k
        assert g.padded(len(canon)) % 4 == 0 and g.padded(len(canon)) - len(canon) < 4

"""Derive the coefficients of exp2_fma (near.cu): the minimax polynomial of degree 5 for
2^f on [-1/2, 1/2] in relative error, by the Remez exchange algorithm (E. Remez, 1934;
see e.g. J.-M. Muller, Elementary Functions, ch. 3), then rounded to float32.

    python remez_exp2.py       # prints the coefficients as C hex-float literals and the
                               # relative error of their float32 Horner evaluation

Not run by the build; the printed literals are the ones written in near.cu.
"""
import numpy as np
from mpmath import lu_solve, matrix, mp, mpf, power

mp.dps = 40


def remez(deg, a=mpf(-0.5), b=mpf(0.5), iters=30, grid=4000):
    f = lambda x: power(2, x)
    n = deg + 2
    xs = [(a + b) / 2 + (b - a) / 2 * mp.cos(mp.pi * (n - 1 - i) / (n - 1)) for i in range(n)]
    c, E = None, None
    for _ in range(iters):
        # p(x_i) - f(x_i) = (-1)^i E f(x_i): equioscillating relative error on the reference set
        A, rhs = matrix(n, n), matrix(n, 1)
        for i, x in enumerate(xs):
            for j in range(deg + 1):
                A[i, j] = x ** j
            A[i, deg + 1] = (-1) ** i * f(x)
            rhs[i] = f(x)
        sol = lu_solve(A, rhs)
        c, E = [sol[j] for j in range(deg + 1)], sol[deg + 1]
        err = lambda x: (sum(c[j] * x ** j for j in range(deg + 1)) - f(x)) / f(x)
        pts = [a + (b - a) * k / grid for k in range(grid + 1)]
        vals = [err(x) for x in pts]
        ext = [a] + [pts[k] for k in range(1, grid) if (vals[k] - vals[k - 1]) * (vals[k + 1] - vals[k]) < 0] + [b]
        if len(ext) == n:
            xs = ext
    return c, E


def horner32(c32, xs):
    """Float32 Horner evaluation with fused multiply-adds (product exact in float64)."""
    p = np.full(xs.shape, float(c32[-1]))
    for v in reversed(c32[:-1]):
        p = (p * xs.astype(np.float64) + float(v)).astype(np.float32).astype(np.float64)
    return p


if __name__ == "__main__":
    c, E = remez(5)
    c32 = [np.float32(float(v)) for v in c]
    print("minimax relative error", mp.nstr(E, 5))
    for k, v in enumerate(c32):
        print(f"c{k} = {float.hex(float(v))}f")
    xs = np.linspace(-0.5, 0.5, 200001, dtype=np.float32)
    print("float32 Horner max relative error", np.max(np.abs(horner32(c32, xs) / np.exp2(xs.astype(np.float64)) - 1)))

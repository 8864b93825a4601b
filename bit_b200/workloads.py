"""Seeded synthetic inputs with the shapes and distributions of the treecode workloads.

No dataset is involved: every workload is generated from a seed.

uniform_cube      N particles uniform in [-1,1]^3, charges uniform in [-1,1]
clustered_blobs   80% in 8 isotropic Gaussian blobs (centres U[-1,1]^3, sigma 0.1),
                  20% uniform in [-1,1]^3, charges uniform in [-1,1]
icosphere         unit icosahedron subdivided L times: flat-triangle centroids, areas, mean
                  edge length (boundary-integral quadrature nodes)
sh_rhs            sum of real spherical harmonics of degree <= lmax with N(0,1) coefficients
batched_systems   many independent systems with log-uniform sizes and mixed kernels
"""
import math

import numpy as np


def uniform_cube(n, seed=1):
    rng = np.random.default_rng(seed)
    p = rng.uniform(-1.0, 1.0, (n, 3))
    q = rng.uniform(-1.0, 1.0, n)
    return p[:, 0].copy(), p[:, 1].copy(), p[:, 2].copy(), q


def clustered_blobs(n, seed=1, nblobs=8, sigma=0.1, frac=0.8):
    rng = np.random.default_rng(seed)
    nb = int(round(frac * n))
    centres = rng.uniform(-1.0, 1.0, (nblobs, 3))
    which = rng.integers(0, nblobs, nb)
    pb = centres[which] + sigma * rng.standard_normal((nb, 3))
    pu = rng.uniform(-1.0, 1.0, (n - nb, 3))
    p = np.concatenate([pb, pu])
    p = p[rng.permutation(n)]
    q = rng.uniform(-1.0, 1.0, n)
    return p[:, 0].copy(), p[:, 1].copy(), p[:, 2].copy(), q


def icosphere(level):
    """Centroids, areas and mean edge length of a unit icosphere with 20*4^level faces."""
    t = (1.0 + math.sqrt(5.0)) / 2.0
    v = np.array([[-1, t, 0], [1, t, 0], [-1, -t, 0], [1, -t, 0],
                  [0, -1, t], [0, 1, t], [0, -1, -t], [0, 1, -t],
                  [t, 0, -1], [t, 0, 1], [-t, 0, -1], [-t, 0, 1]], dtype=np.float64)
    v /= np.linalg.norm(v, axis=1, keepdims=True)
    f = np.array([[0, 11, 5], [0, 5, 1], [0, 1, 7], [0, 7, 10], [0, 10, 11],
                  [1, 5, 9], [5, 11, 4], [11, 10, 2], [10, 7, 6], [7, 1, 8],
                  [3, 9, 4], [3, 4, 2], [3, 2, 6], [3, 6, 8], [3, 8, 9],
                  [4, 9, 5], [2, 4, 11], [6, 2, 10], [8, 6, 7], [9, 8, 1]], dtype=np.int64)
    verts = [tuple(r) for r in v]
    for _ in range(level):
        cache = {}
        vl = verts

        def mid(a, b):
            key = (a, b) if a < b else (b, a)
            if key not in cache:
                m = (np.array(vl[a]) + np.array(vl[b])) * 0.5
                m /= np.linalg.norm(m)
                vl.append(tuple(m))
                cache[key] = len(vl) - 1
            return cache[key]

        nf = []
        for a, b, c in f:
            ab, bc, ca = mid(a, b), mid(b, c), mid(c, a)
            nf += [[a, ab, ca], [b, bc, ab], [c, ca, bc], [ab, bc, ca]]
        f = np.array(nf, dtype=np.int64)
        verts = vl
    V = np.array(verts)
    A, B, Cc = V[f[:, 0]], V[f[:, 1]], V[f[:, 2]]
    cen = (A + B + Cc) / 3.0
    area = 0.5 * np.linalg.norm(np.cross(B - A, Cc - A), axis=1)
    edges = np.concatenate([np.linalg.norm(B - A, axis=1), np.linalg.norm(Cc - B, axis=1),
                            np.linalg.norm(A - Cc, axis=1)])
    return cen, area, float(edges.mean())


def _assoc_legendre(lmax, x):
    """P_l^m(x) (with Condon-Shortley phase) for 0 <= m <= l <= lmax; dict keyed (l, m)."""
    P = {}
    s = np.sqrt(np.maximum(0.0, 1.0 - x * x))
    P[(0, 0)] = np.ones_like(x)
    for m in range(1, lmax + 1):
        P[(m, m)] = -(2 * m - 1) * s * P[(m - 1, m - 1)]
    for m in range(0, lmax):
        P[(m + 1, m)] = (2 * m + 1) * x * P[(m, m)]
    for m in range(0, lmax + 1):
        for l in range(m + 2, lmax + 1):
            P[(l, m)] = ((2 * l - 1) * x * P[(l - 1, m)] - (l + m - 1) * P[(l - 2, m)]) / (l - m)
    return P


def sh_rhs(points, lmax=8, seed=1):
    """f = sum_{l<=lmax, |m|<=l} c_lm Y_lm(direction) with real orthonormal Y and c ~ N(0,1)."""
    rng = np.random.default_rng(seed)
    d = points / np.linalg.norm(points, axis=1, keepdims=True)
    ct = np.clip(d[:, 2], -1.0, 1.0)
    phi = np.arctan2(d[:, 1], d[:, 0])
    P = _assoc_legendre(lmax, ct)
    f = np.zeros(len(points))
    for l in range(lmax + 1):
        for m in range(-l, l + 1):
            am = abs(m)
            norm = math.sqrt((2 * l + 1) / (4 * math.pi) * math.factorial(l - am) / math.factorial(l + am))
            if m == 0:
                y = norm * P[(l, 0)]
            elif m > 0:
                y = math.sqrt(2.0) * norm * P[(l, am)] * np.cos(am * phi)
            else:
                y = math.sqrt(2.0) * norm * P[(l, am)] * np.sin(am * phi)
            f += rng.standard_normal() * y
    return f


def batched_systems(count=2048, nmin=1000, nmax=100000, seed=1):
    """Independent systems: N log-uniform, each uniform in its own unit cube, q ~ U[-1,1];
    half regularised Coulomb (delta = 0.01), half screened with kappa ~ U[0.5, 4];
    p drawn from {4, 6, 8} (nterms = p + 1)."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(count):
        n = int(round(math.exp(rng.uniform(math.log(nmin), math.log(nmax)))))
        p = rng.uniform(0.0, 1.0, (n, 3))
        q = rng.uniform(-1.0, 1.0, n)
        kern = 0 if i % 2 == 0 else 1
        kappa = 0.0 if kern == 0 else float(rng.uniform(0.5, 4.0))
        nterms = int(rng.choice([4, 6, 8])) + 1
        out.append(dict(x=p[:, 0].copy(), y=p[:, 1].copy(), z=p[:, 2].copy(), q=q,
                        kernel=kern, kappa=kappa, del_=1e-4 if kern == 0 else 0.0,
                        nterms=nterms))
    return out


def sample_targets(n, k, seed=1):
    rng = np.random.default_rng(seed)
    k = min(k, n)
    return np.sort(rng.choice(n, k, replace=False)).astype(np.int32)


def rel_l2(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))

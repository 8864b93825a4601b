"""TEST INFRASTRUCTURE -- ctypes binding of the unmodified reference treecode.

The libraries under oracle/_ref/ are built by ``make -C oracle ref`` from the
reference's own src/tree3d.cpp and src/solver.h (one per compile-time DEL,
src/problem.h:12).  Imported only by tests/ and bench.py's reference arm; every
caller must tolerate ``available() == False`` (no reference build on this machine).
"""
import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
# (DEL, KERNEL_ORDER) of every library the recipe builds
TAGS = {(0.01, 0): "d1e-2", (1e-4, 0): "d1e-4", (2.5e-5, 0): "d2.5e-5",
        (0.01, 1): "d1e-2k1", (0.01, 2): "d1e-2k2"}
# The reference's src/ directory, for building only (the libraries travel prebuilt).
REF_SRC = os.environ.get("BIT_REFERENCE_SRC")

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)
_libs = {}


def path(del_, korder=0):
    return os.path.join(HERE, "_ref", f"libref_{TAGS[(del_, korder)]}.so")


def available(del_=0.01, korder=0):
    return (del_, korder) in TAGS and os.path.exists(path(del_, korder))


def build(src=None):
    """Build the reference libraries from the reference's src/ directory (`src`, else
    BIT_REFERENCE_SRC); a no-op when neither names one that holds tree3d.cpp."""
    src = src or REF_SRC
    if src and os.path.exists(os.path.join(src, "tree3d.cpp")):
        subprocess.run(["make", "-s", "-C", HERE, "ref", f"REF_SRC={src}"], check=True)


def build_dropin(src=None):
    """Compile the reference's own tests/treecode.cpp, treecode_mp.cpp and directsum_mp.cpp
    unchanged against the drop-in (oracle/_ref/dropin/); needs libtree3d_b200.so built."""
    src = src or REF_SRC
    if src and os.path.exists(os.path.join(src, "tree3d.cpp")):
        subprocess.run(["make", "-s", "-C", HERE, "dropin", f"REF_SRC={src}"], check=True)


DROPIN_TESTS = ("treecode", "treecode_mp", "directsum_mp")


def dropin_path(name):
    return os.path.join(HERE, "_ref", "dropin", name)


def lib(del_=0.01, korder=0):
    key = (del_, korder)
    if key not in _libs:
        L = C.CDLL(path(del_, korder))
        L.ref_del.restype = C.c_double
        L.ref_boxparticles.argtypes = [C.c_int] + [C.c_double] * 4 + [_dp] * 5
        L.ref_tree_build.restype = C.c_void_p
        L.ref_tree_build.argtypes = [C.c_int] + [_dp] * 5 + [C.c_int] * 3
        L.ref_tree_numtree.restype = C.c_int
        L.ref_tree_numtree.argtypes = [C.c_void_p]
        L.ref_tree_set_charges.argtypes = [C.c_void_p, _dp]
        L.ref_tree_moments.argtypes = [C.c_void_p]
        L.ref_tree_export.argtypes = [C.c_void_p, _ip, _ip, _dp, _ip]
        L.ref_tree_node_moments.argtypes = [C.c_void_p, C.c_int, _dp]
        L.ref_eval_potential.argtypes = [C.c_void_p, C.c_double, C.c_int, _ip, _dp, _dp, _dp,
                                         _dp, C.c_int]
        L.ref_eval_screened.argtypes = [C.c_void_p, C.c_double, C.c_double, C.c_int, _ip, _dp,
                                        _dp, _dp, _dp, C.c_int]
        L.ref_eval_force.argtypes = [C.c_void_p, C.c_double, C.c_int, _ip, _dp, _dp, _dp, _dp,
                                     _dp, _dp, C.c_int]
        L.ref_tree_free.argtypes = [C.c_void_p]
        L.ref_ds_force_reg.argtypes = [C.c_int] + [_dp] * 4 + [C.c_int, _ip] + [_dp] * 3 + [C.c_int]
        L.ref_ds_screened_pot.argtypes = [C.c_int] + [_dp] * 4 + [C.c_double, C.c_int, _ip, _dp,
                                                                  C.c_int]
        L.ref_eval_grad_kernel.argtypes = [C.c_double] * 4 + [C.c_int, _dp]
        L.ref_gmres_dense.restype = C.c_int
        L.ref_gmres_dense.argtypes = [C.c_int, _dp, _dp, _dp]
        L.ref_output_potential.argtypes = [C.c_int] + [_dp] * 4 + [C.c_char_p]
        L.ref_eval_screened_field.argtypes = [C.c_void_p, C.c_double, C.c_double, C.c_int, _ip,
                                              _dp, _dp, _dp, _dp, _dp, _dp, C.c_int]
        L.ref_ds_force_noreg.argtypes = [C.c_int] + [_dp] * 4 + [C.c_int, _ip] + [_dp] * 3 + [C.c_int]
        L.ref_setboundaries.restype = C.c_int
        L.ref_setboundaries.argtypes = [C.c_int] * 3 + [C.c_double] * 3 + [_dp]
        L.ref_panelconstantsreal.argtypes = [C.c_int] * 3 + [C.c_double] * 3 + [_dp]
        _libs[key] = L
    return _libs[key]


def _d(a):
    return a.ctypes.data_as(_dp) if a is not None else None


def _i(a):
    return a.ctypes.data_as(_ip) if a is not None else None


def boxparticles(n, dlength=1.0, dheight=1.0, ddepth=1.0, density=1.0):
    """The reference tests' fixture (src/tree3d.cpp:1698-1740, srand(100))."""
    out = [np.zeros(n) for _ in range(5)]
    lib(0.01).ref_boxparticles(n, dlength, dheight, ddepth, density, *[_d(a) for a in out])
    return out  # x, y, z, tot_charge, weight


class RefTree:
    """treemake + treemoments of the reference on caller particles."""

    def __init__(self, x, y, z, q, nterms, maxmemb, del_=0.01, w=None, cap=None, korder=0):
        self.L = lib(del_, korder)
        self.del_ = del_
        self.x, self.y, self.z, self.q = [np.ascontiguousarray(a, dtype=np.float64) for a in (x, y, z, q)]
        self.w = None if w is None else np.ascontiguousarray(w, dtype=np.float64)
        self.n = len(self.x)
        self.nterms = nterms
        cap = cap or (64 * (self.n // max(maxmemb, 1) + 2) + 64)
        self.h = self.L.ref_tree_build(self.n, _d(self.x), _d(self.y), _d(self.z), _d(self.q),
                                       _d(self.w), nterms, maxmemb, cap)
        self.numtree = self.L.ref_tree_numtree(self.h)
        assert self.numtree <= cap

    def close(self):
        if self.h:
            self.L.ref_tree_free(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def export(self):
        nt = self.numtree
        nm = np.zeros(nt, np.int32)
        ch = np.zeros(nt * 8, np.int32)
        f = np.zeros(nt * 13)
        self.L.ref_tree_export(self.h, _i(nm), _i(ch), _d(f), None)
        mem = np.zeros(int(nm.sum()), np.int32)
        self.L.ref_tree_export(self.h, _i(nm), _i(ch), _d(f), _i(mem))
        return nm, ch.reshape(nt, 8), f.reshape(nt, 13), mem

    def moments(self):
        self.L.ref_tree_moments(self.h)

    def set_charges(self, q):
        self.q = np.ascontiguousarray(q, dtype=np.float64)
        self.L.ref_tree_set_charges(self.h, _d(self.q))

    def node_moments(self, ind):
        n = self.nterms
        out = np.zeros(n * n * n)
        self.L.ref_tree_node_moments(self.h, ind, _d(out))
        return out.reshape(n, n, n)

    def _targets(self, targets, points):
        if points is not None:
            pts = np.ascontiguousarray(points, dtype=np.float64)
            p = np.full(len(pts), -1, np.int32)
            return p, [np.ascontiguousarray(pts[:, a]) for a in range(3)]
        t = np.arange(self.n, dtype=np.int32) if targets is None else np.ascontiguousarray(targets, dtype=np.int32)
        return t, [np.zeros(len(t))] * 3

    def potential(self, acc, targets=None, points=None, nthreads=0):
        p, (tx, ty, tz) = self._targets(targets, points)
        out = np.zeros(len(p))
        self.L.ref_eval_potential(self.h, acc, len(p), _i(p), _d(tx), _d(ty), _d(tz), _d(out),
                                  nthreads)
        return out

    def screened(self, kappa, acc, targets=None, points=None, nthreads=0):
        p, (tx, ty, tz) = self._targets(targets, points)
        out = np.zeros(len(p))
        self.L.ref_eval_screened(self.h, kappa, acc, len(p), _i(p), _d(tx), _d(ty), _d(tz),
                                 _d(out), nthreads)
        return out

    def force(self, acc, targets=None, points=None, nthreads=0):
        p, (tx, ty, tz) = self._targets(targets, points)
        fx, fy, fz = np.zeros(len(p)), np.zeros(len(p)), np.zeros(len(p))
        self.L.ref_eval_force(self.h, acc, len(p), _i(p), _d(tx), _d(ty), _d(tz), _d(fx),
                              _d(fy), _d(fz), nthreads)
        return fx, fy, fz


    def screened_field(self, kappa, acc, targets=None, points=None, nthreads=0):
        """shielded_treeforce: the reference's screened 2-D field."""
        p, (tx, ty, tz) = self._targets(targets, points)
        fx, fy, fz = np.zeros(len(p)), np.zeros(len(p)), np.zeros(len(p))
        self.L.ref_eval_screened_field(self.h, kappa, acc, len(p), _i(p), _d(tx), _d(ty), _d(tz),
                                       _d(fx), _d(fy), _d(fz), nthreads)
        return fx, fy, fz


def ds_force_noreg(x, y, z, q, targets, nthreads=0):
    x, y, z, q = [np.ascontiguousarray(a, dtype=np.float64) for a in (x, y, z, q)]
    t = np.ascontiguousarray(targets, dtype=np.int32)
    fx, fy, fz = np.zeros(len(t)), np.zeros(len(t)), np.zeros(len(t))
    lib(0.01).ref_ds_force_noreg(len(x), _d(x), _d(y), _d(z), _d(q), len(t), _i(t), _d(fx),
                                 _d(fy), _d(fz), nthreads)
    return fx, fy, fz


def ds_force_reg(x, y, z, q, targets, del_=0.01, nthreads=0, korder=0):
    x, y, z, q = [np.ascontiguousarray(a, dtype=np.float64) for a in (x, y, z, q)]
    t = np.ascontiguousarray(targets, dtype=np.int32)
    fx, fy, fz = np.zeros(len(t)), np.zeros(len(t)), np.zeros(len(t))
    lib(del_, korder).ref_ds_force_reg(len(x), _d(x), _d(y), _d(z), _d(q), len(t), _i(t), _d(fx),
                               _d(fy), _d(fz), nthreads)
    return fx, fy, fz


def ds_screened_pot(x, y, z, q, kappa, targets, nthreads=0):
    x, y, z, q = [np.ascontiguousarray(a, dtype=np.float64) for a in (x, y, z, q)]
    t = np.ascontiguousarray(targets, dtype=np.int32)
    out = np.zeros(len(t))
    lib(0.01).ref_ds_screened_pot(len(x), _d(x), _d(y), _d(z), _d(q), kappa, len(t), _i(t),
                                  _d(out), nthreads)
    return out


def grad_kernel(dx, dy, dz, rs, reg, del_=0.01):
    out = np.zeros(3)
    lib(del_).ref_eval_grad_kernel(dx, dy, dz, rs, int(reg), _d(out))
    return out


def gmres_dense(A, b, x0=None):
    """solver::gmres on a dense matrix: (x, Arnoldi steps taken)."""
    A = np.ascontiguousarray(A, dtype=np.float64)
    b = np.ascontiguousarray(b, dtype=np.float64)
    x = np.ones(len(b)) if x0 is None else np.ascontiguousarray(x0, dtype=np.float64).copy()
    steps = lib(0.01).ref_gmres_dense(len(b), _d(A), _d(b), _d(x))
    return x, steps


def setboundaries(xp, yp, zp, dl, dh, dd, del_=0.01):
    """The reference's box panels: (numpan, 17) array, columns as in ref_setboundaries."""
    n = 2 * (xp * yp + zp * yp + xp * zp)
    out = np.zeros(17 * n)
    lib(del_).ref_setboundaries(xp, yp, zp, dl, dh, dd, _d(out))
    return out.reshape(n, 17)


def panelconstantsreal(xp, yp, zp, dl, dh, dd, del_=0.01):
    n = 2 * (xp * yp + zp * yp + xp * zp)
    A = np.zeros(n * n)
    lib(del_).ref_panelconstantsreal(xp, yp, zp, dl, dh, dd, _d(A))
    return A.reshape(n, n)


def output_potential(x, y, z, pot, filename, del_=0.01):
    x, y, z, pot = [np.ascontiguousarray(a, dtype=np.float64) for a in (x, y, z, pot)]
    lib(del_).ref_output_potential(len(x), _d(x), _d(y), _d(z), _d(pot), filename.encode())

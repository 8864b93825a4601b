"""TEST INFRASTRUCTURE -- ctypes binding of the C restatement (oracle/bit_oracle.c).

Imported only by tests/, __graft_entry__.smoke() and bench.py as the checker / CPU
baseline.  Function names follow the reference entry points they restate:
``tree_build`` ~ treemake (src/tree3d.cpp:1345), ``moments`` ~ treemoments (:2631),
``evaluate`` ~ treepotential / shielded_treepot (:4679 / :3448), ``evaluate_force`` ~
treeforce (:851), ``direct`` ~ the direct sums (:298, :1966), ``gmres_dense_ref`` ~
solver::gmres (src/solver.h:157).
"""
import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "lib", "liborc.so")

COULOMB, SCREENED, SCREENED_REG = 0, 1, 2
MODE_REFERENCE, MODE_CONSISTENT = 0, 1
# intG of the reference's screened self term (src/tree3d.cpp:3585)
REF_INTG = -0.0000483811229725

_lib = None


def build():
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            build()
        _lib = C.CDLL(LIB)
        _declare(_lib)
    return _lib


_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)
_lp = C.POINTER(C.c_longlong)


class TreeView(C.Structure):
    _fields_ = [("n", C.c_int), ("numtree", C.c_int), ("nterms", C.c_int),
                ("x", _dp), ("y", _dp), ("z", _dp), ("q", _dp), ("w", _dp),
                ("nummemb", _ip), ("start", _ip), ("children", _ip), ("perm", _ip),
                ("fields", _dp), ("mom", _dp)]


class Params(C.Structure):
    _fields_ = [("kernel", C.c_int), ("mode", C.c_int), ("del_", C.c_double),
                ("mac_del", C.c_double), ("kappa", C.c_double), ("acc", C.c_double),
                ("intg", C.c_double)]


def _declare(L):
    L.orc_tree_build.restype = C.c_int
    L.orc_tree_build.argtypes = [C.c_int, _dp, _dp, _dp, C.c_int, C.c_int, _ip, _ip, _ip,
                                 _ip, _ip, _dp, _ip]
    L.orc_moments.argtypes = [C.POINTER(TreeView), _dp]
    L.orc_eval.argtypes = [C.POINTER(TreeView), C.POINTER(Params), C.c_int, _ip, _dp, _dp,
                           _dp, _dp, C.c_int]
    L.orc_eval_force.argtypes = [C.POINTER(TreeView), C.c_double, C.c_double, C.c_int,
                                 C.c_int, _ip, _dp, _dp, _dp, _dp, _dp, _dp, C.c_int]
    L.orc_count.argtypes = [C.POINTER(TreeView), C.POINTER(Params), C.c_int, _ip, _dp, _dp,
                            _dp, _lp, _lp, _lp, C.c_int]
    L.orc_target_lists.restype = C.c_int
    L.orc_target_lists.argtypes = [C.POINTER(TreeView), C.POINTER(Params), C.c_int,
                                   C.c_double, C.c_double, C.c_double, _ip, _ip, C.c_int]
    L.orc_direct.argtypes = [C.c_int, _dp, _dp, _dp, _dp, C.POINTER(Params), C.c_int, _ip,
                             _dp, _dp, _dp, _dp, C.c_int]
    L.orc_direct_force.argtypes = [C.c_int, _dp, _dp, _dp, _dp, C.c_double, C.c_int,
                                   C.c_int, _ip, _dp, _dp, _dp, C.c_int]
    L.orc_gmres_dense_ref.restype = C.c_int
    L.orc_gmres_dense_ref.argtypes = [C.c_int, _dp, _dp, _dp]
    L.orc_gmres_treecode.restype = C.c_int
    L.orc_gmres_treecode.argtypes = [C.POINTER(TreeView), _dp, C.POINTER(Params), C.c_double,
                                     _dp, _dp, _dp, C.c_int, C.c_double, C.c_int, C.c_int,
                                     _ip, _dp]
    L.orc_moment_index.restype = C.c_int
    L.orc_moment_index.argtypes = [C.c_int] * 4
    L.orc_num_terms.restype = C.c_int
    L.orc_num_terms.argtypes = [C.c_int]
    L.orc_aspect_limit.restype = C.c_double


def _d(a):
    return a.ctypes.data_as(_dp) if a is not None else None


def _i(a):
    return a.ctypes.data_as(_ip) if a is not None else None


def num_terms(nterms):
    return nterms * (nterms + 1) * (nterms + 2) // 6


def moment_order(nterms):
    """(i, j, k) of each packed moment slot: i outermost, then j, then k."""
    out = []
    for i in range(nterms):
        for j in range(nterms - i):
            for k in range(nterms - i - j):
                out.append((i, j, k))
    return out


def params(kernel=COULOMB, mode=MODE_CONSISTENT, del_=0.0, mac_del=0.0, kappa=0.0, acc=0.5,
           intg=REF_INTG):
    return Params(kernel, mode, del_, mac_del, kappa, acc, intg)


class Tree:
    """Flat tree from ``orc_tree_build``: node i owns perm[start[i]:start[i]+nummemb[i]]."""

    def __init__(self, x, y, z, maxmemb, cap=None):
        L = lib()
        self.x = np.ascontiguousarray(x, dtype=np.float64)
        self.y = np.ascontiguousarray(y, dtype=np.float64)
        self.z = np.ascontiguousarray(z, dtype=np.float64)
        n = self.n = len(self.x)
        self.maxmemb = maxmemb
        cap = cap or (64 * (n // max(maxmemb, 1) + 2) + 64)
        self.nummemb = np.zeros(cap, np.int32)
        self.start = np.zeros(cap, np.int32)
        self.children = np.full(cap * 8, -1, np.int32)
        self.level = np.zeros(cap, np.int32)
        self.parent = np.zeros(cap, np.int32)
        self.fields = np.zeros(cap * 13, np.float64)
        self.perm = np.zeros(n, np.int32)
        rc = L.orc_tree_build(n, _d(self.x), _d(self.y), _d(self.z), maxmemb, cap,
                              _i(self.nummemb), _i(self.start), _i(self.children),
                              _i(self.level), _i(self.parent), _d(self.fields), _i(self.perm))
        if rc < 0:
            raise RuntimeError(f"orc_tree_build failed: {rc}")
        nt = self.numtree = rc
        self.nummemb = self.nummemb[:nt].copy()
        self.start = self.start[:nt].copy()
        self.children = self.children[:nt * 8].reshape(nt, 8).copy()
        self.level = self.level[:nt].copy()
        self.parent = self.parent[:nt].copy()
        self.fields = self.fields[:nt * 13].reshape(nt, 13).copy()
        self.q = None
        self.w = None
        self.mom = None
        self.nterms = 0

    def members(self, i):
        s = self.start[i]
        return np.sort(self.perm[s:s + self.nummemb[i]])

    def is_leaf(self, i):
        return bool((self.children[i] < 0).all())

    def view(self):
        v = TreeView()
        v.n, v.numtree, v.nterms = self.n, self.numtree, self.nterms
        v.x, v.y, v.z = _d(self.x), _d(self.y), _d(self.z)
        v.q = _d(self.q)
        v.w = _d(self.w)
        v.nummemb, v.start, v.perm = _i(self.nummemb), _i(self.start), _i(self.perm)
        self._ch = np.ascontiguousarray(self.children.reshape(-1))
        self._f = np.ascontiguousarray(self.fields.reshape(-1))
        v.children, v.fields = _i(self._ch), _d(self._f)
        v.mom = _d(self.mom)
        return v

    def compute_moments(self, q, nterms, w=None):
        self.q = np.ascontiguousarray(q, dtype=np.float64)
        self.w = None if w is None else np.ascontiguousarray(w, dtype=np.float64)
        self.nterms = nterms
        self.mom = np.zeros(self.numtree * num_terms(nterms), np.float64)
        v = self.view()
        lib().orc_moments(C.byref(v), _d(self.mom))
        return self.mom.reshape(self.numtree, num_terms(nterms))

    def evaluate(self, prm, targets=None, points=None, nthreads=0):
        """Potential at particle targets (indices) or external points (m x 3)."""
        v = self.view()
        if points is not None:
            pts = np.ascontiguousarray(points, dtype=np.float64)
            m = len(pts)
            tx, ty, tz = [np.ascontiguousarray(pts[:, a]) for a in range(3)]
            out = np.zeros(m)
            lib().orc_eval(C.byref(v), C.byref(prm), m, None, _d(tx), _d(ty), _d(tz), _d(out),
                           nthreads)
            return out
        t = np.arange(self.n, dtype=np.int32) if targets is None else np.ascontiguousarray(targets, dtype=np.int32)
        out = np.zeros(len(t))
        lib().orc_eval(C.byref(v), C.byref(prm), len(t), _i(t), None, None, None, _d(out),
                       nthreads)
        return out

    def evaluate_force(self, del_, acc, targets=None, kernel_order=0, nthreads=0):
        v = self.view()
        t = np.arange(self.n, dtype=np.int32) if targets is None else np.ascontiguousarray(targets, dtype=np.int32)
        fx, fy, fz = np.zeros(len(t)), np.zeros(len(t)), np.zeros(len(t))
        lib().orc_eval_force(C.byref(v), del_, acc, kernel_order, len(t), _i(t), None, None,
                             None, _d(fx), _d(fy), _d(fz), nthreads)
        return fx, fy, fz

    def count(self, prm, targets=None, nthreads=0):
        v = self.view()
        t = np.arange(self.n, dtype=np.int32) if targets is None else np.ascontiguousarray(targets, dtype=np.int32)
        a, b, c = C.c_longlong(), C.c_longlong(), C.c_longlong()
        lib().orc_count(C.byref(v), C.byref(prm), len(t), _i(t), None, None, None, C.byref(a),
                        C.byref(b), C.byref(c), nthreads)
        return a.value, b.value, c.value

    def target_lists(self, prm, p, xyz=None, cap=4096):
        v = self.view()
        node = np.zeros(cap, np.int32)
        kind = np.zeros(cap, np.int32)
        if xyz is None:
            xyz = (self.x[p], self.y[p], self.z[p])
        n = lib().orc_target_lists(C.byref(v), C.byref(prm), p, *map(float, xyz), _i(node),
                                   _i(kind), cap)
        assert n <= cap
        return node[:n].copy(), kind[:n].copy()


def direct(x, y, z, q, prm, targets=None, points=None, nthreads=0):
    x, y, z, q = [np.ascontiguousarray(a, dtype=np.float64) for a in (x, y, z, q)]
    n = len(x)
    if points is not None:
        pts = np.ascontiguousarray(points, dtype=np.float64)
        tx, ty, tz = [np.ascontiguousarray(pts[:, a]) for a in range(3)]
        out = np.zeros(len(pts))
        lib().orc_direct(n, _d(x), _d(y), _d(z), _d(q), C.byref(prm), len(pts), None, _d(tx),
                         _d(ty), _d(tz), _d(out), nthreads)
        return out
    t = np.arange(n, dtype=np.int32) if targets is None else np.ascontiguousarray(targets, dtype=np.int32)
    out = np.zeros(len(t))
    lib().orc_direct(n, _d(x), _d(y), _d(z), _d(q), C.byref(prm), len(t), _i(t), None, None,
                     None, _d(out), nthreads)
    return out


def direct_force(x, y, z, q, del_, targets, kernel_order=0, nthreads=0):
    x, y, z, q = [np.ascontiguousarray(a, dtype=np.float64) for a in (x, y, z, q)]
    t = np.ascontiguousarray(targets, dtype=np.int32)
    fx, fy, fz = np.zeros(len(t)), np.zeros(len(t)), np.zeros(len(t))
    lib().orc_direct_force(len(x), _d(x), _d(y), _d(z), _d(q), del_, kernel_order, len(t),
                           _i(t), _d(fx), _d(fy), _d(fz), nthreads)
    return fx, fy, fz


def gmres_dense_ref(A, b, x0=None):
    A = np.ascontiguousarray(A, dtype=np.float64)
    b = np.ascontiguousarray(b, dtype=np.float64)
    x = np.ones(len(b)) if x0 is None else np.ascontiguousarray(x0, dtype=np.float64).copy()
    rc = lib().orc_gmres_dense_ref(len(b), _d(A), _d(b), _d(x))
    return x, rc


def gmres_treecode(tree, prm, diag, wts, b, restart=50, tol=1e-8, maxit=500, nthreads=0):
    """Restarted GMRES(m) on (diag*I + K) s = b, K the treecode with charges w*s."""
    b = np.ascontiguousarray(b, dtype=np.float64)
    x = np.zeros(len(b))
    wts = None if wts is None else np.ascontiguousarray(wts, dtype=np.float64)
    if tree.q is None:
        tree.q = np.zeros(tree.n)
    mom = np.zeros(tree.numtree * num_terms(tree.nterms))
    v = tree.view()
    it, rr = C.c_int(), C.c_double()
    rc = lib().orc_gmres_treecode(C.byref(v), _d(mom), C.byref(prm), diag, _d(wts), _d(b),
                                  _d(x), restart, tol, maxit, nthreads, C.byref(it), C.byref(rr))
    return x, it.value, rr.value, rc

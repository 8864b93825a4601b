"""bit_b200 -- B200-native treecode behind the C ABI of include/bit_b200.h.

Host-side mirror of the reference's treecode interface (ongbw/bit, src/tree3d.h):

    ctx  = bit_b200.Context()
    tree = ctx.treemake(x, y, z, maxmemb)          # treemake      src/tree3d.cpp:1345
    tree.treemoments(q, nterms, w=None)            # treemoments   src/tree3d.cpp:2631
    pot  = tree.treepotential(acc, del_)           # treepotential src/tree3d.cpp:4679
    pot  = tree.shielded_treepot(kappa, acc)       # shielded_treepot src/tree3d.cpp:3448
    fx, fy, fz = tree.treeforce(acc, del_)         # treeforce     src/tree3d.cpp:851
    tree.treeempty()                               # treeempty     src/tree3d.cpp:990

Every call goes through libbit_b200.so; there is no CPU fallback.  If the library is
missing, importing works but the first call raises ``BitError``.
"""
import ctypes as C
import os
import weakref

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "lib", "libbit_b200.so")

COULOMB, SCREENED, SCREENED_REG = 0, 1, 2
FP64, MIXED = 0, 1
REFERENCE, CONSISTENT = 0, 1
# intG of the reference's screened self term (src/tree3d.cpp:3585)
REF_INTG = -0.0000483811229725
NTERMS_MAX = 10

STATUS = {0: "ok", 1: "invalid argument", 2: "CUDA error", 3: "out of memory",
          4: "capacity exceeded", 5: "degenerate input", 6: "GMRES breakdown",
          7: "not converged", 8: "no CUDA device", 9: "HBM budget exceeded",
          10: "invalid call order"}


class BitError(RuntimeError):
    def __init__(self, status, msg=""):
        self.status = status
        super().__init__(f"{STATUS.get(status, status)}: {msg}")


class CtxOpts(C.Structure):
    _fields_ = [("device", C.c_int), ("stream", C.c_void_p), ("hbm_budget", C.c_size_t)]


class EvalParams(C.Structure):
    _fields_ = [("kernel", C.c_int), ("mode", C.c_int), ("precision", C.c_int),
                ("del_", C.c_double), ("mac_del", C.c_double), ("kappa", C.c_double),
                ("acc", C.c_double), ("intg", C.c_double)]


class Stats(C.Structure):
    _fields_ = [("t_build", C.c_double), ("t_moments", C.c_double), ("t_lists", C.c_double),
                ("t_far", C.c_double), ("t_near", C.c_double), ("t_total", C.c_double),
                ("far_pairs", C.c_longlong), ("near_pairs", C.c_longlong),
                ("far_entries", C.c_longlong), ("near_entries", C.c_longlong),
                ("batches", C.c_longlong), ("numtree", C.c_int), ("nleaves", C.c_int),
                ("depth", C.c_int), ("nterms", C.c_int), ("far_launches", C.c_int),
                ("near_launches", C.c_int), ("list_fallback", C.c_int),
                ("lists_shared", C.c_int)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class FieldParams(C.Structure):
    _fields_ = [("kind", C.c_int), ("precision", C.c_int), ("del_", C.c_double),
                ("mac_del", C.c_double), ("kappa", C.c_double), ("acc", C.c_double),
                ("kernel_order", C.c_int)]


FIELD_COULOMB, FIELD_SCREENED = 0, 1
KERNEL_ORDER_MAX = 8


class GmresOpts(C.Structure):
    _fields_ = [("restart", C.c_int), ("maxit", C.c_int), ("tol", C.c_double),
                ("precision", C.c_int), ("inner_tol", C.c_double),
                ("max_refinements", C.c_int)]


class GmresInfo(C.Structure):
    _fields_ = [("iterations", C.c_int), ("refinements", C.c_int), ("matvecs_fp64", C.c_int),
                ("matvecs_fp32", C.c_int), ("relres", C.c_double), ("seconds", C.c_double)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class ServerOpts(C.Structure):
    _fields_ = [("device", C.c_int), ("slots", C.c_int), ("hbm_budget", C.c_size_t)]


class RequestInfo(C.Structure):
    _fields_ = [("status", C.c_int), ("slot", C.c_int), ("t_submit", C.c_double),
                ("t_start", C.c_double), ("t_done", C.c_double),
                ("bytes_reserved", C.c_size_t), ("peak_bytes", C.c_size_t),
                ("gmres", GmresInfo)]

    def as_dict(self):
        d = {k: getattr(self, k) for k, _ in self._fields_ if k != "gmres"}
        d["gmres"] = self.gmres.as_dict()
        return d


class ServerInfo(C.Structure):
    _fields_ = [("submitted", C.c_longlong), ("completed", C.c_longlong),
                ("queued", C.c_longlong), ("running", C.c_int), ("max_running", C.c_int),
                ("slots", C.c_int), ("budget", C.c_size_t), ("reserved", C.c_size_t),
                ("max_reserved", C.c_size_t), ("now", C.c_double)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class PicOpts(C.Structure):
    _fields_ = [("steps", C.c_int), ("nterms", C.c_int), ("maxmemb", C.c_int), ("dt", C.c_double),
                ("del_", C.c_double), ("acc", C.c_double), ("charge_constant", C.c_double),
                ("invmass", C.c_double), ("precision", C.c_int)]


class Panel(C.Structure):
    _fields_ = [(k, C.c_double) for k in ("x0", "x1", "y0", "y1", "z0", "z1", "str", "xnrm",
                                          "ynrm", "znrm", "refpot", "midx", "midy", "midz")] + \
               [("type", C.c_int), ("orientation", C.c_int), ("area", C.c_double)]

    FIELDS = ("x0", "x1", "y0", "y1", "z0", "z1", "str", "xnrm", "ynrm", "znrm", "refpot",
              "midx", "midy", "midz", "type", "orientation", "area")


_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)
_vp = C.c_void_p

# (name, restype, argtypes) of every entry point in include/bit_b200.h
SIGNATURES = [
    ("bit_status_string", C.c_char_p, [C.c_int]),
    ("bit_abi_version", C.c_int, []),
    ("bit_kernel_launches", C.c_longlong, []),
    ("bit_ctx_create", C.c_int, [C.POINTER(_vp), C.POINTER(CtxOpts)]),
    ("bit_ctx_destroy", C.c_int, [_vp]),
    ("bit_ctx_last_error", C.c_char_p, [_vp]),
    ("bit_ctx_synchronize", C.c_int, [_vp]),
    ("bit_ctx_set_group_size", C.c_int, [_vp, C.c_int]),
    ("bit_ctx_set_work_queue", C.c_int, [_vp, C.c_int]),
    ("bit_ctx_set_near_config", C.c_int, [_vp, C.c_int, C.c_int]),
    ("bit_ctx_stream", C.c_int, [_vp, C.POINTER(_vp)]),
    ("bit_ctx_memory", C.c_int, [_vp, C.POINTER(C.c_size_t), C.POINTER(C.c_size_t)]),
    ("bit_tree_build", C.c_int, [_vp, C.c_int, _dp, _dp, _dp, C.c_int, C.POINTER(_vp)]),
    ("bit_tree_build_device", C.c_int, [_vp, C.c_int, _vp, _vp, _vp, C.c_int, C.POINTER(_vp)]),
    ("bit_tree_destroy", C.c_int, [_vp]),
    ("bit_tree_info", C.c_int, [_vp, _ip, _ip, _ip]),
    ("bit_tree_set_charges", C.c_int, [_vp, _dp, _dp]),
    ("bit_tree_set_charges_device", C.c_int, [_vp, _vp, _vp]),
    ("bit_tree_moments", C.c_int, [_vp, C.c_int]),
    ("bit_tree_export", C.c_int, [_vp, _ip, _ip, _dp, _ip]),
    ("bit_tree_export_moments", C.c_int, [_vp, _dp]),
    ("bit_eval_particles", C.c_int, [_vp, C.POINTER(EvalParams), _dp]),
    ("bit_eval_particles_device", C.c_int, [_vp, C.POINTER(EvalParams), _vp]),
    ("bit_eval_points", C.c_int, [_vp, C.POINTER(EvalParams), C.c_int, _dp, _dp, _dp, _dp]),
    ("bit_eval_force", C.c_int, [_vp, C.c_double, C.c_double, C.c_int, _dp, _dp, _dp]),
    ("bit_eval_field", C.c_int, [_vp, C.POINTER(FieldParams), _dp, _dp, _dp]),
    ("bit_direct_field", C.c_int, [_vp, C.c_int, _dp, _dp, _dp, _dp, C.c_int, C.c_double,
                                   C.c_int, C.c_int, _ip, _dp, _dp, _dp]),
    ("bit_treecode_potential", C.c_int, [_vp, C.c_int, _dp, _dp, _dp, _dp, _dp, C.c_int,
                                         C.c_int, C.POINTER(EvalParams), _dp]),
    ("bit_tree_stats", C.c_int, [_vp, C.POINTER(Stats)]),
    ("bit_device_fma_peak", C.c_int, [_vp, C.c_int, C.POINTER(C.c_double)]),
    ("bit_device_fp64_math_error", C.c_int, [_vp, C.c_longlong, C.POINTER(C.c_double),
                                             C.POINTER(C.c_double)]),
    ("bit_device_wait_check", C.c_int, [_vp, C.c_int]),
    ("bit_ctx_trim", C.c_int, [_vp, C.c_size_t]),
    ("bit_tree_target_lists", C.c_int, [_vp, C.POINTER(EvalParams), C.c_int, _ip, _ip, C.c_int,
                                        _ip]),
    ("bit_bie_solve", C.c_int, [_vp, C.POINTER(EvalParams), C.c_int, C.c_double, _dp, _dp, _dp,
                                C.POINTER(GmresOpts), C.POINTER(GmresInfo)]),
    ("bit_gmres_dense", C.c_int, [_vp, C.c_int, _dp, _dp, _dp, _ip]),
    ("bit_forest_build", C.c_int, [_vp, C.c_int, _ip, _ip, _dp, _dp, _dp, C.POINTER(_vp)]),
    ("bit_forest_build_device", C.c_int, [_vp, C.c_int, _ip, _ip, _vp, _vp, _vp,
                                          C.POINTER(_vp)]),
    ("bit_forest_moments", C.c_int, [_vp, _ip]),
    ("bit_forest_eval", C.c_int, [_vp, C.POINTER(EvalParams), _dp]),
    ("bit_forest_eval_device", C.c_int, [_vp, C.POINTER(EvalParams), _vp]),
    ("bit_forest_systems", C.c_int, [_vp, _ip]),
    ("bit_direct_potential", C.c_int, [_vp, C.c_int, _dp, _dp, _dp, _dp, C.POINTER(EvalParams),
                                       C.c_int, _ip, _dp]),
    ("bit_direct_potential_device", C.c_int, [_vp, C.c_int, _vp, _vp, _vp, _vp,
                                              C.POINTER(EvalParams), C.c_int, _vp, _vp]),
    ("bit_server_create", C.c_int, [C.POINTER(_vp), C.POINTER(ServerOpts)]),
    ("bit_server_destroy", C.c_int, [_vp]),
    ("bit_server_submit_eval", C.c_int, [_vp, C.c_int, _dp, _dp, _dp, _dp, C.c_int, C.c_int,
                                         C.POINTER(EvalParams), C.POINTER(C.c_longlong)]),
    ("bit_server_submit_solve", C.c_int, [_vp, C.c_int, _dp, _dp, _dp, _dp, _dp, C.c_int,
                                          C.c_int, C.POINTER(EvalParams), C.c_double,
                                          C.POINTER(GmresOpts), C.POINTER(C.c_longlong)]),
    ("bit_server_wait", C.c_int, [_vp, C.c_longlong, _dp, C.POINTER(RequestInfo)]),
    ("bit_server_poll", C.c_int, [_vp, C.c_longlong, _ip]),
    ("bit_server_stats", C.c_int, [_vp, C.POINTER(ServerInfo)]),
    ("bit_server_last_error", C.c_char_p, [_vp]),
    ("bit_pic_steps", C.c_int, [_vp, C.c_int, _vp, _vp, _vp, _vp, _vp, _vp, _vp,
                                C.POINTER(PicOpts), _vp, _vp, _vp]),
    ("bit_panels_box", C.c_int, [C.c_int, C.c_int, C.c_int, C.c_double, C.c_double, C.c_double,
                                 C.POINTER(Panel), _ip]),
    ("bit_panel_matrix", C.c_int, [_vp, C.c_int, C.POINTER(Panel), C.c_double, _dp]),
    ("bit_panel_solve", C.c_int, [_vp, C.c_int, C.POINTER(Panel), C.c_int, _dp, _dp, _dp, _dp,
                                  C.c_double, C.c_int, C.c_double, C.c_int,
                                  C.POINTER(GmresOpts), C.POINTER(GmresInfo)]),
    ("bit_write_potential", C.c_int, [C.c_char_p, C.c_int, _dp, _dp, _dp, _dp]),
    ("bit_write_potential_device", C.c_int, [_vp, C.c_char_p, C.c_int, _vp, _vp, _vp, _vp]),
    ("bit_gmres_dense_static", C.c_int, [_vp, C.c_int, _dp, _dp, _dp, _ip, C.c_char_p,
                                         C.c_int]),
]

_lib = None


def lib():
    """The loaded libbit_b200.so (raises BitError if it was not built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise BitError(2, f"{LIB_PATH} not built (run python -m bit_b200.build)")
        L = C.CDLL(LIB_PATH)
        for name, res, args in SIGNATURES:
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def _d(a):
    return a.ctypes.data_as(_dp)


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def panels_box(xpanels, ypanels, zpanels, dlength, dheight, ddepth):
    """setboundaries: a ctypes array of Panel (and .as_array(): (numpan, 17) floats)."""
    n = C.c_int()
    st = lib().bit_panels_box(xpanels, ypanels, zpanels, dlength, dheight, ddepth, None,
                              C.byref(n))
    if st:
        raise BitError(st, "bit_panels_box")
    arr = (Panel * n.value)()
    lib().bit_panels_box(xpanels, ypanels, zpanels, dlength, dheight, ddepth, arr, C.byref(n))
    return arr


def panels_as_array(pan):
    return np.array([[getattr(p, k) for k in Panel.FIELDS] for p in pan], dtype=np.float64)


def write_potential(path, x, y, z, pot):
    """output_potential: 'i\tx\ty\tz\tpot' per particle, 14 significant digits."""
    x, y, z, pot = map(_f64, (x, y, z, pot))
    st = lib().bit_write_potential(path.encode(), len(x), _d(x), _d(y), _d(z), _d(pot))
    if st:
        raise BitError(st, f"bit_write_potential {path}")


def kernel_launches():
    """Kernels launched by libbit_b200 in this process so far."""
    return lib().bit_kernel_launches()


def params(kernel=COULOMB, mode=CONSISTENT, precision=FP64, del_=0.0, mac_del=0.0, kappa=0.0,
           acc=0.5, intg=REF_INTG):
    return EvalParams(kernel, mode, precision, del_, mac_del, kappa, acc, intg)


class Context:
    """One CUDA stream on one device (bit_ctx_create)."""

    def __init__(self, device=0, stream=None, hbm_budget=0):
        self.h = _vp()
        self._trees = weakref.WeakSet()
        opts = CtxOpts(device, stream, hbm_budget)
        st = lib().bit_ctx_create(C.byref(self.h), C.byref(opts))
        if st:
            raise BitError(st, "bit_ctx_create")

    def check(self, st, what):
        if st:
            msg = lib().bit_ctx_last_error(self.h)
            raise BitError(st, f"{what}: {msg.decode() if msg else ''}")

    def close(self):
        if self.h:
            for t in list(self._trees):
                t.treeempty()
            lib().bit_ctx_destroy(self.h)
            self.h = _vp()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def stream(self):
        s = _vp()
        lib().bit_ctx_stream(self.h, C.byref(s))
        return s.value

    def fma_peak(self, precision):
        """Measured FMA throughput of the device in flop/s (FP64 or MIXED = FP32)."""
        v = C.c_double()
        self.check(lib().bit_device_fma_peak(self.h, precision, C.byref(v)), "bit_device_fma_peak")
        return v.value

    def fp64_math_error(self, n=1 << 22):
        """Largest difference, in ulps of CUDA's result, of the FP64 near field's own exp
        and rsqrt from CUDA's, over n seeded arguments: {"exp": e, "rsqrt": r}."""
        e, r = C.c_double(), C.c_double()
        self.check(lib().bit_device_fp64_math_error(self.h, n, C.byref(e), C.byref(r)),
                   "bit_device_fp64_math_error")
        return {"exp": e.value, "rsqrt": r.value}

    def wait_check(self, limit=1000):
        """Run the device-side give-up path of a bounded wait (a barrier nothing
        completes); returns the status (BIT_ERR_CUDA when the wait gave up, as it must)."""
        return lib().bit_device_wait_check(self.h, limit)

    def memory(self):
        a, b = C.c_size_t(), C.c_size_t()
        lib().bit_ctx_memory(self.h, C.byref(a), C.byref(b))
        return a.value, b.value

    def trim(self, keep=0):
        """Free the context's cached device blocks until it holds at most `keep` bytes."""
        self.check(lib().bit_ctx_trim(self.h, keep), "bit_ctx_trim")

    def set_group_size(self, targets):
        """Leaf packing (0: off, else 32..1024 targets per group): a tuning knob."""
        self.check(lib().bit_ctx_set_group_size(self.h, targets), "bit_ctx_set_group_size")

    def set_near_config(self, tile=0, threads_per_target=0):
        """Near-field source tile and threads-per-target cap (0, 0: the defaults)."""
        self.check(lib().bit_ctx_set_near_config(self.h, tile, threads_per_target),
                   "bit_ctx_set_near_config")

    def set_work_queue(self, on):
        """Forests: one persistent kernel per field over a device work queue (True, the
        default) or one launch per (nterms, kernel) class (False)."""
        self.check(lib().bit_ctx_set_work_queue(self.h, int(bool(on))), "bit_ctx_set_work_queue")

    def synchronize(self):
        self.check(lib().bit_ctx_synchronize(self.h), "synchronize")

    def treemake(self, x, y, z, maxmemb):
        return Tree(self, x, y, z, maxmemb)

    def treemake_device(self, n, xptr, yptr, zptr, maxmemb):
        return Tree(self, None, None, None, maxmemb, device=(n, xptr, yptr, zptr))

    def treecode_potential(self, x, y, z, q, nterms, maxmemb, prm, w=None):
        x, y, z, q = map(_f64, (x, y, z, q))
        w = None if w is None else _f64(w)
        out = np.zeros(len(x))
        st = lib().bit_treecode_potential(self.h, len(x), _d(x), _d(y), _d(z), _d(q),
                                          None if w is None else _d(w), nterms, maxmemb,
                                          C.byref(prm), _d(out))
        self.check(st, "bit_treecode_potential")
        return out

    def forest(self, x, y, z, sizes, maxmemb):
        """Independent systems in one tree: system s is the next sizes[s] particles."""
        return Forest(self, x, y, z, sizes, maxmemb)

    def forest_device(self, sizes, maxmemb, xptr, yptr, zptr):
        return Forest(self, None, None, None, sizes, maxmemb, device=(xptr, yptr, zptr))

    def direct(self, x, y, z, q, prm, targets):
        """FP64 direct sum at particle targets (bit_direct_potential)."""
        x, y, z, q = map(_f64, (x, y, z, q))
        tg = np.ascontiguousarray(targets, dtype=np.int32)
        out = np.zeros(len(tg))
        self.check(lib().bit_direct_potential(self.h, len(x), _d(x), _d(y), _d(z), _d(q),
                                              C.byref(prm), len(tg), tg.ctypes.data_as(_ip),
                                              _d(out)), "bit_direct_potential")
        return out

    def direct_field(self, x, y, z, q, targets, del_=0.0, regularised=True, kernel_order=0):
        """FP64 field direct sum at particle targets (bit_direct_field):
        force_particle_ds_reg / force_particle_ds_noreg.  Returns (fx, fy, fz)."""
        x, y, z, q = map(_f64, (x, y, z, q))
        tg = np.ascontiguousarray(targets, dtype=np.int32)
        fx, fy, fz = np.zeros(len(tg)), np.zeros(len(tg)), np.zeros(len(tg))
        self.check(lib().bit_direct_field(self.h, len(x), _d(x), _d(y), _d(z), _d(q),
                                          int(bool(regularised)), del_, kernel_order, len(tg),
                                          tg.ctypes.data_as(_ip), _d(fx), _d(fy), _d(fz)),
                   "bit_direct_field")
        return fx, fy, fz

    def direct_device(self, n, xp, yp, zp, qp, prm, m, tgp, outp):
        self.check(lib().bit_direct_potential_device(self.h, n, xp, yp, zp, qp, C.byref(prm), m,
                                                     tgp, outp), "bit_direct_potential_device")

    def pic_steps_device(self, n, ptrs, qptr, opts, fptrs=(None, None, None)):
        """bit_pic_steps on device arrays: ptrs = (x, y, z, u, v, w) updated in place."""
        self.check(lib().bit_pic_steps(self.h, n, *ptrs, qptr, C.byref(opts), *fptrs),
                   "bit_pic_steps")

    def panel_matrix(self, pan, del_):
        n = len(pan)
        A = np.zeros(n * n)
        self.check(lib().bit_panel_matrix(self.h, n, pan, del_, _d(A)), "bit_panel_matrix")
        return A.reshape(n, n)

    def panel_solve(self, pan, x, y, z, q, del_, nterms, acc, maxmemb, restart=50, tol=1e-10,
                    maxit=1000):
        """Sets pan[i].str; returns (sigma, info, status)."""
        x, y, z, q = map(_f64, (x, y, z, q))
        opts = GmresOpts(restart, maxit, tol, FP64, 0.0, 0)
        info = GmresInfo()
        st = lib().bit_panel_solve(self.h, len(pan), pan, len(x), _d(x), _d(y), _d(z), _d(q),
                                   del_, nterms, acc, maxmemb, C.byref(opts), C.byref(info))
        if st not in (0, 7):
            self.check(st, "bit_panel_solve")
        return np.array([p.str for p in pan]), info.as_dict(), st

    def write_potential_device(self, path, n, xp, yp, zp, potp):
        self.check(lib().bit_write_potential_device(self.h, path.encode(), n, xp, yp, zp, potp),
                   "bit_write_potential_device")

    def gmres_dense(self, A, b, x0=None):
        """solver::gmres (src/solver.h:157) on the device."""
        A, b = _f64(A), _f64(b)
        x = np.ones(len(b)) if x0 is None else _f64(x0).copy()
        it = C.c_int()
        st = lib().bit_gmres_dense(self.h, len(b), _d(A), _d(b), _d(x), C.byref(it))
        if st not in (0, 6):
            self.check(st, "bit_gmres_dense")
        return x, it.value, st


class Tree:
    def __init__(self, ctx, x, y, z, maxmemb, device=None):
        self.ctx = ctx
        self.h = _vp()
        if device is None:
            self.x, self.y, self.z = map(_f64, (x, y, z))
            self.n = len(self.x)
            st = lib().bit_tree_build(ctx.h, self.n, _d(self.x), _d(self.y), _d(self.z),
                                      maxmemb, C.byref(self.h))
        else:
            self.n, xp, yp, zp = device
            st = lib().bit_tree_build_device(ctx.h, self.n, xp, yp, zp, maxmemb,
                                             C.byref(self.h))
        ctx.check(st, "bit_tree_build")
        ctx._trees.add(self)
        self.maxmemb = maxmemb
        self.nterms = 0
        a, b, c = C.c_int(), C.c_int(), C.c_int()
        lib().bit_tree_info(self.h, C.byref(a), C.byref(b), C.byref(c))
        self.numtree, self.nleaves, self.depth = a.value, b.value, c.value

    def treeempty(self):
        if self.h:
            if self.ctx.h:
                lib().bit_tree_destroy(self.h)
            self.h = _vp()

    close = treeempty

    def __del__(self):
        try:
            self.treeempty()
        except Exception:
            pass

    def set_charges(self, q, w=None):
        q = _f64(q)
        w = None if w is None else _f64(w)
        self.ctx.check(lib().bit_tree_set_charges(self.h, _d(q), None if w is None else _d(w)),
                       "bit_tree_set_charges")

    def set_charges_device(self, qptr, wptr=None):
        self.ctx.check(lib().bit_tree_set_charges_device(self.h, qptr, wptr),
                       "bit_tree_set_charges_device")

    def moments(self, nterms):
        self.ctx.check(lib().bit_tree_moments(self.h, nterms), "bit_tree_moments")
        self.nterms = nterms

    def treemoments(self, q, nterms, w=None):
        self.set_charges(q, w)
        self.moments(nterms)

    def export(self):
        nt = self.numtree
        nm = np.zeros(nt, np.int32)
        ch = np.zeros(nt * 8, np.int32)
        f = np.zeros(nt * 13)
        self.ctx.check(lib().bit_tree_export(self.h, nm.ctypes.data_as(_ip), ch.ctypes.data_as(_ip),
                                             _d(f), None), "bit_tree_export")
        mem = np.zeros(int(nm.sum()), np.int32)
        self.ctx.check(lib().bit_tree_export(self.h, None, None, None, mem.ctypes.data_as(_ip)),
                       "bit_tree_export")
        return nm, ch.reshape(nt, 8), f.reshape(nt, 13), mem

    def export_moments(self):
        T = self.nterms * (self.nterms + 1) * (self.nterms + 2) // 6
        m = np.zeros(self.numtree * T)
        self.ctx.check(lib().bit_tree_export_moments(self.h, _d(m)), "bit_tree_export_moments")
        return m.reshape(self.numtree, T)

    def evaluate(self, prm, points=None, out=None):
        """Potential at every particle (or at `points`).  `out`: an optional C-contiguous
        float64 array of the right length to write into, so that repeated calls reuse one
        buffer instead of faulting in fresh pages each time."""
        m = self.n if points is None else len(points)
        if out is None:
            out = np.zeros(m)
        elif (not isinstance(out, np.ndarray) or out.dtype != np.float64 or out.shape != (m,)
              or not out.flags["C_CONTIGUOUS"] or not out.flags["WRITEABLE"]):
            raise ValueError(f"out must be a writeable C-contiguous float64 array of length {m}")
        if points is not None:
            pts = _f64(points)
            tx, ty, tz = [np.ascontiguousarray(pts[:, a]) for a in range(3)]
            self.ctx.check(lib().bit_eval_points(self.h, C.byref(prm), len(pts), _d(tx), _d(ty),
                                                 _d(tz), _d(out)), "bit_eval_points")
            return out
        self.ctx.check(lib().bit_eval_particles(self.h, C.byref(prm), _d(out)),
                       "bit_eval_particles")
        return out

    def evaluate_device(self, prm, outptr):
        self.ctx.check(lib().bit_eval_particles_device(self.h, C.byref(prm), outptr),
                       "bit_eval_particles_device")

    def treepotential(self, acc, del_, mode=CONSISTENT, precision=FP64, points=None):
        return self.evaluate(params(COULOMB, mode, precision, del_=del_, acc=acc), points)

    def shielded_treepot(self, kappa, acc, mode=CONSISTENT, precision=FP64, mac_del=0.0,
                         intg=REF_INTG, points=None):
        return self.evaluate(params(SCREENED, mode, precision, mac_del=mac_del, kappa=kappa,
                                    acc=acc, intg=intg), points)

    def treeforce(self, acc, del_, precision=FP64):
        fx, fy, fz = np.zeros(self.n), np.zeros(self.n), np.zeros(self.n)
        self.ctx.check(lib().bit_eval_force(self.h, del_, acc, precision, _d(fx), _d(fy), _d(fz)),
                       "bit_eval_force")
        return fx, fy, fz

    def field(self, kind=FIELD_COULOMB, acc=0.5, del_=0.0, kappa=0.0, mac_del=0.0,
              kernel_order=0, precision=FP64):
        """bit_eval_field: treeforce with KERNEL_ORDER (FIELD_COULOMB) or shielded_treeforce's
        screened 2-D field (FIELD_SCREENED) at every particle; returns (fx, fy, fz)."""
        fx, fy, fz = np.zeros(self.n), np.zeros(self.n), np.zeros(self.n)
        prm = FieldParams(kind, precision, del_, mac_del, kappa, acc, kernel_order)
        self.ctx.check(lib().bit_eval_field(self.h, C.byref(prm), _d(fx), _d(fy), _d(fz)),
                       "bit_eval_field")
        return fx, fy, fz

    def stats(self):
        s = Stats()
        self.ctx.check(lib().bit_tree_stats(self.h, C.byref(s)), "bit_tree_stats")
        return s.as_dict()

    def target_lists(self, prm, p, cap=8192):
        node = np.zeros(cap, np.int32)
        kind = np.zeros(cap, np.int32)
        n = C.c_int()
        self.ctx.check(lib().bit_tree_target_lists(self.h, C.byref(prm), p,
                                                   node.ctypes.data_as(_ip),
                                                   kind.ctypes.data_as(_ip), cap, C.byref(n)),
                       "bit_tree_target_lists")
        return node[:n.value].copy(), kind[:n.value].copy()

    def bie_solve(self, prm, nterms, diag, w, f, restart=50, tol=1e-8, maxit=1000,
                  precision=FP64, inner_tol=0.0, max_refinements=0):
        """GMRES(m) on (diag*I + K) s = f with the treecode as the matvec."""
        w, f = _f64(w), _f64(f)
        s = np.zeros(self.n)
        opts = GmresOpts(restart, maxit, tol, precision, inner_tol, max_refinements)
        info = GmresInfo()
        st = lib().bit_bie_solve(self.h, C.byref(prm), nterms, diag, _d(w), _d(f), _d(s),
                                 C.byref(opts), C.byref(info))
        if st not in (0, 7):
            self.ctx.check(st, "bit_bie_solve")
        return s, info.as_dict(), st


class Forest(Tree):
    """Many independent systems in one tree (bit_forest_build): system s owns the next
    sizes[s] particles, is split with maxmemb[s] and rooted at node s.  Each system is
    evaluated with its own parameters and expansion order, and its result equals a
    separate single-system evaluation."""

    def __init__(self, ctx, x, y, z, sizes, maxmemb, device=None):
        self.ctx = ctx
        self.h = _vp()
        self.sizes = np.ascontiguousarray(sizes, dtype=np.int32)
        self.nsys = len(self.sizes)
        mm = np.broadcast_to(np.asarray(maxmemb, dtype=np.int32), (self.nsys,))
        self.maxmembs = np.ascontiguousarray(mm)
        self.n = int(self.sizes.sum())
        if device is None:
            self.x, self.y, self.z = map(_f64, (x, y, z))
            if self.n != len(self.x):
                raise ValueError("sizes must add up to the number of particles")
            st = lib().bit_forest_build(ctx.h, self.nsys, self.sizes.ctypes.data_as(_ip),
                                        self.maxmembs.ctypes.data_as(_ip), _d(self.x),
                                        _d(self.y), _d(self.z), C.byref(self.h))
        else:
            xp, yp, zp = device
            st = lib().bit_forest_build_device(ctx.h, self.nsys, self.sizes.ctypes.data_as(_ip),
                                               self.maxmembs.ctypes.data_as(_ip), xp, yp, zp,
                                               C.byref(self.h))
        ctx.check(st, "bit_forest_build")
        ctx._trees.add(self)
        self.maxmemb = int(self.maxmembs.min())
        self.nterms = 0
        self.nterms_sys = np.zeros(self.nsys, np.int32)
        a, b, c = C.c_int(), C.c_int(), C.c_int()
        lib().bit_tree_info(self.h, C.byref(a), C.byref(b), C.byref(c))
        self.numtree, self.nleaves, self.depth = a.value, b.value, c.value
        self.offsets = np.concatenate([[0], np.cumsum(self.sizes)])

    def moments(self, nterms):
        nt = np.ascontiguousarray(np.broadcast_to(np.asarray(nterms, np.int32), (self.nsys,)))
        self.ctx.check(lib().bit_forest_moments(self.h, nt.ctypes.data_as(_ip)),
                       "bit_forest_moments")
        self.nterms_sys = nt.copy()
        self.nterms = int(nt.max())

    def export_moments(self):
        raise NotImplementedError("forest moments differ in size per system; use export()")

    def _params(self, prm):
        if isinstance(prm, EvalParams):
            prm = [prm] * self.nsys
        if len(prm) != self.nsys:
            raise ValueError("one parameter set per system expected")
        arr = (EvalParams * self.nsys)()
        for i, p in enumerate(prm):
            arr[i] = p
        return arr

    def evaluate(self, prm, points=None):
        """prm: one EvalParams for all systems, or a sequence of one per system."""
        if points is not None:
            raise ValueError("external points need a single-system tree")
        arr = self._params(prm)
        out = np.zeros(self.n)
        self.ctx.check(lib().bit_forest_eval(self.h, arr, _d(out)), "bit_forest_eval")
        return out

    def evaluate_device(self, prm, outptr):
        arr = prm if isinstance(prm, C.Array) else self._params(prm)
        self.ctx.check(lib().bit_forest_eval_device(self.h, arr, outptr), "bit_forest_eval_device")

    def system(self, s, a):
        """System s's slice of a per-particle array."""
        return a[self.offsets[s]:self.offsets[s + 1]]


class Server:
    """Request loop with continuous batching (bit_server_*): evaluate and solve requests
    of any size, admitted as slots and HBM budget free up, overlapping on the device."""

    def __init__(self, device=0, slots=4, hbm_budget=0):
        self.h = _vp()
        self.sizes = {}
        opts = ServerOpts(device, slots, hbm_budget)
        st = lib().bit_server_create(C.byref(self.h), C.byref(opts))
        if st:
            raise BitError(st, "bit_server_create")

    def _check(self, st, what):
        if st:
            msg = lib().bit_server_last_error(self.h)
            raise BitError(st, f"{what}: {msg.decode() if msg else ''}")

    def submit_eval(self, x, y, z, q, nterms, maxmemb, prm):
        x, y, z, q = map(_f64, (x, y, z, q))
        rid = C.c_longlong()
        self._check(lib().bit_server_submit_eval(self.h, len(x), _d(x), _d(y), _d(z), _d(q),
                                                 nterms, maxmemb, C.byref(prm), C.byref(rid)),
                    "bit_server_submit_eval")
        self.sizes[rid.value] = len(x)
        return rid.value

    def submit_solve(self, x, y, z, w, f, nterms, maxmemb, prm, diag, restart=50, tol=1e-8,
                     maxit=1000, precision=FP64, inner_tol=0.0, max_refinements=0):
        x, y, z, w, f = map(_f64, (x, y, z, w, f))
        rid = C.c_longlong()
        opts = GmresOpts(restart, maxit, tol, precision, inner_tol, max_refinements)
        self._check(lib().bit_server_submit_solve(self.h, len(x), _d(x), _d(y), _d(z), _d(w),
                                                  _d(f), nterms, maxmemb, C.byref(prm), diag,
                                                  C.byref(opts), C.byref(rid)),
                    "bit_server_submit_solve")
        self.sizes[rid.value] = len(x)
        return rid.value

    def wait(self, rid):
        """(result, info dict, status) of a request; blocks until it is done."""
        out = np.zeros(self.sizes.pop(rid))
        info = RequestInfo()
        st = lib().bit_server_wait(self.h, rid, _d(out), C.byref(info))
        return out, info.as_dict(), st

    def done(self, rid):
        d = C.c_int()
        self._check(lib().bit_server_poll(self.h, rid, C.byref(d)), "bit_server_poll")
        return bool(d.value)

    def stats(self):
        si = ServerInfo()
        self._check(lib().bit_server_stats(self.h, C.byref(si)), "bit_server_stats")
        return si.as_dict()

    def close(self):
        if self.h:
            lib().bit_server_destroy(self.h)
            self.h = _vp()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

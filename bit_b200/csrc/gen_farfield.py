"""Generate farfield_gen.cuh: unrolled far-field Taylor recurrences for nterms = 1..10.

Moments are read in shell order (total degree, then i, then j descending: the order the
coefficients are produced in) from a staging copy, four at a time.

For every nterms and kernel this writes one straight-line device function that evaluates
the Taylor coefficients of the cluster kernel degree by degree and folds each one into
the moment dot product as soon as it exists, so only the last two degree shells stay live
in registers.  The coefficient of each index pattern follows the reference's recurrence
for that pattern (constants 1/k etc. folded into literals):

  Coulomb potential   treetaylorpotential, src/tree3d.cpp:4484-4629  (sum: :4632-4638,
                      to degree nterms-1)
  screened potential  shielded_treetaylorpot, src/tree3d.cpp:3042-3214 (sum: :3219-3225)
  Coulomb force       treetaylorforce, src/tree3d.cpp:472-612 (sum: :794-808)

Usage: python gen_farfield.py <out.cuh>
"""
import sys

AX = "xyz"


def lit(v):
    return f"T({float(v)!r})"


def name(p, v):
    return f"{p}{v[0]}_{v[1]}_{v[2]}"


def sub(v, a, by):
    w = list(v)
    w[a] -= by
    return tuple(w)


def shells(maxdeg):
    for d in range(maxdeg + 1):
        for i in range(d, -1, -1):
            for j in range(d - i, -1, -1):
                yield (i, j, d - i - j)


def moment_index(nt):
    idx, out = 0, {}
    for i in range(nt):
        for j in range(nt - i):
            for k in range(nt - i - j):
                out[(i, j, k)] = idx
                idx += 1
    return out


def shell_index(nt):
    """Position of each (i, j, k), degree < nt, in the order the recurrences produce them."""
    return {v: n for n, v in enumerate(shells(nt - 1))}


def padded(n):
    return (n + 3) // 4 * 4


class MomentLoads:
    """Moments are consumed in shell order: load them four at a time (16-byte vectors)."""

    def __init__(self):
        self.done = set()

    def get(self, L, idx):
        q = idx // 4
        if q not in self.done:
            L.append(f"  const V4<T> mv{q} = ld4(M, {q});")
            self.done.add(q)
        return f"mv{q}.{'xyzw'[idx % 4]}"


def classify(v):
    nz = sum(1 for a in v if a == 0)
    n1 = sum(1 for a in v if a == 1)
    ax = [a for a in range(3) if v[a] > 0]
    return nz, n1, ax


# ---------------------------------------------------------------------------- Coulomb
def coul_expr(v):
    b = lambda w: name("b", w)
    d = lambda a: "d" + AX[a]
    d2 = lambda a: "d" + AX[a] + "2"
    nz, n1, ax = classify(v)
    if nz == 3:
        return "sqfac"
    if nz == 2:
        u, k = ax[0], v[ax[0]]
        if k == 1:
            return f"fac*{d(u)}*sqfac"
        ik = 1.0 / k
        return f"fac*({lit(2.0 - ik)}*{d(u)}*{b(sub(v, u, 1))} - {lit(1 - ik)}*{b(sub(v, u, 2))})"
    if nz == 1 and n1 == 2:
        u, w = ax
        return f"fac*({d(u)}*{b(sub(v, u, 1))} + {d2(w)}*{b(sub(v, w, 1))})"
    if nz == 1 and n1 == 0:
        u, w = ax
        ii = 1.0 / v[u]
        return (f"fac*({lit(2.0 - ii)}*{d(u)}*{b(sub(v, u, 1))} + {d2(w)}*{b(sub(v, w, 1))}"
                f" - {lit(1 - ii)}*{b(sub(v, u, 2))} - {b(sub(v, w, 2))})")
    if n1 >= 1:
        f = next(a for a in range(3) if v[a] == 1)
        s = f"{d(f)}*{b(sub(v, f, 1))}"
        for a in range(3):
            if a != f and v[a] > 0:
                s += f" + {d2(a)}*{b(sub(v, a, 1))}"
        for a in range(3):
            if a != f and v[a] >= 2:
                s += f" - {b(sub(v, a, 2))}"
        return f"fac*({s})"
    ii = 1.0 / v[0]
    return (f"fac*({lit(2.0 * (1 - 0.5 * ii))}*dx*{b(sub(v, 0, 1))} + dy2*{b(sub(v, 1, 1))}"
            f" + dz2*{b(sub(v, 2, 1))} - {lit(1.0 - ii)}*{b(sub(v, 0, 2))}"
            f" - {b(sub(v, 1, 2))} - {b(sub(v, 2, 2))})")


def gen_coulomb(nt):
    mi = shell_index(nt)
    ml = MomentLoads()
    L = ["  const T dx2 = T(2)*dx, dy2 = T(2)*dy, dz2 = T(2)*dz;",
         "  const T fac = T(1) / rs;",
         "  const T sqfac = sqrt_t(fac);",
         "  T s = T(0);"]
    for v in shells(nt - 1):
        L.append(f"  const T {name('b', v)} = {coul_expr(v)};")
        m = ml.get(L, mi[v])
        L.append(f"  s = fma_t({m}, {name('b', v)}, s);")
    L.append("  return s;")
    return L


# ---------------------------------------------------------------------------- screened
def scr_expr(v):
    a_ = lambda w: name("a", w)
    b_ = lambda w: name("c", w)
    d = lambda a: "d" + AX[a]
    dd = lambda a: "d" + AX[a] + "2"
    kd = lambda a: "kd" + AX[a]
    nz, n1, ax = classify(v)
    if nz == 2 and n1 == 1:
        u = ax[0]
        return (f"{kd(u)}*a0_0_0", f"fac*{d(u)}*(a0_0_0 + kappa*c0_0_0)")
    if n1 == 0:
        u = ax[0]
        i = v[u]
        cf1, cf2, cf3 = 1.0 / i, 1.0 - 1.0 / (2.0 * i), 1.0 - 1.0 / i
        bexp = f"(kappa*{lit(cf1)})*({d(u)}*{a_(sub(v, u, 1))} - {a_(sub(v, u, 2))})"
        s = f"{dd(u)}*{lit(cf2)}*{a_(sub(v, u, 1))}"
        for a in ax[1:]:
            s += f" + {dd(a)}*{a_(sub(v, a, 1))}"
        s += f" - {lit(cf3)}*{a_(sub(v, u, 2))}"
        for a in ax[1:]:
            s += f" - {a_(sub(v, a, 2))}"
        s += f" + (kappa*{lit(cf1)})*({d(u)}*{b_(sub(v, u, 1))} - {b_(sub(v, u, 2))})"
        return (bexp, f"fac*({s})")
    f = next(a for a in range(3) if v[a] == 1)
    bexp = f"{kd(f)}*{a_(sub(v, f, 1))}"
    s = f"{d(f)}*{a_(sub(v, f, 1))}"
    for a in range(3):
        if a != f and v[a] > 0:
            s += f" + {dd(a)}*{a_(sub(v, a, 1))}"
    for a in range(3):
        if a != f and v[a] >= 2:
            s += f" - {a_(sub(v, a, 2))}"
    s += f" + {kd(f)}*{b_(sub(v, f, 1))}"
    return (bexp, f"fac*({s})")


def gen_screened(nt):
    mi = shell_index(nt)
    ml = MomentLoads()
    L = ["  const T dx2 = T(2)*dx, dy2 = T(2)*dy, dz2 = T(2)*dz;",
         "  const T kdx = kappa*dx, kdy = kappa*dy, kdz = kappa*dz;",
         "  const T rinv = rsqrt_t(dist2);",
         "  const T fac = rinv * rinv;",
         "  const T c0_0_0 = exp_t(-kappa * (dist2 * rinv));",
         "  const T a0_0_0 = c0_0_0 * rinv;",
         "  T s = T(0);"]
    m = ml.get(L, 0)
    L.append(f"  s = fma_t({m}, a0_0_0, s);")
    for v in shells(nt - 1):
        if v == (0, 0, 0):
            continue
        bexp, aexp = scr_expr(v)
        L.append(f"  const T {name('c', v)} = {bexp};")
        L.append(f"  const T {name('a', v)} = {aexp};")
        m = ml.get(L, mi[v])
        L.append(f"  s = fma_t({m}, {name('a', v)}, s);")
    L.append("  return s;")
    return L


# ------------------------------------------------------- scaled forms (FP32 path)
# The same recurrences on scaled coefficients: with R the (regularised) distance, u = d/R
# the unit vector and n = |v|, the Coulomb b~_v = b_v R^(n+1), the screened a~_v = a_v R^(n+1)
# and c~_v = c_v R^n, rho = kappa R.  Substituting d = R u and fac = R^-2 into each pattern
# of the reference's recurrence removes the fac multiply (e.g. the screened generic pattern
# a~_v = u_f a~_{v-f} + 2 u_a a~_{v-a} - a~_{v-2a} + rho u_f c~_{v-f}).  The moments come
# normalised by h^n (h = 2^e above the cluster radius), so the potential is
# sum_n S_n (h/R)^n / R with S_n the dot product of shell n: q_n = (h/R)^n / R <= 1/R at
# any scale, where the unscaled coefficients (~R^-(n+1)) overflow FP32 for R below ~1e-4.
# Subtracted terms start each fma chain, so they cost no separate instruction.


def _chain(start, terms):
    """fma_t chain: terms [(mult, var)] added in order onto `start` (None: the first term
    is a plain product)."""
    e = start
    for m, v in terms:
        e = f"{m}*{v}" if e is None else f"fma_t({m}, {v}, {e})"
    return e


def _neg_sum(vs):
    return None if not vs else ("-" + vs[0] if len(vs) == 1 else "-(" + " + ".join(vs) + ")")


class ShellSum:
    """Per-shell dot products folded into s with the factor q_n = (h/R)^n / R."""

    def __init__(self, L, mi):
        self.L, self.mi, self.ml, self.deg, self.first = L, mi, MomentLoads(), 0, True

    def add(self, v, var):
        L = self.L
        d = sum(v)
        if d != self.deg:
            self.flush()
            self.deg, self.first = d, True
        m = self.ml.get(L, self.mi[v])
        if self.first:
            L.append(f"  S = {m} * {var};")
            self.first = False
        else:
            L.append(f"  S = fma_t({m}, {var}, S);")

    def flush(self):
        if self.deg == 0:
            self.L.append("  T s = S * q;")
        else:
            self.L.append("  q = q * eta;")
            self.L.append("  s = fma_t(S, q, s);")

    def done(self):
        self.flush()
        self.L.append("  return s;")


def coul_scaled_expr(v, hs=None):
    """hs: a Hoisted whose (2 - 1/i) u_a products replace the literal multiplies."""
    b = lambda w: "E" if w == (0, 0, 0) else name("B", w)
    axis = lambda a, i: (f"{U(a)}, {lit(2.0 - 1.0 / i)}*" if hs is None else f"{hs.uc(a, i)}, ")
    U = lambda a: "u" + AX[a]
    U2 = lambda a: "u" + AX[a] + "2"
    nz, n1, ax = classify(v)
    if nz == 2:
        u, k = ax[0], v[ax[0]]
        if k == 1:
            return U(u)
        ik = 1.0 / k
        return f"fma_t({axis(u, k)}{b(sub(v, u, 1))}, -({lit(1 - ik)}*{b(sub(v, u, 2))}))"
    if nz == 1 and n1 == 2:
        u, w = ax
        return _chain(None, [(U(u), b(sub(v, u, 1))), (U2(w), b(sub(v, w, 1)))])
    if nz == 1 and n1 == 0:
        u, w = ax
        ii = 1.0 / v[u]
        e = f"fma_t({lit(-(1 - ii))}, {b(sub(v, u, 2))}, -{b(sub(v, w, 2))})"
        e = _chain(e, [(U2(w), b(sub(v, w, 1)))])
        return f"fma_t({axis(u, v[u])}{b(sub(v, u, 1))}, {e})"
    if n1 >= 1:
        f = next(a for a in range(3) if v[a] == 1)
        subs = [b(sub(v, a, 2)) for a in range(3) if a != f and v[a] >= 2]
        ns = _neg_sum(subs)
        e = f"{U(f)}*{b(sub(v, f, 1))}" if ns is None else f"fma_t({U(f)}, {b(sub(v, f, 1))}, {ns})"
        return _chain(e, [(U2(a), b(sub(v, a, 1))) for a in range(3) if a != f and v[a] > 0])
    ii = 1.0 / v[0]
    e = f"fma_t({lit(-(1.0 - ii))}, {b(sub(v, 0, 2))}, -({b(sub(v, 1, 2))} + {b(sub(v, 2, 2))}))"
    e = _chain(e, [("uy2", b(sub(v, 1, 1))), ("uz2", b(sub(v, 2, 1)))])
    return f"fma_t({axis(0, v[0])}{b(sub(v, 0, 1))}, {e})"


def gen_coulomb_scaled(nt, hoisted=True):
    """hoisted: the (2 - 1/i) u_a products formed once per pair (the FP32 kernels); else
    the literal multiplies in place (the FP64 kernels, which hold more registers)."""
    mi = shell_index(nt)
    head = ["  const T rinv = rsqrt_t(rs);",
            "  const T ux = dx * rinv, uy = dy * rinv, uz = dz * rinv;",
            "  const T ux2 = ux + ux, uy2 = uy + uy, uz2 = uz + uz;",
            "  const T eta = h * rinv;",
            "  const T E = T(1);",
            "  T q = rinv, S;"]
    hs = Hoisted() if hoisted else None
    L = []
    sh = ShellSum(L, mi)
    for v in shells(nt - 1):
        if v != (0, 0, 0):
            L.append(f"  const T {name('B', v)} = {coul_scaled_expr(v, hs)};")
        sh.add(v, "E" if v == (0, 0, 0) else name("B", v))
    sh.done()
    return head + (hs.place(L) if hs else L)


def scr_scaled_expr(v):
    A = lambda w: "E" if w == (0, 0, 0) else name("A", w)
    C = lambda w: "E" if w == (0, 0, 0) else name("C", w)
    U = lambda a: "u" + AX[a]
    U2 = lambda a: "u" + AX[a] + "2"
    K = lambda a: "ku" + AX[a]
    nz, n1, ax = classify(v)
    if nz == 2 and n1 == 1:
        u = ax[0]
        return f"{K(u)}*E", f"{U(u)}*E1"
    if n1 == 0:
        u = ax[0]
        i = v[u]
        cf1, cf2, cf3 = 1.0 / i, 1.0 - 1.0 / (2.0 * i), 1.0 - 1.0 / i
        cexp = f"{lit(cf1)}*fma_t({K(u)}, {A(sub(v, u, 1))}, -(rho*{A(sub(v, u, 2))}))"
        ns = _neg_sum([A(sub(v, a, 2)) for a in ax[1:]])
        e = f"{lit(-cf3)}*{A(sub(v, u, 2))}" if ns is None else f"fma_t({lit(-cf3)}, {A(sub(v, u, 2))}, {ns})"
        e = _chain(e, [(U2(a), A(sub(v, a, 1))) for a in ax[1:]])
        e = f"fma_t({U(u)}, {lit(2.0 * cf2)}*{A(sub(v, u, 1))}, {e})"
        e = f"fma_t({lit(cf1)}, fma_t({K(u)}, {C(sub(v, u, 1))}, -(rho*{C(sub(v, u, 2))})), {e})"
        return cexp, e
    f = next(a for a in range(3) if v[a] == 1)
    cexp = f"{K(f)}*{A(sub(v, f, 1))}"
    ns = _neg_sum([A(sub(v, a, 2)) for a in range(3) if a != f and v[a] >= 2])
    e = f"{U(f)}*{A(sub(v, f, 1))}" if ns is None else f"fma_t({U(f)}, {A(sub(v, f, 1))}, {ns})"
    e = _chain(e, [(U2(a), A(sub(v, a, 1))) for a in range(3) if a != f and v[a] > 0])
    e = _chain(e, [(K(f), C(sub(v, f, 1)))])
    return cexp, e


class Hoisted:
    """Products of per-pair factors and literals, formed once per pair and placed where
    they are first needed."""

    def __init__(self):
        self.pre = {}
        self.order = []

    def hoist(self, nm, expr):
        if nm not in self.pre:
            self.pre[nm] = expr
            self.order.append(nm)
        return nm

    def place(self, L):
        """L with the hoisted products placed: one used in a single statement is written
        into it (a multiply either way), the others are defined just before their first
        use, so that none holds a register longer than it must."""
        import re
        word = lambda nm: re.compile(r"\b" + re.escape(nm) + r"\b")
        pre = dict(self.pre)
        while True:
            uses = {nm: sum(1 for ln in L + [pre[o] for o in pre if o != nm] if word(nm).search(ln))
                    for nm in pre}
            once = [nm for nm in reversed(self.order) if nm in pre and uses[nm] <= 1]
            if not once:
                break
            nm = once[0]
            rx = word(nm)
            L = [rx.sub(f"({pre[nm]})", ln) for ln in L]
            for o in pre:
                if o != nm:
                    pre[o] = rx.sub(f"({pre[nm]})", pre[o])
            del pre[nm]
        out, done = [], set()

        def define(nm):
            for o in self.order:
                if o in pre and o not in done and o != nm and word(o).search(pre[nm]):
                    define(o)
            out.append(f"  const T {nm} = {pre[nm]};")
            done.add(nm)

        for ln in L:
            for nm in self.order:
                if nm in pre and nm not in done and word(nm).search(ln):
                    define(nm)
            out.append(ln)
        return out

    def uc(self, a, i):
        return self.hoist(f"uc{AX[a]}_{i}", f"{lit(2.0 - 1.0 / i)}*u{AX[a]}")


class ScreenedScaled(Hoisted):
    """The scaled screened recurrence with its per-pair products hoisted.

    Every pattern of the recurrence is a sum of (factor, coefficient) products whose
    factors are u_a, 2 u_a, kappa-scaled u (ku_a = rho u_a), rho, and literals 1/i,
    2 - 1/i, 1 - 1/i.  Products of a pair factor and a literal (e.g. (1/i) ku_a, the
    (2 - 1/i) u_a of the axis term) are formed once per pair ("hoisted"), so each term
    of a pattern costs one fma.  A coefficient c~_w that is a single product ku_g a~_{w-g}
    (w has a component equal to 1; g the first such axis) is never formed: its consumers
    take ku_f ku_g (or (1/i) ku_f ku_g, (1/i) rho ku_g) times a~_{w-g} instead.  At
    nterms 9 this takes the pair from 886 fma + 447 mul to about 1,100 operations."""

    @staticmethod
    def A(w):
        return "E" if w == (0, 0, 0) else name("A", w)

    @staticmethod
    def lazy(w):
        """(g, w - g) where c~_w = ku_g a~_{w-g} is left unformed, else None."""
        if w == (0, 0, 0):
            return None
        nz, n1, ax = classify(w)
        if n1 == 0:
            return None
        g = next(a for a in range(3) if w[a] == 1)
        return g, sub(w, g, 1)

    def kk(self, a, b):
        a, b = min(a, b), max(a, b)
        return self.hoist(f"kk{AX[a]}{AX[b]}", f"ku{AX[a]}*ku{AX[b]}")

    def kc(self, a, i):
        return self.hoist(f"kc{AX[a]}_{i}", f"{lit(1.0 / i)}*ku{AX[a]}")

    def rc(self, i):
        return self.hoist(f"rc_{i}", f"{lit(1.0 / i)}*rho")


    def cterm(self, mult, w):
        """(factor, coefficient) of `mult` * c~_w; mult is ("k", a) for ku_a,
        ("kc", a, i) for (1/i) ku_a, or ("rc", i) for (1/i) rho."""
        lz = self.lazy(w)
        if lz is None:
            var = "E" if w == (0, 0, 0) else name("C", w)
            if mult[0] == "k":
                return f"ku{AX[mult[1]]}", var
            if mult[0] == "kc":
                return self.kc(mult[1], mult[2]), var
            return self.rc(mult[1]), var
        g, x = lz
        if mult[0] == "k":
            return self.kk(mult[1], g), self.A(x)
        if mult[0] == "kc":
            a, i = mult[1], mult[2]
            kc = self.kc(a, i)
            return self.hoist(f"kkc{AX[a]}{AX[g]}_{i}", f"{kc}*ku{AX[g]}"), self.A(x)
        i = mult[1]
        rc = self.rc(i)
        return self.hoist(f"rck{AX[g]}_{i}", f"{rc}*ku{AX[g]}"), self.A(x)

    def pattern(self, v):
        """(c~_v expression or None when it stays unformed, a~_v expression)."""
        A, U, U2 = self.A, (lambda a: "u" + AX[a]), (lambda a: "u" + AX[a] + "2")
        nz, n1, ax = classify(v)
        if nz == 2 and n1 == 1:
            return None, f"{U(ax[0])}*E1"
        if n1 == 0:
            u = ax[0]
            i = v[u]
            cexp = f"fma_t({self.kc(u, i)}, {A(sub(v, u, 1))}, -({self.rc(i)}*{A(sub(v, u, 2))}))"
            ns = _neg_sum([A(sub(v, a, 2)) for a in ax[1:]])
            rm, rv = self.cterm(("rc", i), sub(v, u, 2))
            km, kv = self.cterm(("kc", u, i), sub(v, u, 1))
            terms = [(lit(-(1.0 - 1.0 / i)), A(sub(v, u, 2))), (f"-{rm}", rv)]
            terms += [(U2(a), A(sub(v, a, 1))) for a in ax[1:]]
            terms += [(self.uc(u, i), A(sub(v, u, 1))), (km, kv)]
            return cexp, _chain(ns, terms)
        f = next(a for a in range(3) if v[a] == 1)
        ns = _neg_sum([A(sub(v, a, 2)) for a in range(3) if a != f and v[a] >= 2])
        terms = [(U(f), A(sub(v, f, 1)))]
        terms += [(U2(a), A(sub(v, a, 1))) for a in range(3) if a != f and v[a] > 0]
        terms.append(self.cterm(("k", f), sub(v, f, 1)))
        return None, _chain(ns, terms)


def gen_screened_scaled_plain(nt):
    """The scaled screened recurrence pattern by pattern, each c~ and a~ formed as the
    reference's recurrence writes it (the FP64 kernels: with the hoisted form's extra live
    products the FP64 variant spilled and ran no faster)."""
    mi = shell_index(nt)
    L = ["  const T rinv = rsqrt_t(dist2);",
         "  const T ux = dx * rinv, uy = dy * rinv, uz = dz * rinv;",
         "  const T ux2 = ux + ux, uy2 = uy + uy, uz2 = uz + uz;",
         "  const T rho = kappa * (dist2 * rinv);",
         "  const T kux = rho * ux, kuy = rho * uy, kuz = rho * uz;",
         "  const T eta = h * rinv;",
         "  const T E = exp_t(-rho);",
         "  const T E1 = fma_t(rho, E, E);",
         "  T q = rinv, S;"]
    sh = ShellSum(L, mi)
    for v in shells(nt - 1):
        if v != (0, 0, 0):
            cexp, aexp = scr_scaled_expr(v)
            L.append(f"  const T {name('C', v)} = {cexp};")
            L.append(f"  const T {name('A', v)} = {aexp};")
        sh.add(v, "E" if v == (0, 0, 0) else name("A", v))
    sh.done()
    return L


def gen_screened_scaled(nt):
    """The scaled screened recurrence with hoisted products (ScreenedScaled): the FP32
    kernels."""
    mi = shell_index(nt)
    head = ["  const T rinv = rsqrt_t(dist2);",
            "  const T ux = dx * rinv, uy = dy * rinv, uz = dz * rinv;",
            "  const T ux2 = ux + ux, uy2 = uy + uy, uz2 = uz + uz;",
            "  const T rho = kappa * (dist2 * rinv);",
            "  const T kux = rho * ux, kuy = rho * uy, kuz = rho * uz;",
            "  const T eta = h * rinv;",
            "  const T E = exp_t(-rho);",
            "  const T E1 = fma_t(rho, E, E);",
            "  T q = rinv, S;"]
    g = ScreenedScaled()
    L = []
    sh = ShellSum(L, mi)
    for v in shells(nt - 1):
        if v != (0, 0, 0):
            cexp, aexp = g.pattern(v)
            if cexp is not None:
                L.append(f"  const T {name('C', v)} = {cexp};")
            L.append(f"  const T {name('A', v)} = {aexp};")
        sh.add(v, "E" if v == (0, 0, 0) else name("A", v))
    sh.done()
    return head + g.place(L)


# ---------------------------------------------------------------------------- force
def force_expr(v):
    b = lambda w: name("b", w)
    d = lambda a: "d" + AX[a]
    nz, n1, ax = classify(v)
    deg = sum(v)
    if nz == 3:
        return "sqfac"
    if nz == 2:
        u, k = ax[0], v[ax[0]]
        if k == 1:
            return f"-fac*{d(u)}*sqfac"
        ik = 1.0 / k
        return f"fac*({lit(ik - 2.0)}*{b(sub(v, u, 1))}*{d(u)} + {lit(ik - 1.0)}*{b(sub(v, u, 2))})"
    if nz == 1 and n1 == 2:
        u, w = ax
        return f"{lit(-1.5)}*fac*({d(u)}*{b(sub(v, u, 1))} + {d(w)}*{b(sub(v, w, 1))})"
    if nz == 1 and n1 == 1:
        u, w = ax
        k = deg - 1
        g = u if v[u] >= 2 else w
        return (f"(fac*{lit(1.0 / (k + 1))})*({lit(-2 * k - 1.0)}*({d(u)}*{b(sub(v, u, 1))} + "
                f"{d(w)}*{b(sub(v, w, 1))}) + {lit(-k)}*{b(sub(v, g, 2))})")
    if nz == 1:
        u, w = ax
        s = v[u] + v[w]
        return (f"(fac*{lit(1.0 / s)})*({lit(1 - 2 * s)}*({d(u)}*{b(sub(v, u, 1))} + "
                f"{d(w)}*{b(sub(v, w, 1))}) + {lit(1 - s)}*({b(sub(v, u, 2))} + {b(sub(v, w, 2))}))")
    s3 = f"(dx*{b(sub(v, 0, 1))} + dy*{b(sub(v, 1, 1))} + dz*{b(sub(v, 2, 1))})"
    if n1 == 3:
        return f"(fac*{lit(-5.0 / 3.0)})*{s3}"
    if n1 == 2:
        w = next(a for a in range(3) if v[a] >= 2)
        i = v[w]
        return f"(fac*{lit(1.0 / (2.0 + i))})*({lit(-3.0 - 2 * i)}*{s3} + {lit(-1.0 - i)}*{b(sub(v, w, 2))})"
    if n1 == 1:
        f = next(a for a in range(3) if v[a] == 1)
        u, w = [a for a in range(3) if a != f]
        s = v[u] + v[w]
        return (f"(fac*{lit(1.0 / (1 + s))})*({lit(-1.0 - 2 * s)}*{s3} + {lit(-s)}*"
                f"({b(sub(v, u, 2))} + {b(sub(v, w, 2))}))")
    s = deg
    return (f"(fac*{lit(1.0 / s)})*({lit(1 - 2 * s)}*{s3} + {lit(1 - s)}*({b(sub(v, 0, 2))} + "
            f"{b(sub(v, 1, 2))} + {b(sub(v, 2, 2))}))")


def gen_force(nt):
    """Field sum of treetaylorforce: returns (fx, fy, fz) through references."""
    mi = shell_index(nt)
    L = ["  const T fac = T(1) / rs;",
         "  const T sqfac = sqrt_t(fac);",
         "  T sx = T(0), sy = T(0), sz = T(0);"]
    # coefficient (i,j,k) of degree d is consumed by moments of degree d-1
    for v in shells(nt):
        L.append(f"  const T {name('b', v)} = {force_expr(v)};")
        d = sum(v)
        if d == 0:
            continue
        for a, acc in ((0, "sx"), (1, "sy"), (2, "sz")):
            if v[a] == 0:
                continue
            m = sub(v, a, 1)  # moment index (i, k, m) with this coefficient on axis a
            if sum(m) >= nt:
                continue
            sign = 1.0 if (sum(m) + 1) % 2 == 0 else -1.0
            coef = sign * (m[a] + 1)
            L.append(f"  {acc} = fma_t(M[{mi[m]}] * {lit(coef)}, {name('b', v)}, {acc});")
    L.append("  fx += sx; fy += sy; fz += sz;")
    return L


def gen_screened_curl(nt):
    """Field sum of shielded_treetaylorforce (src/tree3d.cpp:2745-2973): the screened
    coefficients a_v of shielded_treetaylorpot's recurrence (the same index patterns and
    formulas, :2796-2938) to degree nterms, then fx -= (j+1) M_ijk a_(i,j+1,k) and
    fy += (i+1) M_ijk a_(i+1,j,k) (:2946-2958); the reference sets fz = 0."""
    mi = shell_index(nt)
    L = ["  const T dx2 = T(2)*dx, dy2 = T(2)*dy, dz2 = T(2)*dz;",
         "  const T kdx = kappa*dx, kdy = kappa*dy, kdz = kappa*dz;",
         "  const T rinv = rsqrt_t(dist2);",
         "  const T fac = rinv * rinv;",
         "  const T c0_0_0 = exp_t(-kappa * (dist2 * rinv));",
         "  const T a0_0_0 = c0_0_0 * rinv;",
         "  T sx = T(0), sy = T(0);"]
    for v in shells(nt):
        if v != (0, 0, 0):
            bexp, aexp = scr_expr(v)
            L.append(f"  const T {name('c', v)} = {bexp};")
            L.append(f"  const T {name('a', v)} = {aexp};")
        if v[1] >= 1:
            m = sub(v, 1, 1)
            if sum(m) < nt:
                L.append(f"  sx = fma_t(M[{mi[m]}] * {lit(-(m[1] + 1))}, {name('a', v)}, sx);")
        if v[0] >= 1:
            m = sub(v, 0, 1)
            if sum(m) < nt:
                L.append(f"  sy = fma_t(M[{mi[m]}] * {lit(m[0] + 1)}, {name('a', v)}, sy);")
    L.append("  fx += sx; fy += sy;")
    return L


def korder_expr(v):
    """Correction of order l to the Taylor coefficient v of the regularised Coulomb field
    (treetaylorforce's KERNEL_ORDER loop, src/tree3d.cpp:614-791).  Every index pattern of
    that loop is the one recurrence for the coefficients of (r^2 + del)^-(l + 1/2):
    d_v = fac/s ((1 - 2l - 2s) sum_a x_a d_(v-e_a) + (1 - 2l - s) sum_a d_(v-2e_a)),
    s = |v| (e.g. :637-639 for s = 1, :667-669 for v = (1, 1, 0), :725-728 for v = (1, 1, 1))."""
    d = lambda w: name("d", w)
    s = sum(v)
    s1 = " + ".join(f"d{AX[a]}*{d(sub(v, a, 1))}" for a in range(3) if v[a] >= 1)
    s2 = [d(sub(v, a, 2)) for a in range(3) if v[a] >= 2]
    e = f"(T({float(1 - 2 * s)!r}) - T(2)*lf)*({s1})"
    if s2:
        e += f" + (T({float(1 - s)!r}) - T(2)*lf)*({' + '.join(s2)})"
    return f"(fac*{lit(1.0 / s)})*({e})"


def gen_force_korder(nt):
    """treetaylorforce with its KERNEL_ORDER loop (src/tree3d.cpp:456-810): the order-0
    coefficients of gen_force, then for l = 1..korder the correction recurrence seeded with
    choose(-1/2, l) (-del)^l / (r (r^2+del)^l) (:617-631), added into every coefficient;
    the field sum of :794-808 over the corrected coefficients."""
    mi = shell_index(nt)
    L = ["  const T fac = T(1) / rs;",
         "  const T sqfac = sqrt_t(fac);",
         "  const T r = sqrt_t(rs);"]
    for v in shells(nt):
        L.append(f"  T {name('b', v)} = {force_expr(v)};")
    L.append("  for (int l = 1; l <= korder; l++) {")
    L.append("    const T lf = T(l);")
    L.append("    T binom = T(1), fact = T(1);")
    L.append("    for (int j = 1; j <= l; j++) {")
    L.append("      binom = binom * (T(-0.5) - T(j) + T(1)) * (-del);")
    L.append("      fact = fact * T(j);")
    L.append("    }")
    L.append("    const T d0_0_0 = (binom / fact) * T(1) / (r * pow_t(rs, lf));")
    L.append("    b0_0_0 += d0_0_0;")
    for v in shells(nt):
        if v == (0, 0, 0):
            continue
        L.append(f"    const T {name('d', v)} = {korder_expr(v)};")
        L.append(f"    {name('b', v)} += {name('d', v)};")
    L.append("  }")
    L.append("  T sx = T(0), sy = T(0), sz = T(0);")
    for v in shells(nt):
        if sum(v) == 0:
            continue
        for a, acc in ((0, "sx"), (1, "sy"), (2, "sz")):
            if v[a] == 0:
                continue
            m = sub(v, a, 1)
            if sum(m) >= nt:
                continue
            sign = 1.0 if (sum(m) + 1) % 2 == 0 else -1.0
            L.append(f"  {acc} = fma_t(M[{mi[m]}] * {lit(sign * (m[a] + 1))}, {name('b', v)}, {acc});")
    L.append("  fx += sx; fy += sy; fz += sz;")
    return L


def count_flops(lines):
    """Floating-point operations of generated lines: every binary + - * /, 2 per fma_t,
    1 per sqrt_t / rsqrt_t / exp_t (literals and the moment loads are not arithmetic)."""
    import re
    n = 0
    for ln in lines:
        if "=" not in ln or "ld4(" in ln:
            continue
        e = re.sub(r"T\([^()]*\)", "C", ln.split("=", 1)[1])
        n += 2 * e.count("fma_t(") + e.count("sqrt_t(") + e.count("exp_t(")
        e = re.sub(r"[a-z_]+\(", "(", e)
        n += e.count("*") + e.count("/") + e.count("+")
        # binary minus: preceded by an operand (name, number, closing parenthesis)
        n += len(re.findall(r"[\w)]\s*-", e))
    return n


def flops_per_pair(nt):
    """Flops of one (target, cluster) far-field evaluation: the reference's recurrence to
    degree nterms-1 plus the moment dot product, as generated."""
    return {"coulomb": count_flops(gen_coulomb(nt)), "screened": count_flops(gen_screened(nt)),
            "force": count_flops(gen_force(nt))}


def main(out):
    parts = ["// GENERATED by gen_farfield.py -- do not edit.",
             "#pragma once",
             "namespace bit {",
             "template <int NT> struct FarField;"]
    for nt in range(1, 11):
        canon = moment_index(nt)
        order = list(shells(nt - 1))
        table = [canon[v] for v in order] + [0] * (padded(len(order)) - len(order))
        parts.append(f"__constant__ unsigned short kShellCanon{nt}[{len(table)}] = {{"
                     + ", ".join(map(str, table)) + "};")
        parts.append(f"template <> struct FarField<{nt}> {{")
        parts.append(f"  static constexpr int kPadded = {len(table)};")
        parts.append("  // canonical (i outer, j, k inner) index of the k-th moment in shell order")
        parts.append(f"  static __device__ __forceinline__ int canon(int k) {{ return kShellCanon{nt}[k]; }}")
        parts.append("  template <class T> static __device__ __forceinline__ T coulomb("
                     "T dx, T dy, T dz, T rs, const T* __restrict__ M) {")
        parts += gen_coulomb(nt)
        parts.append("  }")
        parts.append("  template <class T> static __device__ __forceinline__ T screened("
                     "T dx, T dy, T dz, T dist2, T kappa, const T* __restrict__ M) {")
        parts += gen_screened(nt)
        parts.append("  }")
        parts.append("  // scaled forms for normalised moments (M_v / h^|v|), used by the FP32 path")
        parts.append("  template <class T> static __device__ __forceinline__ T coulomb_s("
                     "T dx, T dy, T dz, T rs, T h, const T* __restrict__ M) {")
        parts += gen_coulomb_scaled(nt)
        parts.append("  }")
        parts.append("  template <class T> static __device__ __forceinline__ T coulomb_sp("
                     "T dx, T dy, T dz, T rs, T h, const T* __restrict__ M) {")
        parts += gen_coulomb_scaled(nt, hoisted=False)
        parts.append("  }")
        parts.append("  template <class T> static __device__ __forceinline__ T screened_s("
                     "T dx, T dy, T dz, T dist2, T kappa, T h, const T* __restrict__ M) {")
        parts += gen_screened_scaled(nt)
        parts.append("  }")
        parts.append("  template <class T> static __device__ __forceinline__ T screened_sp("
                     "T dx, T dy, T dz, T dist2, T kappa, T h, const T* __restrict__ M) {")
        parts += gen_screened_scaled_plain(nt)
        parts.append("  }")
        parts.append("  template <class T> static __device__ __forceinline__ void force("
                     "T dx, T dy, T dz, T rs, const T* __restrict__ M, T& fx, T& fy, T& fz) {")
        parts += gen_force(nt)
        parts.append("  }")
        parts.append("  template <class T> static __device__ __forceinline__ void force_korder("
                     "T dx, T dy, T dz, T rs, T del, int korder, const T* __restrict__ M, "
                     "T& fx, T& fy, T& fz) {")
        parts += gen_force_korder(nt)
        parts.append("  }")
        parts.append("  template <class T> static __device__ __forceinline__ void screened_curl("
                     "T dx, T dy, T dz, T dist2, T kappa, const T* __restrict__ M, T& fx, T& fy) {")
        parts += gen_screened_curl(nt)
        parts.append("  }")
        parts.append("};")
    parts.append("}  // namespace bit")
    with open(out, "w") as f:
        f.write("\n".join(parts) + "\n")


if __name__ == "__main__":
    main(sys.argv[1])

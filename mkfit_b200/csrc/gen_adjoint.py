"""Generates generated_adjoint.cuh: the forward step and its reverse-mode
adjoint for the barrel Kalman fit step (propagation to the hit radius with
the iterative helix and its Jacobian, material effects, covariance
transport, Kalman update and chi2), as explicit straight-line code.

The step is written once below against a small expression tracer (the same
arithmetic, in the same order, as kalman.cuh, which restates
helixAtRFromIterativeCCS_impl, applyMaterialEffects, propagateHelixToRMPlex
and kalmanOperation of the reference). The tracer folds constants (the
known-zero Jacobian entries vanish), shares common subexpressions, and the
emitter writes

  * the forward sweep (SSA, one statement per operation), and
  * the reverse sweep: adjoints accumulated in reverse statement order, one
    rule per operation (sum, product, quotient, sqrt, log, sin/cos, |x|,
    max, select); branches of the forward code are selects whose adjoint
    flows into the taken operand; table lookups (material grid) are opaque
    with zero derivative.

Both are C++ templates over the arithmetic type: float in the CUDA kernels,
double on the host for checking the derivation against finite differences.

    python gen_adjoint.py      # rewrites generated_adjoint.cuh
"""
import os

HERE = os.path.dirname(os.path.abspath(__file__))


# ----------------------------------------------------------------------------- tracer
class Node:
    __slots__ = ("op", "args", "val", "id", "is_bool", "name")

    def __init__(self, op, args, val=None, is_bool=False, name=None):
        self.op, self.args, self.val, self.is_bool, self.name = op, args, val, is_bool, name
        self.id = None

    # arithmetic
    def __add__(self, o): return G.add(self, o)
    def __radd__(self, o): return G.add(o, self)
    def __sub__(self, o): return G.sub(self, o)
    def __rsub__(self, o): return G.sub(o, self)
    def __mul__(self, o): return G.mul(self, o)
    def __rmul__(self, o): return G.mul(o, self)
    def __truediv__(self, o): return G.div(self, o)
    def __rtruediv__(self, o): return G.div(o, self)
    def __neg__(self): return G.sub(0.0, self)
    # comparisons (boolean nodes, no derivative)
    def __lt__(self, o): return G.cmp("<", self, o)
    def __gt__(self, o): return G.cmp(">", self, o)
    def __le__(self, o): return G.cmp("<=", self, o)
    def __ge__(self, o): return G.cmp(">=", self, o)


class Graph:
    def __init__(self):
        self.nodes = []
        self.memo = {}
        self.consts = {}

    def _add(self, n):
        n.id = len(self.nodes)
        self.nodes.append(n)
        return n

    def const(self, v):
        v = float(v)
        if v not in self.consts:
            self.consts[v] = self._add(Node("const", (), val=v))
        return self.consts[v]

    def lift(self, x):
        return x if isinstance(x, Node) else self.const(x)

    def inp(self, name, diff=True):
        return self._add(Node("in" if diff else "in_nd", (), name=name))

    def op(self, op, *args, is_bool=False):
        args = tuple(self.lift(a) for a in args)
        key = (op,) + tuple(a.id for a in args)
        if key in self.memo:
            return self.memo[key]
        n = self._add(Node(op, args, is_bool=is_bool))
        self.memo[key] = n
        return n

    @staticmethod
    def cv(n):
        return n.val if n.op == "const" else None

    def add(self, a, b):
        a, b = self.lift(a), self.lift(b)
        if self.cv(a) == 0.0: return b
        if self.cv(b) == 0.0: return a
        if self.cv(a) is not None and self.cv(b) is not None: return self.const(a.val + b.val)
        return self.op("add", a, b)

    def sub(self, a, b):
        a, b = self.lift(a), self.lift(b)
        if self.cv(b) == 0.0: return a
        if self.cv(a) is not None and self.cv(b) is not None: return self.const(a.val - b.val)
        if self.cv(a) == 0.0: return self.op("neg", b)
        return self.op("sub", a, b)

    def mul(self, a, b):
        a, b = self.lift(a), self.lift(b)
        if self.cv(a) == 0.0 or self.cv(b) == 0.0: return self.const(0.0)
        if self.cv(a) == 1.0: return b
        if self.cv(b) == 1.0: return a
        if self.cv(a) is not None and self.cv(b) is not None: return self.const(a.val * b.val)
        return self.op("mul", a, b)

    def div(self, a, b):
        a, b = self.lift(a), self.lift(b)
        if self.cv(a) == 0.0: return self.const(0.0)
        if self.cv(b) == 1.0: return a
        return self.op("div", a, b)

    def cmp(self, rel, a, b):
        return self.op("cmp" + rel, a, b, is_bool=True)

    def land(self, a, b): return self.op("and", a, b, is_bool=True)
    def lor(self, a, b): return self.op("or", a, b, is_bool=True)

    def select(self, c, a, b):
        a, b = self.lift(a), self.lift(b)
        if a is b: return a
        return self.op("select", c, a, b)

    def sqrt(self, a): return self.op("sqrt", a)
    def log(self, a): return self.op("log", a)
    def sin(self, a): return self.op("sin", a)
    def cos(self, a): return self.op("cos", a)
    def abs(self, a): return self.op("abs", a)
    def max(self, a, b): return self.op("max", a, b)

    def opaque(self, fn, nout, *args):
        """Call fn(args..., out0, out1, ...) with zero derivative."""
        call = self.op("call:" + fn, *args)
        return [self.op("out%d" % i, call) for i in range(nout)]


G = Graph()


# ----------------------------------------------------------------------------- model
def sidx(i, j):
    return i * (i + 1) // 2 + j if i >= j else j * (j + 1) // 2 + i


PI = 3.14159265358979323846
TWO_PI = 6.28318530717958647692


def squash_phi(phi):
    phi = G.select(phi >= PI, phi - TWO_PI, phi)
    return G.select(phi < -PI, phi + TWO_PI, phi)


def sincos4(x):
    x2 = x * x
    c = 1.0 - 0.5 * x2 + 0.04166667 * x2 * x2
    s = x - 0.16666667 * x * x2
    return s, c


def hipo(x, y):
    return G.sqrt(x * x + y * y)


def helix_to_r(inp, k, r, niter=5):
    """helixAtRFromIterativeCCS_impl (mkFit/PropagationMPlex.icc:5-246);
    same statement order as kalman.cuh helix_to_r."""
    J = [G.const(0.0)] * 36
    r0 = hipo(inp[0], inp[1])
    xin, yin, ipt, phiin, theta = inp[0], inp[1], inp[3], inp[4], inp[5]
    kinv = 1.0 / k
    pt = 1.0 / ipt
    D = G.const(0.0)
    cosP, sinP = G.cos(phiin), G.sin(phiin)
    pxin = cosP * pt
    pyin = sinP * pt
    dDdx = G.select(r0 > 0.0, -xin / r0, 0.0)
    dDdy = G.select(r0 > 0.0, -yin / r0, 0.0)
    dDdipt = G.const(0.0)
    dDdphi = G.const(0.0)
    ox, oy = inp[0], inp[1]
    fail = None
    sinah = cosah = cosa = sina = None
    for it in range(niter):
        r0 = hipo(ox, oy)
        oodotp = r0 * pt / (pxin * ox + pyin * oy)
        bad = G.lor(oodotp > 5.0, oodotp < 0.0)
        fail = bad if fail is None else G.lor(fail, bad)
        idd = G.select(bad, 0.0, (r - r0) * oodotp)
        D = D + idd
        sinah, cosah = sincos4(idd * ipt * kinv * 0.5)
        cosa = 1.0 - 2.0 * sinah * sinah
        sina = 2.0 * sinah * cosah
        if it + 1 != niter:
            x, y = ox, oy
            near = G.land(r0 > 0.0, G.abs(r - r0) < 0.0001)
            oor0 = G.select(near, 1.0 / r0, 0.0)
            dadipt = idd * kinv
            dadx = -x * ipt * kinv * oor0
            dady = -y * ipt * kinv * oor0
            pxca = pxin * cosa
            pxsa = pxin * sina
            pyca = pyin * cosa
            pysa = pyin * sina
            tmp = k * dadx
            dDdx = dDdx - (x * (1.0 + tmp * (pxca - pysa)) + y * tmp * (pyca + pxsa)) * oor0
            tmp = k * dady
            dDdy = dDdy - (x * tmp * (pxca - pysa) + y * (1.0 + tmp * (pyca + pxsa))) * oor0
            tmp = dadipt * ipt
            dDdipt = dDdipt - k * (x * (pxca * tmp - pysa * tmp - pyca - pxsa + pyin) +
                                   y * (pyca * tmp + pxsa * tmp - pysa + pxca - pxin)) * pt * oor0
            dDdphi = dDdphi + k * (x * (pysa - pxin + pxca) - y * (pxsa - pyin + pyca)) * oor0
        ox = ox + 2.0 * k * sinah * (pxin * cosah - pyin * sinah)
        oy = oy + 2.0 * k * sinah * (pyin * cosah + pxin * sinah)
        pxold = pxin
        pxin = pxin * cosa - pyin * sina
        pyin = pyin * cosa + pxold * sina
    alpha = D * ipt * kinv
    dadx = dDdx * ipt * kinv
    dady = dDdy * ipt * kinv
    dadipt = (ipt * dDdipt + D) * kinv
    dadphi = dDdphi * ipt * kinv
    sina, cosa = sincos4(alpha)
    J[0] = 1.0 + k * dadx * (cosP * cosa - sinP * sina) * pt
    J[1] = k * dady * (cosP * cosa - sinP * sina) * pt
    J[3] = k * (cosP * (ipt * dadipt * cosa - sina) + sinP * ((1.0 - cosa) - ipt * dadipt * sina)) * pt * pt
    J[4] = k * (cosP * dadphi * cosa - sinP * dadphi * sina - sinP * sina + cosP * cosa - cosP) * pt
    J[6] = k * dadx * (sinP * cosa + cosP * sina) * pt
    J[7] = 1.0 + k * dady * (sinP * cosa + cosP * sina) * pt
    J[9] = k * (sinP * (ipt * dadipt * cosa - sina) + cosP * (ipt * dadipt * sina - (1.0 - cosa))) * pt * pt
    J[10] = k * (sinP * dadphi * cosa + cosP * dadphi * sina + sinP * cosa + cosP * sina - sinP) * pt
    cosT, sinT = G.cos(theta), G.sin(theta)
    isinT = 1.0 / sinT
    out = [ox, oy, inp[2] + k * alpha * cosT * pt * isinT, ipt, inp[4] + alpha, theta]
    J[12] = k * cosT * dadx * pt * isinT
    J[13] = k * cosT * dady * pt * isinT
    J[14] = G.const(1.0)
    J[15] = k * cosT * (ipt * dadipt - alpha) * pt * pt * isinT
    J[16] = k * dadphi * cosT * pt * isinT
    J[17] = -k * alpha * pt * isinT * isinT
    J[21] = G.const(1.0)
    J[24] = dadx
    J[25] = dady
    J[27] = dadipt
    J[28] = 1.0 + dadphi
    J[35] = G.const(1.0)
    return out, J, fail


def material_effects(radL, xi, sign, C, par):
    """applyMaterialEffects (mkFit/PropagationMPlex.cc:716-767), barrel."""
    C, par = list(C), list(par)
    theta = par[5]
    pt = 1.0 / par[3]
    p = pt / G.sin(theta)
    p2 = p * p
    mpi = 0.140
    mpi2 = mpi * mpi
    beta2 = p2 / (p2 + mpi2)
    beta = G.sqrt(beta2)
    invCos = p / pt
    radL2 = radL * invCos
    ok = G.land(radL >= 1e-13, radL2 >= 1e-13)
    # The log's argument is kept positive on the skipped branch so that its
    # adjoint stays finite there (the branch value is discarded).
    tms = 0.0136 * (1.0 + 0.038 * G.log(G.select(ok, radL2, 1.0))) / (beta * p)
    tms2 = tms * tms * radL2
    gamma2 = (p2 + mpi2) / mpi2
    gamma = G.sqrt(gamma2)
    me = 0.0005
    wmax = 2.0 * me * beta2 * gamma2 / (1.0 + 2.0 * gamma * me / mpi + me * me / (mpi * mpi))
    I = 16.0e-9 * 10.75
    import math
    dh0 = math.log(28.816e-9 * math.sqrt(2.33 * 0.498) / I)
    deltahalf = dh0 + G.log(beta * gamma) - 0.5
    dEdx = G.select(beta < 1.0,
                    2.0 * (xi * invCos * (0.5 * G.log(2.0 * me * beta2 * gamma2 * wmax / (I * I)) -
                                          beta2 - deltahalf) / beta2), 0.0)
    dP = sign * dEdx / beta
    new_ipt = p / (G.max(p + dP, 0.001) * pt)
    C[14] = G.select(ok, C[14] + tms2, C[14])
    C[20] = G.select(ok, C[20] + tms2, C[20])
    C[9] = G.select(ok, C[9] + dP * dP / (p2 * pt * pt), C[9])
    par[3] = G.select(ok, new_ipt, par[3])
    return C, par


def similarity(J, C):
    """J C J^T on the packed symmetric C (MultHelixProp + Transp)."""
    T = [[None] * 6 for _ in range(6)]
    for i in range(6):
        for j in range(6):
            s = G.const(0.0)
            for kk in range(6):
                s = s + J[i * 6 + kk] * C[sidx(kk, j)]
            T[i][j] = s
    out = [None] * 21
    for i in range(6):
        for j in range(i + 1):
            s = G.const(0.0)
            for kk in range(6):
                s = s + T[i][kk] * J[j * 6 + kk]
            out[sidx(i, j)] = s
    return out


def kalman_barrel(par, err, mpos, merr):
    """kalmanOperation (mkFit/KalmanUtilsMPlex.cc:548-681), chi2 + update;
    same formulas as kalman.cuh kalman_barrel."""
    r = hipo(mpos[0], mpos[1])
    r00 = -(mpos[1] + par[1]) / (2.0 * r)
    r01 = (mpos[0] + par[0]) / (2.0 * r)
    res0, res1, res2 = mpos[0] - par[0], mpos[1] - par[1], mpos[2] - par[2]
    g = [err[i] + merr[i] for i in range(6)]
    loc0 = r00 * res0 + r01 * res1
    loc1 = res2
    t0 = r00 * g[0] + r01 * g[1]
    t1 = r00 * g[1] + r01 * g[2]
    s0 = t0 * r00 + t1 * r01
    s1 = g[3] * r00 + g[4] * r01
    s2 = g[5]
    det = s0 * s2 - s1 * s1
    sdet = 1.0 / det
    i0, i1, i2 = sdet * s2, -(s1 * sdet), sdet * s0
    chi2 = i0 * loc0 * loc0 + i2 * loc1 * loc1 + 2.0 * (i1 * loc1 * loc0)
    h00, h01, h10, h11, h20, h21 = r00 * i0, r00 * i1, r01 * i0, r01 * i1, i1, i2
    K = []
    for i in range(6):
        c0, c1, c2 = err[sidx(i, 0)], err[sidx(i, 1)], err[sidx(i, 2)]
        K.append((c0 * h00 + c1 * h10 + c2 * h20, c0 * h01 + c1 * h11 + c2 * h21))
    opar = [par[i] + K[i][0] * loc0 + K[i][1] * loc1 for i in range(6)]
    opar[4] = squash_phi(opar[4])
    # (K H) C with H rows (r00, r01, 0 | 0, 0, 1): KH[i] = (K0 r00, K0 r01, K1, 0, 0, 0).
    oerr = [None] * 21
    for i in range(6):
        kh = (K[i][0] * r00, K[i][0] * r01, K[i][1])
        for j in range(i + 1):
            s = kh[0] * err[sidx(0, j)] + kh[1] * err[sidx(1, j)] + kh[2] * err[sidx(2, j)]
            oerr[sidx(i, j)] = err[sidx(i, j)] - s
    return opar, oerr, chi2


def barrel_step(with_material):
    """One fit step on a barrel layer with alignment parameters:
    hit moved by a (r-phi, along the local tangent) and b (z); material
    (radiation length and xi) scaled by s."""
    global G
    G = Graph()
    par = [G.inp("par[%d]" % i) for i in range(6)]
    err = [G.inp("err[%d]" % i) for i in range(21)]
    mraw = [G.inp("mpos[%d]" % i, diff=False) for i in range(3)]
    merr = [G.inp("merr[%d]" % i, diff=False) for i in range(6)]
    a, b, s = G.inp("a"), G.inp("b"), G.inp("s")
    k = G.inp("k", diff=False)
    # Alignment: shift along (-y, x)/r in the transverse plane, and in z.
    rh = hipo(mraw[0], mraw[1])
    m = [mraw[0] + a * (-mraw[1] / rh), mraw[1] + a * (mraw[0] / rh), mraw[2] + b]
    r = hipo(m[0], m[1])
    p, J, fail = helix_to_r(par, k, r)
    C = list(err)
    if with_material:
        rl0, xi0 = G.opaque("mat_lookup", 2, p[2], r, fail)
        r_in = hipo(par[0], par[1])
        sign = G.select(r > r_in, 1.0, -1.0)
        C, p = material_effects(rl0 * s, xi0 * s, sign, C, p)
    p[4] = squash_phi(p[4])
    Co = similarity(J, C)
    pp = [G.select(fail, par[i], p[i]) for i in range(6)]
    pe = [G.select(fail, err[i], Co[i]) for i in range(21)]
    opar, oerr, chi2 = kalman_barrel(pp, pe, m, merr)
    inputs = par + err + [a, b, s]
    in_names = (["par[%d]" % i for i in range(6)] + ["err[%d]" % i for i in range(21)] +
                ["a", "b", "s"])
    outputs = opar + oerr + [chi2]
    out_names = (["opar[%d]" % i for i in range(6)] + ["oerr[%d]" % i for i in range(21)] +
                 ["chi2"])
    return G, inputs, in_names, outputs, out_names


# ----------------------------------------------------------------------------- emitter
def cnum(v):
    r = repr(float(v))
    if "e" not in r and "." not in r and "inf" not in r and "nan" not in r:
        r += ".0"
    return "T(%s)" % r


class Emitter:
    def __init__(self, g):
        self.g = g
        self.names = {}

    def ref(self, n):
        if n.op == "const":
            return cnum(n.val)
        return self.names[n.id]

    def live(self, outputs):
        seen = set()
        stack = list(outputs)
        while stack:
            n = stack.pop()
            if n.id in seen:
                continue
            seen.add(n.id)
            stack.extend(n.args)
        return sorted(seen)

    def forward(self, outputs, lines):
        order = self.live(outputs)
        calls = {}
        for i in order:
            n = self.g.nodes[i]
            if n.op == "const":
                continue
            if n.op in ("in", "in_nd"):
                self.names[i] = n.name
                continue
            v = "v%d" % i
            self.names[i] = v
            A = [self.ref(x) for x in n.args]
            op = n.op
            if op.startswith("call:"):
                calls[i] = op[5:]
                self.names[i] = "c%d" % i
                continue
            if op.startswith("out"):
                call = n.args[0]
                if not hasattr(self, "_done_calls"):
                    self._done_calls = set()
                if call.id not in self._done_calls:
                    self._done_calls.add(call.id)
                    outs = [x for x in order if self.g.nodes[x].op.startswith("out") and
                            self.g.nodes[x].args[0] is call]
                    for x in outs:
                        lines.append("  T v%d;" % x)
                    cargs = ", ".join([self.ref(a) for a in call.args] + ["v%d" % x for x in outs])
                    lines.append("  %s(mat, %s);" % (calls[call.id], cargs))
                continue
            if n.is_bool:
                rel = {"cmp<": "<", "cmp>": ">", "cmp<=": "<=", "cmp>=": ">=", "and": "&&",
                       "or": "||"}[op]
                lines.append("  const bool %s = %s %s %s;" % (v, A[0], rel, A[1]))
                continue
            expr = {
                "add": lambda: "%s + %s" % (A[0], A[1]),
                "sub": lambda: "%s - %s" % (A[0], A[1]),
                "mul": lambda: "%s * %s" % (A[0], A[1]),
                "div": lambda: "%s / %s" % (A[0], A[1]),
                "neg": lambda: "-%s" % A[0],
                "sqrt": lambda: "ad_sqrt(%s)" % A[0],
                "log": lambda: "ad_log(%s)" % A[0],
                "sin": lambda: "ad_sin(%s)" % A[0],
                "cos": lambda: "ad_cos(%s)" % A[0],
                "abs": lambda: "ad_abs(%s)" % A[0],
                "max": lambda: "ad_max(%s, %s)" % (A[0], A[1]),
                "select": lambda: "%s ? %s : %s" % (A[0], A[1], A[2]),
            }[op]()
            lines.append("  const T %s = %s;" % (v, expr))
        return order

    def reverse(self, order, outputs, out_bar_names, inputs, lines):
        gname = {}
        node = self.g.nodes

        def acc(n, expr):
            if n.op in ("const", "in_nd") or n.is_bool or n.op.startswith("out"):
                return
            if n.id in gname:
                lines.append("  %s += %s;" % (gname[n.id], expr))
            else:
                gname[n.id] = "g%d" % n.id
                lines.append("  T %s = %s;" % (gname[n.id], expr))

        for o, ob in zip(outputs, out_bar_names):
            acc(o, ob)
        for i in reversed(order):
            n = node[i]
            if i not in gname or n.op in ("in", "in_nd", "const") or n.is_bool:
                continue
            g = gname[i]
            A = n.args
            R = [self.ref(x) for x in A]
            op = n.op
            if op == "add":
                acc(A[0], g)
                acc(A[1], g)
            elif op == "sub":
                acc(A[0], g)
                acc(A[1], "-" + g)
            elif op == "neg":
                acc(A[0], "-" + g)
            elif op == "mul":
                if A[0] is A[1]:
                    acc(A[0], "T(2) * %s * %s" % (g, R[0]))
                else:
                    acc(A[0], "%s * %s" % (g, R[1]))
                    acc(A[1], "%s * %s" % (g, R[0]))
            elif op == "div":
                q = "q%d" % i
                lines.append("  const T %s = %s / %s;" % (q, g, R[1]))
                acc(A[0], q)
                acc(A[1], "-%s * %s" % (q, self.names[i]))
            elif op == "sqrt":
                acc(A[0], "T(0.5) * %s / %s" % (g, self.names[i]))
            elif op == "log":
                acc(A[0], "%s / %s" % (g, R[0]))
            elif op == "sin":
                acc(A[0], "%s * ad_cos(%s)" % (g, R[0]))
            elif op == "cos":
                acc(A[0], "-%s * ad_sin(%s)" % (g, R[0]))
            elif op == "abs":
                acc(A[0], "(%s >= T(0) ? %s : -%s)" % (R[0], g, g))
            elif op == "max":
                acc(A[0], "(%s >= %s ? %s : T(0))" % (R[0], R[1], g))
                acc(A[1], "(%s >= %s ? T(0) : %s)" % (R[0], R[1], g))
            elif op == "select":
                acc(A[1], "(%s ? %s : T(0))" % (R[0], g))
                acc(A[2], "(%s ? T(0) : %s)" % (R[0], g))
            else:
                raise ValueError(op)
        return gname


def emit_step(with_material, suffix):
    g, inputs, in_names, outputs, out_names = barrel_step(with_material)
    sig_in = ("const T (&par)[6], const T (&err)[21], const T (&mpos)[3], const T (&merr)[6], "
              "T a, T b, T s, T k, const MatT& mat")
    fwd = ["template <typename T, typename MatT>",
           "AD_FN void barrel_step_fwd%s(%s,\n    T (&opar)[6], T (&oerr)[21], T& chi2) {" % (suffix, sig_in)]
    fwd.append("  (void)mat; (void)a; (void)b; (void)s;")
    em = Emitter(g)
    em.forward(outputs, fwd)
    for o, name in zip(outputs, out_names):
        fwd.append("  %s = %s;" % (name, em.ref(o)))
    fwd.append("}")

    rev = ["template <typename T, typename MatT>",
           "AD_FN void barrel_step_rev%s(%s,\n    const T (&opar_bar)[6], const T (&oerr_bar)[21], T chi2_bar,\n"
           "    T (&par_bar)[6], T (&err_bar)[21], T& a_bar, T& b_bar, T& s_bar) {" % (suffix, sig_in)]
    rev.append("  (void)mat; (void)a; (void)b; (void)s;")
    em2 = Emitter(g)
    order = em2.forward(outputs, rev)
    bars = (["opar_bar[%d]" % i for i in range(6)] + ["oerr_bar[%d]" % i for i in range(21)] +
            ["chi2_bar"])
    gname = em2.reverse(order, outputs, bars, inputs, rev)
    for n, name in zip(inputs, in_names):
        bar = name.replace("par[", "par_bar[").replace("err[", "err_bar[")
        if name in ("a", "b", "s"):
            bar = name + "_bar"
        rev.append("  %s = %s;" % (bar, gname.get(n.id, "T(0)")))
    rev.append("}")
    n_ops = sum(1 for i in order if g.nodes[i].op not in ("const", "in", "in_nd"))
    return "\n".join(fwd), "\n".join(rev), n_ops


HEADER = """// GENERATED by gen_adjoint.py -- do not edit.
// Barrel Kalman fit step with alignment / material-scale parameters and its
// reverse-mode adjoint, as straight-line code templated on the arithmetic
// type (float on the device, double on the host).
//   forward : (par, err; hit, a, b, s) -> (par', err', chi2)
//   reverse : adjoints of (par', err', chi2) -> adjoints of (par, err, a, b, s)
// a: hit shift along the transverse tangent (r-phi), b: hit shift in z,
// s: scale of the material (radiation length and xi) at the layer.
// The reverse function recomputes the forward sweep it needs.
#pragma once

#ifndef AD_FN
#ifdef __CUDACC__
#define AD_FN __host__ __device__ __forceinline__
#else
#define AD_FN inline
#endif
#endif

namespace mkfg {
namespace adj {
"""

FOOTER = """
}  // namespace adj
}  // namespace mkfg
"""


def main():
    parts = [HEADER]
    stats = []
    for with_mat, suf in ((False, "_nomat"), (True, "_mat")):
        f, r, n = emit_step(with_mat, suf)
        parts += [f, "", r, ""]
        stats.append("// %s: %d forward operations" % (suf[1:], n))
    parts.insert(1, "\n".join(stats) + "\n")
    parts.append(FOOTER)
    out = os.path.join(HERE, "generated_adjoint.cuh")
    with open(out, "w") as fh:
        fh.write("\n".join(parts))
    print("wrote", out, "; ".join(stats))


if __name__ == "__main__":
    main()

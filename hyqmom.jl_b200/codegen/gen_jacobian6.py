"""Generate the closed form of jacobian6 (rows 3, 5, 6) from its definition.

jacobian6 (reference src/autogen/jacobian6.jl:14-59) is the Jacobian of the
x-fluxes of W = (m02, m12, m22, m03, m13, m04) of the 2-D HyQMOM closure,
m_ab = E[x^a y^b] with x the flux direction:
    flux(m02, m12, m22, m03, m13, m04) = (m12, m22, m32, m13, m23, m14)
where m32, m23, m14 are closed by the HyQMOM fifth-order formulas
(src/moments/hyqmom_3D.jl:156-178 restricted to two dimensions).  Rows 1, 2
and 4 are the unit rows e2, e3, e5.

Only the central moments C02, C12, C22, C03, C13, C04 depend on W, with
dC_ab/dm_pq = binom(a,p) binom(b,q) (-u)^(a-p) (-v)^(b-q) / m00.  This script
derives d{m32, m23, m14}/d{C02, C12, C22, C03, C13, C04} symbolically (the
standardised moments use sx = sqrt(C20), sy = sqrt(C02); every derivative is
rational in the C's), chains it with dC/dW, applies common-subexpression
elimination and writes one C++ function body.  The device code and the CPU
oracle include the same generated body, so both evaluate the same arithmetic
in the same order.

    python hyqmom.jl_b200/codegen/gen_jacobian6.py [outdir ...]

The body expects `R` (the scalar type), `m[15]` in jacobian6 argument order
(m00, m01, m02, m03, m04, m10, m11, m12, m13, m20, m21, m22, m30, m31, m40)
and writes `r3[6]`, `r5[6]`, `r6[6]` (rows 3, 5, 6, columns in W order).
"""
import os
import sys

import sympy as sp
from sympy.printing.c import C99CodePrinter

HERE = os.path.dirname(os.path.abspath(__file__))
OUTPUTS = [os.path.join(HERE, "..", "csrc", "gen_jacobian6.inc"),
           os.path.join(HERE, "..", "..", "oracle", "gen_jacobian6.inc")]

ARGS = [(0, 0), (0, 1), (0, 2), (0, 3), (0, 4), (1, 0), (1, 1), (1, 2), (1, 3), (2, 0), (2, 1), (2, 2), (3, 0), (3, 1), (4, 0)]
W = [(0, 2), (1, 2), (2, 2), (0, 3), (1, 3), (0, 4)]
CLIST = [(2, 0), (1, 1), (0, 2), (3, 0), (2, 1), (1, 2), (0, 3), (4, 0), (3, 1), (2, 2), (1, 3), (0, 4)]
C = {ab: sp.Symbol(f"C{ab[0]}{ab[1]}") for ab in CLIST}
u, v, m00 = sp.symbols("u v m00")
sx, sy = sp.symbols("sx sy", positive=True)


def S(a, b):
    return C[(a, b)] / (sx ** a * sy ** b)


def c32(Sj3, Si3, Si4, Sij, Sijj, Siij, Siijj, Siiij):
    h = sp.Rational(1, 2)
    return ((Sj3 * Si3 ** 2) * h - Sj3 + Sj3 * (Si3 ** 2 - Si4 + 1)) * Sij + (Si4 - 3 * h * Si3 ** 2) * Sijj + \
        (-3 * h * Sj3 * Si3) * Siij + (3 * h * Si3) * Siijj + Sj3 * Siiij - Si3 * h


def c41(Si3, Si4, Sij, Siij, Siiij):
    q = sp.Rational(1, 4)
    return (Si3 - 2 * Si3 * Si4 + 9 * q * Si3 ** 3) * Sij + (10 * q * Si4 - 15 * q * Si3 ** 2 - 6 * q) * Siij + (2 * Si3) * Siiij


def closures():
    S32 = c32(S(0, 3), S(3, 0), S(4, 0), S(1, 1), S(1, 2), S(2, 1), S(2, 2), S(3, 1))
    S23 = c32(S(3, 0), S(0, 3), S(0, 4), S(1, 1), S(2, 1), S(1, 2), S(2, 2), S(1, 3))
    S14 = c41(S(0, 3), S(0, 4), S(1, 1), S(1, 2), S(1, 3))
    return {(3, 2): S32 * sx ** 3 * sy ** 2, (2, 3): S23 * sx ** 2 * sy ** 3, (1, 4): S14 * sx * sy ** 4}


def raw(a, b, clo):
    def Ct(p, q):
        if p + q == 0:
            return sp.Integer(1)
        if p + q == 1:
            return sp.Integer(0)
        return clo[(p, q)] if (p, q) in clo else C[(p, q)]
    return m00 * sum(sp.binomial(a, p) * sp.binomial(b, q) * Ct(p, q) * u ** (a - p) * v ** (b - q)
                     for p in range(a + 1) for q in range(b + 1))


def derive():
    clo = closures()
    wc = [C[ab] for ab in W]          # the W-dependent central moments, W order
    rows = []
    for m in (raw(3, 2, clo), raw(2, 3, clo), raw(1, 4, clo)):
        dmdc = []
        for c in wc:
            d = sp.diff(m, c)
            if c == C[(0, 2)]:         # sy = sqrt(C02)
                d = d + sp.diff(m, sy) / (2 * sy)
            d = sp.expand(d).subs({sx: sp.sqrt(C[(2, 0)]), sy: sp.sqrt(C[(0, 2)])})
            dmdc.append(sp.together(sp.expand(d)))
        rows.append(dmdc)
    return rows


class Printer(C99CodePrinter):
    """Integer powers as explicit products (no pow calls)."""

    def _print_Pow(self, e):
        b, n = e.args
        if n.is_Integer:
            k = int(n)
            base = self.parenthesize(b, 100)
            if k > 0:
                return "(" + {2: f"{base}*{base}", 3: f"{base}*{base}*{base}", 4: f"({base}*{base})*({base}*{base})"}[k] + ")"
            if k == -1:
                return f"(R(1.0)/{base})"
            return f"(R(1.0)/{self._print(b ** (-k))})"
        return super()._print_Pow(e)


def emit():
    rows = derive()
    nu_, nv_ = sp.symbols("nu nv")
    P = Printer()
    L = []
    L.append("  const R m00 = m[0];")
    L.append("  const R u = m[5] / m00, v = m[1] / m00, nu = -u, nv = -v;")
    L.append("  const R nu2 = nu * nu, nu3 = nu2 * nu, nu4 = nu2 * nu2, nv2 = nv * nv, nv3 = nv2 * nv, nv4 = nv2 * nv2;")
    for n, (a, b) in enumerate(ARGS):
        if a + b >= 2:
            L.append(f"  const R r{a}{b} = m[{n}] / m00;")
    pw = {0: None, 1: "{}", 2: "{}2", 3: "{}3", 4: "{}4"}
    # central moments: C_ab = sum binom(a,p) binom(b,q) nu^(a-p) nv^(b-q) r_pq,
    # r00 = 1, r10 = -nu, r01 = -nv (terms summed in increasing p, q)
    for (a, b) in CLIST:
        terms = []
        for p in range(a + 1):
            for q in range(b + 1):
                co = sp.binomial(a, p) * sp.binomial(b, q)
                fac = []
                if a - p:
                    fac.append(pw[a - p].format("nu"))
                if b - q:
                    fac.append(pw[b - q].format("nv"))
                if p + q == 0:
                    pass
                elif (p, q) == (1, 0):
                    fac.append("u")
                elif (p, q) == (0, 1):
                    fac.append("v")
                else:
                    fac.append(f"r{p}{q}")
                t = "*".join(fac) if fac else "R(1.0)"
                if co != 1:
                    t = f"R({int(co)}.0)*{t}"
                terms.append(t)
        L.append(f"  const R C{a}{b} = " + " + ".join(terms) + ";")
    flat = [e for row in rows for e in row]
    repl, red = sp.cse(flat, symbols=sp.numbered_symbols("t"), optimizations="basic")
    for sym, e in repl:
        L.append(f"  const R {sym} = {P.doprint(e)};")
    names = ["d32", "d23", "d14"]
    for i, nm in enumerate(names):
        vals = ", ".join(P.doprint(red[i * 6 + j]) for j in range(6))
        L.append(f"  const R {nm}[6] = {{{vals}}};  // d m{nm[1:]} / d(C02, C12, C22, C03, C13, C04)")
    # chain with dC/dW (W order m02, m12, m22, m03, m13, m04), all / m00
    # dC02: m02 1;  dC12: m12 1, m02 nu;  dC22: m22 1, m12 2nu, m02 nu^2
    # dC03: m03 1, m02 3nv;  dC13: m13 1, m03 nu, m12 3nv, m02 3nu nv
    # dC04: m04 1, m03 4nv, m02 6nv^2
    L.append("  const R im = R(1.0) / m00;")
    for nm, out in zip(names, ("r3", "r5", "r6")):
        L.append(f"  {out}[0] = ({nm}[0] + {nm}[1]*nu + {nm}[2]*nu2 + R(3.0)*{nm}[3]*nv + R(3.0)*{nm}[4]*(nu*nv) + R(6.0)*{nm}[5]*nv2) * im;")
        L.append(f"  {out}[1] = ({nm}[1] + R(2.0)*{nm}[2]*nu + R(3.0)*{nm}[4]*nv) * im;")
        L.append(f"  {out}[2] = {nm}[2] * im;")
        L.append(f"  {out}[3] = ({nm}[3] + {nm}[4]*nu + R(4.0)*{nm}[5]*nv) * im;")
        L.append(f"  {out}[4] = {nm}[4] * im;")
        L.append(f"  {out}[5] = {nm}[5] * im;")
    head = ("// Generated by gen_jacobian6.py (package codegen/) from the definition of\n"
            "// jacobian6: closed-form rows 3, 5, 6 of the x-flux Jacobian of the 2-D\n"
            "// HyQMOM closure.  Do not edit by hand.  Expects scalar type R, input\n"
            "// m[15] (m00,m01,m02,m03,m04,m10,m11,m12,m13,m20,m21,m22,m30,m31,m40),\n"
            "// outputs r3[6], r5[6], r6[6] in W = (m02,m12,m22,m03,m13,m04) order.\n")
    return head + "\n".join(L) + "\n"


if __name__ == "__main__":
    text = emit()
    outs = [os.path.join(d, "gen_jacobian6.inc") for d in sys.argv[1:]] or OUTPUTS
    for dst in outs:
        with open(dst, "w") as f:
            f.write(text)
    print("wrote", ", ".join(os.path.normpath(o) for o in outs))

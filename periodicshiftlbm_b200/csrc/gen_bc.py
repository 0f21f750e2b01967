"""Derive the D3Q27 moment-based boundary conditions and emit code for them.

Build-time tool (sympy, exact rationals).  Running it regenerates

* ``periodicshiftlbm_b200/csrc/psl_bc_generated.cuh`` -- straight-line ``__host__ __device__``
  templates (one function per outer normal) used by the CUDA kernels;
* ``oracle/bc_oracle_generated.h`` -- the same matrices as plain coefficient tables, which
  the CPU oracle evaluates with generic loops (a second, independent evaluation path).

The derivation restates the reference's method (paper.pdf pp. 5-14 and the reference's
generator symbolicHelperTools/CppCodeGenerator/helperMain.py:103-373), so that the
emitted formulas equal, entry for entry, the reference's shipped headers
include/boundaryConditions/{applyMBBC,restoreRho,restoreUxUyUz,restoreRhoUxUyUz}.h and
symbolicHelperTools/CppCodeGenerator/results/applyMirror.h:

1. After streaming, a boundary cell with outer normal n misses the populations whose
   velocity has any component pointing into the domain from outside:
   unknown = { q : min_a(c_qa * n_a) < 0 } (helperMain.py:152-155).
2. Moments m_abc = sum_q c_qx^a c_qy^b c_qz^c f_q over 23 exponent triples in a fixed order
   (helperMain.py:22-27).  Their imposed equilibrium values are the reference's table
   (helperMain.py:29-52): the product-form equilibrium moments without the monomials
   that contain all three velocity components; here they are generated by that rule.
3. Moment-based BC (applyMBBC): pick moment rows greedily, in list order, starting with
   row 0, keeping a row when it raises the rank of the unknown-population block, until
   there are as many rows as unknowns; then f_u = (S Mfu)^-1 (S m_eq - S Mfk f_k)
   (helperMain.py:170-183, 280-305).
4. Missing macroscopic values: left null space of Mfu (rows of the moment system that do
   not involve unknowns), basis vectors sorted by the summed order of the moments they
   touch; the linear part of m_eq in (rho, rho*u) is Q.  restoreRhoUxUyUz keeps the
   first 4 rank-raising rows of C^T Q, restoreUxUyUz the first 3 of C^T Qu (always keeping
   row 0), restoreRho row 0 (helperMain.py:185-278, 307-356).
5. Free slip (applyMirror): each unknown takes the population whose velocity equals its
   own with the components that point into the domain reversed (applyMirror.py).

Usage:  python periodicshiftlbm_b200/csrc/gen_bc.py
"""
from __future__ import annotations

import os
from fractions import Fraction

import sympy as sp

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.abspath(os.path.join(HERE, "..", ".."))
CUDA_OUT = os.path.join(HERE, "psl_bc_generated.cuh")
ORACLE_OUT = os.path.join(REPO, "oracle", "bc_oracle_generated.h")

# D3Q27 velocity ordering of the reference (include/applyStreaming.h:1-8).
CX = [0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, -1, 1, 0, 0, -1, 1, 0, 0, -1, 1, -1, 1, 1, -1, -1, 1]
CY = [0, 0, 0, 0, 0, -1, 1, 0, 0, 0, 0, -1, 1, 1, -1, 1, -1, 1, -1, 1, -1, -1, 1, -1, 1, -1, 1]
CZ = [0, 0, 0, -1, 1, 0, 0, -1, 1, 1, -1, 0, 0, -1, 1, 0, 0, 1, -1, -1, 1, 1, -1, -1, 1, -1, 1]
W = [sp.Rational(8, 27)] + [sp.Rational(2, 27)] * 6 + [sp.Rational(1, 54)] * 12 + [sp.Rational(1, 216)] * 8

# Exponent triples, in the order the moment system is assembled.
MOMENTS = ["000", "100", "010", "001", "200", "020", "002", "011", "101", "110", "111",
           "210", "201", "120", "021", "102", "012", "022", "202", "220", "211", "121", "112"]

# The 26 outer normals in the reference's enumeration order.
NORMALS = [(1, 0, 0), (0, 1, 0), (0, 0, 1), (-1, 0, 0), (0, -1, 0), (0, 0, -1),
           (0, 1, 1), (1, 0, 1), (1, 1, 0), (0, -1, -1), (-1, 0, -1), (-1, -1, 0),
           (0, 1, -1), (1, 0, -1), (1, -1, 0), (0, -1, 1), (-1, 0, 1), (-1, 1, 0),
           (1, 1, 1), (-1, -1, -1), (-1, 1, 1), (1, -1, 1), (1, 1, -1), (1, -1, -1), (-1, 1, -1), (-1, -1, 1)]

rho, ux, uy, uz = sp.symbols("rho ux uy uz")


def normal_index(n):
    """Outer normal -> 0..26 (13 is the interior, (0,0,0))."""
    return (n[0] + 1) * 9 + (n[1] + 1) * 3 + (n[2] + 1)


def moment_order(m):
    return sum(int(ch) for ch in m)


def velocity_power(q, m):
    a, b, c = (int(ch) for ch in m)
    return CX[q] ** a * CY[q] ** b * CZ[q] ** c


def equilibrium_moments():
    """Equilibrium moments the boundary conditions impose, as polynomials in rho, u.

    The reference's table (helperMain.py:29-52) is the factorised ("product form")
    equilibrium rho * M(ux) * M(uy) * M(uz), with M_0 = 1, M_1 = u, M_2 = 1/3 + u^2 per
    axis, minus every monomial that contains all three velocity components (so m_111 = 0
    and m_211 = rho uy uz / 3).  The rule is asserted below against a few entries.
    """
    per_axis = {0: lambda u: sp.Integer(1), 1: lambda u: u, 2: lambda u: sp.Rational(1, 3) + u * u}
    out = []
    for m in MOMENTS:
        a, b, c = (int(ch) for ch in m)
        full = sp.expand(rho * per_axis[a](ux) * per_axis[b](uy) * per_axis[c](uz))
        poly = sp.Poly(full, rho, ux, uy, uz)
        kept = sum(coef * rho ** pr * ux ** px * uy ** py * uz ** pz
                   for (pr, px, py, pz), coef in poly.terms() if not (px and py and pz))
        out.append(sp.expand(kept))
    table = dict(zip(MOMENTS, out))
    assert table["111"] == 0
    assert sp.expand(table["211"] - rho * uy * uz / 3) == 0
    assert sp.expand(table["210"] - (rho * uy / 3 + rho * ux * ux * uy)) == 0
    assert sp.expand(table["022"] - (rho / 9 + rho * uy ** 2 / 3 + rho * uz ** 2 / 3 + rho * uy ** 2 * uz ** 2)) == 0
    return out


def linear_part(expr):
    """Coefficients of (rho, rho*ux, rho*uy, rho*uz) in an m_eq polynomial (terms of
    higher order in u are dropped): the reference's Q matrix row."""
    poly = sp.Poly(sp.expand(expr), rho, ux, uy, uz)
    row = [sp.Integer(0)] * 4
    for (pr, px, py, pz), coef in poly.terms():
        if pr != 1:
            continue
        if (px, py, pz) == (0, 0, 0):
            row[0] += coef
        elif (px, py, pz) == (1, 0, 0):
            row[1] += coef
        elif (px, py, pz) == (0, 1, 0):
            row[2] += coef
        elif (px, py, pz) == (0, 0, 1):
            row[3] += coef
    return row


def greedy_rows(mat, count, first=0):
    """Rows of `mat`, taken in order starting at `first`, that raise the rank."""
    keep = [first]
    i = first + 1
    while len(keep) < count:
        if i >= mat.rows:
            raise RuntimeError("ran out of independent rows")
        if mat.extract(keep + [i], list(range(mat.cols))).rank() > mat.extract(keep, list(range(mat.cols))).rank():
            keep.append(i)
        i += 1
    return keep


class NormalBC:
    """All boundary-condition matrices for one outer normal."""

    def __init__(self, n, meq, qlin):
        self.n = n
        self.index = normal_index(n)
        prod = [min(CX[q] * n[0], CY[q] * n[1], CZ[q] * n[2]) for q in range(27)]
        self.unknown = [q for q in range(27) if prod[q] < 0]
        self.known = [q for q in range(27) if prod[q] >= 0]
        M = sp.Matrix([[velocity_power(q, m) for q in range(27)] for m in MOMENTS])
        Mu = M.extract(list(range(len(MOMENTS))), self.unknown)
        Mk = M.extract(list(range(len(MOMENTS))), self.known)
        nu = len(self.unknown)

        # --- moment-based BC ---
        self.srows = greedy_rows(Mu, nu)
        SMu = Mu.extract(self.srows, list(range(nu)))
        self.mbbc_inv = SMu.inv()                       # nu x nu
        self.mbbc_known = Mk.extract(self.srows, list(range(len(self.known))))  # nu x nk
        self.mbbc_meq = [meq[r] for r in self.srows]

        # --- left null space of Mu, sorted by the order of the moments it touches ---
        basis = Mu.T.nullspace()
        basis = sorted(basis, key=lambda v: sum(moment_order(MOMENTS[i]) for i in range(len(v)) if v[i] != 0))
        C = sp.Matrix.hstack(*basis)                    # 23 x m
        Q = sp.Matrix(qlin)                             # 23 x 4
        CQ = C.T * Q
        CMk = C.T * Mk

        # restoreRhoUxUyUz: (rho, j) = (Sq C^T Q)^-1 Sq C^T Mk f_k
        sq = greedy_rows(CQ, 4)
        self.rhou_rows = (CQ.extract(sq, [0, 1, 2, 3]).inv() * CMk.extract(sq, list(range(len(self.known)))))

        # restoreUxUyUz (given rho): u = (Su C^T Qu)^-1 ((Su C^T Mk f_k)/rho - Su C^T Qrho)
        CQu = CQ.extract(list(range(CQ.rows)), [1, 2, 3])
        CQr = CQ.extract(list(range(CQ.rows)), [0])
        su = greedy_rows(CQu, 3)
        self.u_inv = CQu.extract(su, [0, 1, 2]).inv()
        self.u_known = CMk.extract(su, list(range(len(self.known))))
        self.u_rho = CQr.extract(su, [0])

        # restoreRho (given u): rho = (C^T Mk f_k)_0 / ((C^T Qrho)_0 + (C^T Qu)_0 . u)
        if CQr[0, 0] == 0:
            raise RuntimeError("restoreRho: first null-space row has no rho term")
        self.r_known = CMk.extract([0], list(range(len(self.known))))
        self.r_rho = CQr[0, 0]
        self.r_u = CQu.extract([0], [0, 1, 2])

        # free slip
        self.mirror = {}
        for q in self.unknown:
            c = [CX[q], CY[q], CZ[q]]
            r = [-c[a] if c[a] == -n[a] else c[a] for a in range(3)]
            src = next(p for p in range(27) if [CX[p], CY[p], CZ[p]] == r)
            self.mirror[q] = src


# ---------------------------------------------------------------------------------------
# code emission
# ---------------------------------------------------------------------------------------
def c_rational(x) -> str:
    """A rational constant in type T, exact for small denominators (T(p)/T(q) folds to
    the correctly rounded value in both float and double, like the reference's 1.f/3.f)."""
    x = sp.Rational(x)
    if x.q == 1:
        return f"T({x.p})"
    return f"(T({x.p}) / T({x.q}))"


# --- expressions in the reference's evaluation order ---------------------------------------
# The reference's generated headers are left-to-right sums of "coef * value" terms, where a
# coefficient of +1/-1 is written as a bare "+ x"/"- x".  The emitted code evaluates the
# same operations in the same order with explicit round-to-nearest operations (rn_add,
# rn_sub, rn_mul, rn_div), so the compiler cannot contract them into FMAs: given equal
# inputs, the CUDA boundary conditions round exactly like the reference's host build.
def term_value(coef, name) -> tuple:
    """(sign, code) of one term: sign +1/-1 for bare terms, 0 for 'coef * name' terms."""
    coef = sp.Rational(coef)
    if coef == 1:
        return (1, name)
    if coef == -1:
        return (-1, name)
    return (0, f"rn_mul({c_rational(coef)}, {name})")


def ordered_sum(terms) -> str:
    """Left-to-right sum of (sign, code) terms; the first bare '- x' is a negation."""
    terms = [t for t in terms if t is not None]
    if not terms:
        return "T(0)"
    sign, code = terms[0]
    acc = f"(-{code})" if sign == -1 else code
    for sign, code in terms[1:]:
        acc = f"rn_sub({acc}, {code})" if sign == -1 else f"rn_add({acc}, {code})"
    return acc


def lin_terms(coefs, names):
    return [term_value(c, n) for c, n in zip(coefs, names) if sp.Rational(c) != 0]


def meq_terms(expr):
    """The imposed equilibrium moment as the reference writes it: terms by increasing
    degree (x before y before z within a degree), each 'coef * rho * ux * ... * uz'
    multiplied left to right, e.g. (1.f/3.f) * rho + rho * ux * ux."""
    poly = sp.Poly(sp.expand(expr / rho), ux, uy, uz)
    terms = sorted(poly.terms(), key=lambda t: (sum(t[0]), tuple(-e for e in t[0])))
    out = []
    for (px, py, pz), coef in terms:
        coef = sp.Rational(coef)
        factors = ["ux"] * px + ["uy"] * py + ["uz"] * pz
        if coef == 1:
            code = "rho"
        else:
            code = f"rn_mul({c_rational(coef)}, rho)"
        for fct in factors:
            code = f"rn_mul({code}, {fct})"
        out.append((1, code))
    return out


def emit_cuda(bcs) -> str:
    L = []
    L.append("// GENERATED by periodicshiftlbm_b200/csrc/gen_bc.py -- do not edit.")
    L.append("//")
    L.append("// D3Q27 moment-based boundary conditions, one straight-line function per outer")
    L.append("// normal (normal index = (nx+1)*9 + (ny+1)*3 + (nz+1); 13 is the interior).")
    L.append("// Same formulas, evaluated in the same order, as the reference's")
    L.append("// include/boundaryConditions/applyMBBC.h, restoreRho.h, restoreUxUyUz.h,")
    L.append("// restoreRhoUxUyUz.h and the free-slip generator output")
    L.append("// symbolicHelperTools/CppCodeGenerator/results/applyMirror.h.  Every operation is an")
    L.append("// explicit round-to-nearest op (no FMA contraction), and every array index is a")
    L.append("// compile-time constant so the populations stay in registers.")
    L.append("#pragma once")
    L.append("")
    L.append('#include "psl_rn.cuh"')
    L.append("")
    L.append("namespace psl {")
    L.append("namespace bc {")
    L.append("")
    for b in bcs:
        n = b.n
        tag = f"n{b.index}"
        kn = [f"f[{q}]" for q in b.known]
        L.append(f"// ---- outer normal ({n[0]:+d},{n[1]:+d},{n[2]:+d}): {len(b.unknown)} unknown populations ----")
        # MBBC (applyMBBC.h): smf = S Mfk fk; m = S m_eq; s = m - smf; f_u = inv * s
        L.append("template <typename T>")
        L.append(f"PSL_HDI void mbbc_{tag}(T (&f)[27], const T rho, const T ux, const T uy, const T uz) {{")
        for r in range(len(b.srows)):
            row = [b.mbbc_known[r, j] for j in range(len(b.known))]
            L.append(f"  const T smf{r} = {ordered_sum(lin_terms(row, kn))};")
        for r in range(len(b.srows)):
            L.append(f"  const T m{r} = {ordered_sum(meq_terms(b.mbbc_meq[r]))};")
        for r in range(len(b.srows)):
            L.append(f"  const T s{r} = rn_sub(m{r}, smf{r});")
        sn = [f"s{r}" for r in range(len(b.srows))]
        for i, q in enumerate(b.unknown):
            row = [b.mbbc_inv[i, r] for r in range(len(b.srows))]
            L.append(f"  f[{q}] = {ordered_sum(lin_terms(row, sn))};")
        L.append("}")
        # restoreRhoUxUyUz.h: q = (Sq C^T Q)^-1 Sq C^T Mfk fk; rho = q0; u = q/rho
        L.append("template <typename T>")
        L.append(f"PSL_HDI void restore_rho_u_{tag}(const T (&f)[27], T& rho, T& ux, T& uy, T& uz) {{")
        for r in range(4):
            row = [b.rhou_rows[r, j] for j in range(len(b.known))]
            L.append(f"  const T q{r} = {ordered_sum(lin_terms(row, kn))};")
        L.append("  rho = q0;")
        L.append("  ux = rn_div(q1, rho);")
        L.append("  uy = rn_div(q2, rho);")
        L.append("  uz = rn_div(q3, rho);")
        L.append("}")
        # restoreUxUyUz.h: scmf = (Su C^T Mfk fk)/rho; s = scmf - Su C^T Qrho; u = inv * s
        L.append("template <typename T>")
        L.append(f"PSL_HDI void restore_u_{tag}(const T (&f)[27], const T rho, T& ux, T& uy, T& uz) {{")
        for r in range(3):
            row = [b.u_known[r, j] for j in range(len(b.known))]
            L.append(f"  const T scmf{r} = rn_div({ordered_sum(lin_terms(row, kn))}, rho);")
        for r in range(3):
            L.append(f"  const T s{r} = rn_sub(scmf{r}, {c_rational(b.u_rho[r, 0])});")
        for a, nm in enumerate(["ux", "uy", "uz"]):
            row = [b.u_inv[a, r] for r in range(3)]
            L.append(f"  {nm} = {ordered_sum(lin_terms(row, ['s0', 's1', 's2']))};")
        L.append("}")
        # restoreRho.h: rho = (C^T Mfk fk)_0 / ((C^T Qrho)_0 + (C^T Qu)_0 . u)
        L.append("template <typename T>")
        L.append(f"PSL_HDI void restore_rho_{tag}(const T (&f)[27], T& rho, const T ux, const T uy, const T uz) {{")
        uterms = []
        for a, nm in enumerate(["ux", "uy", "uz"]):
            cf = sp.Rational(b.r_u[0, a])
            if cf != 0:
                uterms.append((0, f"rn_mul({c_rational(cf)}, {nm})"))
        L.append(f"  const T scqu = {ordered_sum(uterms)};")
        L.append(f"  const T s = rn_add({c_rational(b.r_rho)}, scqu);")
        row = [b.r_known[0, j] for j in range(len(b.known))]
        L.append(f"  const T scmf = {ordered_sum(lin_terms(row, kn))};")
        L.append("  rho = rn_div(scmf, s);")
        L.append("}")
        # applyMirror.h (sources are always known populations, so order does not matter)
        L.append("template <typename T>")
        L.append(f"PSL_HDI void mirror_{tag}(T (&f)[27]) {{")
        for q in b.unknown:
            L.append(f"  f[{q}] = f[{b.mirror[q]}];")
        L.append("}")
        L.append("")

    def dispatcher(name, sig, call):
        L.append("template <typename T>")
        L.append(f"PSL_HDI void {name}({sig}) {{")
        L.append("  switch (normal) {")
        for b in bcs:
            L.append(f"    case {b.index}: {call.format(tag='n' + str(b.index))}; break;")
        L.append("    default: break;")
        L.append("  }")
        L.append("}")

    dispatcher("mbbc", "const int normal, T (&f)[27], const T rho, const T ux, const T uy, const T uz",
               "mbbc_{tag}(f, rho, ux, uy, uz)")
    dispatcher("restore_rho_u", "const int normal, const T (&f)[27], T& rho, T& ux, T& uy, T& uz",
               "restore_rho_u_{tag}(f, rho, ux, uy, uz)")
    dispatcher("restore_u", "const int normal, const T (&f)[27], const T rho, T& ux, T& uy, T& uz",
               "restore_u_{tag}(f, rho, ux, uy, uz)")
    dispatcher("restore_rho", "const int normal, const T (&f)[27], T& rho, const T ux, const T uy, const T uz",
               "restore_rho_{tag}(f, rho, ux, uy, uz)")
    dispatcher("mirror", "const int normal, T (&f)[27]", "mirror_{tag}(f)")
    L.append("")
    L.append("}  // namespace bc")
    L.append("}  // namespace psl")
    L.append("")
    return "\n".join(L)


def frac_str(x) -> str:
    x = sp.Rational(x)
    return f"{x.p}.0 / {x.q}.0" if x.q != 1 else f"{x.p}.0"


def emit_oracle(bcs, meq) -> str:
    """Coefficient tables (indexed by normal index) for the oracle's generic evaluator."""
    L = []
    L.append("// GENERATED by periodicshiftlbm_b200/csrc/gen_bc.py -- do not edit.")
    L.append("//")
    L.append("// ORACLE / TEST INFRASTRUCTURE ONLY.  D3Q27 moment-based boundary-condition")
    L.append("// matrices as coefficient tables over all 27 populations (zero where a population")
    L.append("// does not enter), evaluated by generic loops in oracle/psl_oracle.cpp.  Follows")
    L.append("// the reference's include/boundaryConditions/*.h and")
    L.append("// symbolicHelperTools/CppCodeGenerator/results/applyMirror.h.")
    L.append("#pragma once")
    L.append("")
    L.append("namespace oracle_bc {")
    L.append("")
    L.append("struct NormalTable {")
    L.append("  int valid;")
    L.append("  int n_unknown;")
    L.append("  int unknown[19];")
    L.append("  int mbbc_moment[19];          // moment ids (into the 23-moment list) of S")
    L.append("  double mbbc_inv[19][19];      // (S Mfu)^-1")
    L.append("  double mbbc_known[19][27];    // S Mfk over all populations")
    L.append("  double rhou[4][27];           // (Sq C^T Q)^-1 Sq C^T Mfk")
    L.append("  double u_inv[3][3];           // (Su C^T Qu)^-1")
    L.append("  double u_known[3][27];        // Su C^T Mfk")
    L.append("  double u_rho[3];              // Su C^T Qrho")
    L.append("  double r_known[27];           // (C^T Mfk)_0")
    L.append("  double r_rho;                 // (C^T Qrho)_0")
    L.append("  double r_u[3];                // (C^T Qu)_0")
    L.append("  int mirror_src[27];           // -1 where the population is known")
    L.append("};")
    L.append("")
    # moment exponent table
    L.append("// Imposed equilibrium moments: m_eq[m] = rho * sum_t coef * ux^px uy^py uz^pz.")
    L.append("struct MeqTerm { double coef; int px, py, pz; };")
    L.append("struct MeqPoly { int n; MeqTerm t[9]; };")
    L.append("static const MeqPoly kMeq[23] = {")
    for e in meq:
        poly = sp.Poly(sp.expand(e / rho), ux, uy, uz)
        terms = [(coef, px, py, pz) for (px, py, pz), coef in poly.terms()]
        body = ", ".join("{%s, %d, %d, %d}" % (frac_str(cf), px, py, pz) for cf, px, py, pz in terms)
        L.append("  {%d, {%s}}," % (len(terms), body))
    L.append("};")
    L.append("")
    L.append("static const int kMomentExp[23][3] = {")
    L.append("  " + ", ".join("{%s,%s,%s}" % tuple(m) for m in MOMENTS))
    L.append("};")
    L.append("")
    by_index = {b.index: b for b in bcs}
    L.append("static const NormalTable kNormals[27] = {")
    for idx in range(27):
        b = by_index.get(idx)
        if b is None:
            L.append("  {0},  // interior")
            continue
        nk = len(b.known)

        def full(rowvals):
            out = [sp.Integer(0)] * 27
            for j, q in enumerate(b.known):
                out[q] = rowvals[j]
            return "{" + ", ".join(frac_str(v) for v in out) + "}"

        nu = len(b.unknown)
        parts = []
        parts.append("1")
        parts.append(str(nu))
        parts.append("{" + ", ".join(str(q) for q in b.unknown) + "}")
        parts.append("{" + ", ".join(str(r) for r in b.srows) + "}")
        parts.append("{" + ", ".join("{" + ", ".join(frac_str(b.mbbc_inv[i, j]) for j in range(nu)) + "}"
                                     for i in range(nu)) + "}")
        parts.append("{" + ", ".join(full([b.mbbc_known[r, j] for j in range(nk)]) for r in range(nu)) + "}")
        parts.append("{" + ", ".join(full([b.rhou_rows[r, j] for j in range(nk)]) for r in range(4)) + "}")
        parts.append("{" + ", ".join("{" + ", ".join(frac_str(b.u_inv[i, j]) for j in range(3)) + "}"
                                     for i in range(3)) + "}")
        parts.append("{" + ", ".join(full([b.u_known[r, j] for j in range(nk)]) for r in range(3)) + "}")
        parts.append("{" + ", ".join(frac_str(b.u_rho[r, 0]) for r in range(3)) + "}")
        parts.append(full([b.r_known[0, j] for j in range(nk)]))
        parts.append(frac_str(b.r_rho))
        parts.append("{" + ", ".join(frac_str(b.r_u[0, a]) for a in range(3)) + "}")
        ms = [-1] * 27
        for q, s in b.mirror.items():
            ms[q] = s
        parts.append("{" + ", ".join(str(v) for v in ms) + "}")
        L.append(f"  /* {idx}: normal ({b.n[0]:+d},{b.n[1]:+d},{b.n[2]:+d}) */ {{" + ", ".join(parts) + "},")
    L.append("};")
    L.append("")
    L.append("}  // namespace oracle_bc")
    L.append("")
    return "\n".join(L)


def main():
    meq = equilibrium_moments()
    qlin = [linear_part(e) for e in meq]
    bcs = [NormalBC(n, meq, qlin) for n in NORMALS]
    with open(CUDA_OUT, "w") as fh:
        fh.write(emit_cuda(bcs))
    with open(ORACLE_OUT, "w") as fh:
        fh.write(emit_oracle(bcs, meq))
    print(f"wrote {CUDA_OUT}\nwrote {ORACLE_OUT}")


if __name__ == "__main__":
    main()

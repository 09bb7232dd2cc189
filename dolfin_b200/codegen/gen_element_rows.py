#!/usr/bin/env python3
"""Generates ``csrc/generated/element_rows.h``: the reference tensors of the
named Lagrange forms, contracted with a geometry tensor, one element-matrix
ROW at a time.

Why rows: the engine assembles by rows (each CUDA thread owns one global
matrix row and pulls the contributions of the cells around it, in cell
order), so it needs, per (cell, local row), one row of the element matrix.
The cell is relabelled so that the row's node is canonical (vertex 0 for a
vertex node, the edge (0,1) for an edge node); only the two canonical rows
are generated.

Formulation (Kirby & Logg, "A compiler for variational forms", ACM TOMS
2006: element tensor = reference tensor x geometry tensor), written in
barycentric gradients g_a = grad(lambda_a) of the affine simplex T:

    grad(phi_i) = sum_a dphi_i/dlambda_a g_a
    A_ij = sum_{a,b} W_ab * R_ijab(kappa)
    R_ijab(kappa) = (1/|T|) int_T kappa dphi_i/dlambda_a dphi_j/dlambda_b dx

with the geometry tensor W_ab = |T| g_a.g_b for kappa*grad(u).grad(v) and
W_ab = |T| (lmbda g_a[c] g_b[e] + mu g_a[e] g_b[c] + mu delta_ce g_a.g_b) for
inner(sigma(u), epsilon(v)) (test component c, trial component e).  The
integrals of barycentric monomials are exact rationals:
int_T lambda^alpha dx = |T| d! alpha! / (d + |alpha|)!.

The same reference tensors are what FFC 2019.1.0's tabulate_tensor
evaluates for these forms (its generated code is not part of the reference
tree); the CPU oracle computes them independently by quadrature.

Run:  python dolfin_b200/codegen/gen_element_rows.py   (rewrites the header)
"""
from __future__ import annotations

import itertools
import os
from math import factorial

import sympy as sp

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "..", "csrc", "generated", "element_rows.h")

TET_EDGES = [(2, 3), (1, 3), (1, 2), (0, 3), (0, 2), (0, 1)]
TRI_EDGES = [(1, 2), (0, 2), (0, 1)]


def edges(d):
    return TET_EDGES if d == 3 else TRI_EDGES


def lam_symbols(d):
    return sp.symbols(f"l0:{d + 1}")


def basis(d, p):
    """Scalar Lagrange basis (UFC order) as polynomials in barycentrics."""
    L = lam_symbols(d)
    if p == 1:
        return [L[a] for a in range(d + 1)]
    phis = [L[a] * (2 * L[a] - 1) for a in range(d + 1)]
    phis += [4 * L[pq[0]] * L[pq[1]] for pq in edges(d)]
    return phis


def integrate(expr, d):
    """(1/|T|) int_T expr dx for a polynomial in the barycentrics."""
    L = lam_symbols(d)
    poly = sp.Poly(sp.expand(expr), *L)
    total = sp.Integer(0)
    for monom, coeff in poly.terms():
        num = factorial(d)
        for e in monom:
            num *= factorial(e)
        total += coeff * sp.Rational(num, factorial(d + sum(monom)))
    return total


def canonical_row(d, p, kind):
    """Index of the canonical row and its active barycentric set A."""
    if kind == "v":
        return 0, [0]
    # edge (0,1) is the last local edge in both tables
    e01 = edges(d).index((0, 1))
    return (d + 1) + e01, [0, 1]


def lit(v):
    v = sp.Rational(v)
    if v.q == 1:
        return f"CT({int(v.p)})"
    return f"CT({float(v)!r})"


def emit_assign(lines, name, expr):
    """Emit C for a sympy expression whose atoms are already C names."""
    def rec(e):
        if e.is_Number:
            return lit(e)
        if e.is_Symbol:
            return str(e)
        if e.is_Add:
            text = ""
            for a in e.args:
                c, _ = a.as_coeff_Mul()
                if c < 0:
                    text = f"{text} - {rec(-a)}" if text else f"-{rec(-a)}"
                else:
                    text = f"{text} + {rec(a)}" if text else rec(a)
            return "(" + text + ")"
        if e.is_Mul:
            return "(" + " * ".join(rec(a) for a in e.args) + ")"
        if e.is_Pow and e.exp == 2:
            b = rec(e.base)
            return f"({b} * {b})"
        raise ValueError(f"unsupported {e}")
    lines.append(f"  {name} = {rec(expr)};")


def gen_grad_grad(d, p, kind, with_kappa):
    """Row of sum_ab W_ab R_ijab(kappa) for the canonical row."""
    L = lam_symbols(d)
    phis = basis(d, p)
    i_star, A = canonical_row(d, p, kind)
    nb = d + 1
    W = [[sp.Symbol(f"W[{ia}][{b}]") for b in range(nb)] for ia in range(len(A))]
    kap = [sp.Symbol(f"kap[{k}]") for k in range(nb)]
    kappa = sum(kap[k] * L[k] for k in range(nb)) if with_kappa else sp.Integer(1)
    outs = []
    for j, phj in enumerate(phis):
        expr = sp.Integer(0)
        for ia, a in enumerate(A):
            da = sp.diff(phis[i_star], L[a])
            if da == 0:
                continue
            for b in range(nb):
                db = sp.diff(phj, L[b])
                if db == 0:
                    continue
                coef = integrate(kappa * da * db, d)
                if coef != 0:
                    expr += W[ia][b] * sp.collect(sp.expand(coef), kap)
        outs.append(expr)
    return outs, len(A)


def gen_load(d, p, kind, with_f):
    L = lam_symbols(d)
    phis = basis(d, p)
    i_star, _ = canonical_row(d, p, kind)
    nb = d + 1
    fv = [sp.Symbol(f"f[{k}]") for k in range(nb)]
    f = sum(fv[k] * L[k] for k in range(nb)) if with_f else sp.Integer(1)
    return sp.expand(integrate(f * phis[i_star], d))


def load_kappa_text(name, d, p, kind):
    """out[m] = (1/|T|) int lambda_m f phi_i dx: derivative of the load row of
    L = kappa*f*v*dx with respect to the P1 weight kappa (f a P1 field)."""
    L = lam_symbols(d)
    phis = basis(d, p)
    i_star, _ = canonical_row(d, p, kind)
    nb = d + 1
    fv = [sp.Symbol(f"f[{k}]") for k in range(nb)]
    f = sum(fv[k] * L[k] for k in range(nb))
    lines = ["template <typename CT>",
             f"DB2_HD void {name}(const CT (&f)[{nb}], CT (&out)[{nb}]) {{"]
    for m in range(nb):
        e = sp.expand(integrate(L[m] * f * phis[i_star], d))
        emit_assign(lines, f"out[{m}]", e)
    lines.append("}")
    return "\n".join(lines)


def _rational_gcd(values):
    """Largest rational g with every value / g an integer."""
    from math import gcd
    num, den = 0, 1
    for v in values:
        v = sp.Rational(v)
        if v == 0:
            continue
        num = gcd(num, abs(int(v.p)))
        den = den * int(v.q) // gcd(den, int(v.q))
    return sp.Rational(num, den) if num else sp.Integer(1)


def _int_coeffs(expr):
    return [sp.Rational(c) for c in sp.Poly(expr, *sorted(expr.free_symbols, key=str)).coeffs()] \
        if expr.free_symbols else [sp.Rational(expr)]


def function_text(name, d, p, kind, with_kappa):
    """Row function in scaled form.  With s = NAME_scale (the largest rational
    that divides every reference-tensor coefficient of the row), the caller
    passes W' = s W and the function returns the row; every coefficient left
    is a small integer, so each output is an FMA chain over the W' entries
    (one multiply of an integer-weight kappa combination per term) and one
    final integer factor."""
    outs, na = gen_grad_grad(d, p, kind, with_kappa)
    nb = d + 1
    nj = len(outs)
    Wsyms = [sp.Symbol(f"W[{ia}][{b}]") for ia in range(na) for b in range(nb)]
    coeffs = []
    for e in outs:
        e = sp.expand(e)
        if e != 0:
            coeffs += _int_coeffs(e)
    sigma = _rational_gcd(coeffs)
    # per output: integer factor g_j and the terms W * q(kappa), q with
    # coprime integer coefficients
    rows = []
    for e in outs:
        e = sp.expand(e / sigma)
        if e == 0:
            rows.append((0, []))
            continue
        g = _rational_gcd(_int_coeffs(e))
        e = sp.expand(e / g)
        terms = []
        for w in Wsyms:
            q = sp.expand(e.coeff(w))
            if q != 0:
                terms.append((w, q))
        rows.append((g, terms))
    args = f"const CT (&W)[{na}][{nb}]"
    if with_kappa:
        args += f", const CT (&kap)[{nb}]"
    args += f", CT (&out)[{nj}]"
    lines = [
        f"constexpr double {name}_scale = {float(sigma)!r};  // {sigma}",
        "template <typename CT>",
        f"DB2_HD void {name}({args}) {{",
    ]
    # common kappa combinations over the whole row
    qs = [q for _, terms in rows for _, q in terms if q.free_symbols]
    uniq = list(dict.fromkeys(qs))
    repl, reduced = sp.cse(uniq, symbols=sp.numbered_symbols("t"), optimizations="basic")
    for sym, ex in repl:
        emit_assign(lines, f"const CT {sym}", ex)
    qname = {}
    for k, (q, r) in enumerate(zip(uniq, reduced)):
        if r.is_Symbol:
            qname[q] = str(r)
        else:
            emit_assign(lines, f"const CT q{k}", r)
            qname[q] = f"q{k}"

    def factor(q):
        if q.free_symbols:
            return qname[q]
        return lit(q)

    for j, (g, terms) in enumerate(rows):
        if not terms:
            lines.append(f"  out[{j}] = CT(0);")
            continue
        w0, q0 = terms[0]
        acc = f"{w0} * {factor(q0)}" if q0 != 1 else f"{w0}"
        if q0 == -1:
            acc = f"-{w0}"
        for w, q in terms[1:]:
            if q == 1:
                acc = f"({acc} + {w})"
            elif q == -1:
                acc = f"({acc} - {w})"
            else:
                acc = f"fma({w}, {factor(q)}, {acc})"
        if g != 1:
            acc = f"{lit(g)} * ({acc})"
        lines.append(f"  out[{j}] = {acc};")
    lines.append("}")
    return "\n".join(lines), nj, na


def load_text(name, d, p, kind, with_f):
    e = gen_load(d, p, kind, with_f)
    nb = d + 1
    args = f"const CT (&f)[{nb}]" if with_f else ""
    lines = ["template <typename CT>", f"DB2_HD CT {name}({args}) {{"]
    tmp = []
    emit_assign(tmp, "const CT r", e)
    lines.extend(tmp)
    lines.append("  return r;")
    lines.append("}")
    return "\n".join(lines)


def main():
    parts = [
        "// GENERATED by dolfin_b200/codegen/gen_element_rows.py -- do not edit.",
        "//",
        "// Canonical element-matrix rows of the named Lagrange forms, as reference",
        "// tensor (exact rationals) x geometry tensor W.  Row 'v': the row of local",
        "// vertex 0; row 'e': the row of the edge (0,1).  Columns follow the UFC local",
        "// node order of the (relabelled) cell: vertices, then edges in the order of",
        "// TetrahedronCell/TriangleCell::create_entities.",
        "//   grad_grad_*_k1 : out_j = sum_ab W_ab (1/|T|) int dphi_i/dl_a dphi_j/dl_b,",
        "//                    called with W * grad_grad_*_scale (integer coefficients remain)",
        "//   grad_grad_*_kp1: same with a P1 weight kappa = sum_k kap_k l_k inside",
        "//   load_*_f1      : (1/|T|) int phi_i ;  load_*_fp1: (1/|T|) int f phi_i",
        "#pragma once",
        "#include <cmath>",
        "#ifndef DB2_HD",
        "#if defined(__CUDACC__)",
        "#define DB2_HD __host__ __device__ __forceinline__",
        "#else",
        "#define DB2_HD inline",
        "#endif",
        "#endif",
        "",
        "namespace db2 {",
        "namespace gen {",
        "",
    ]
    for d, dname in ((2, "tri"), (3, "tet")):
        for p in (1, 2):
            kinds = ["v"] if p == 1 else ["v", "e"]
            for kind in kinds:
                el = f"p{p}{dname}_{kind}"
                for with_k, suf in ((False, "k1"), (True, "kp1")):
                    txt, nj, na = function_text(f"grad_grad_{el}_{suf}", d, p, kind, with_k)
                    parts.append(txt)
                    parts.append("")
                for with_f, suf in ((False, "f1"), (True, "fp1")):
                    parts.append(load_text(f"load_{el}_{suf}", d, p, kind, with_f))
                    parts.append("")
                parts.append(load_kappa_text(f"load_{el}_kfp1", d, p, kind))
                parts.append("")
    parts += ["}  // namespace gen", "}  // namespace db2", ""]
    os.makedirs(os.path.dirname(OUT), exist_ok=True)
    with open(OUT, "w") as fh:
        fh.write("\n".join(parts))
    print("wrote", os.path.relpath(OUT))


if __name__ == "__main__":
    main()

#!/usr/bin/env python3
"""Generates ``csrc/generated/facet_rows.h``: rows of the exterior-facet
tensors of the Lagrange P1/P2 spaces, for the facet kernels.

An exterior facet F of a triangle (an edge) or tetrahedron (a triangle) is a
simplex of dimension fd = d - 1 with barycentrics mu_0..mu_fd.  The trace of
the cell's P1/P2 basis on F is the P1/P2 basis of F; in canonical facet order
the facet nodes are the facet vertices, then (P2) the facet edges in the
local edge order of a triangle ((1,2), (0,2), (0,1)) or the single edge of
an interval.  The row of a node is generated for the canonical node only --
facet vertex 0 ('v') or facet edge (0,1) ('e'); the engine relabels each
(node, facet) incidence so that the node is canonical.

    facet_mass_*  : out_j = (1/|F|) int_F w phi_i phi_j ds    (u*v*ds, Robin)
    facet_load_*  : out   = (1/|F|) int_F w phi_i ds          (g*v*ds, Neumann)

with w = 1 (c1) or the P1 field w = sum_k w_k mu_k (cp1).  Exact integrals of
barycentric monomials: (1/|F|) int_F mu^alpha ds = fd! alpha! / (fd + |alpha|)!.
These are the tensors FFC 2019.1.0 generates for the exterior facet integrals
of these forms (ufc::exterior_facet_integral, called at
dolfin/fem/Assembler.cpp:277-281); the CPU oracle computes them independently
by quadrature.

Run:  python dolfin_b200/codegen/gen_facet_rows.py   (rewrites the header)
"""
from __future__ import annotations

import os
from math import factorial

import sympy as sp

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "..", "csrc", "generated", "facet_rows.h")


def facet_edges(fd):
    return [(1, 2), (0, 2), (0, 1)] if fd == 2 else [(0, 1)]


def basis(fd, p):
    m = sp.symbols(f"m0:{fd + 1}")
    if p == 1:
        return m, [m[a] for a in range(fd + 1)]
    ph = [m[a] * (2 * m[a] - 1) for a in range(fd + 1)]
    ph += [4 * m[a] * m[b] for a, b in facet_edges(fd)]
    return m, ph


def integrate(expr, m, fd):
    poly = sp.Poly(sp.expand(expr), *m)
    tot = sp.Integer(0)
    for monom, coeff in poly.terms():
        num = factorial(fd)
        for e in monom:
            num *= factorial(e)
        tot += coeff * sp.Rational(num, factorial(fd + sum(monom)))
    return tot


def lit(v):
    v = sp.Rational(v)
    return f"CT({int(v.p)})" if v.q == 1 else f"CT({float(v)!r})"


def emit(e):
    e = sp.expand(e)
    if e == 0:
        return "CT(0)"
    terms = []
    for t in sp.Add.make_args(e):
        c, rest = t.as_coeff_Mul()
        terms.append((c, rest))
    out = ""
    for c, rest in terms:
        body = lit(abs(c)) if rest == 1 else (str(rest) if abs(c) == 1 else f"{lit(abs(c))} * {rest}")
        if not out:
            out = f"-{body}" if c < 0 else body
        else:
            out += f" - {body}" if c < 0 else f" + {body}"
    return out


def row_index(fd, p, kind):
    return 0 if kind == "v" else len(basis(fd, p)[1]) - 1


def gen(fd, p, kind, with_w, what):
    m, ph = basis(fd, p)
    K = len(ph)
    i = row_index(fd, p, kind)
    wsym = [sp.Symbol(f"w[{k}]") for k in range(fd + 1)]
    w = sum(wsym[k] * m[k] for k in range(fd + 1)) if with_w else sp.Integer(1)
    cell = "tri" if fd == 1 else "tet"
    name = f"facet_{what}_p{p}{cell}_{kind}_{'cp1' if with_w else 'c1'}"
    args = f"const CT (&w)[{fd + 1}], " if with_w else ""
    lines = ["template <typename CT>"]
    if what == "mass":
        lines.append(f"DB2_HD void {name}({args}CT (&out)[{K}]) {{")
        for j in range(K):
            lines.append(f"  out[{j}] = {emit(integrate(w * ph[i] * ph[j], m, fd))};")
    else:
        lines.append(f"DB2_HD CT {name}({args.rstrip(', ')}) {{")
        lines.append(f"  return {emit(integrate(w * ph[i], m, fd))};")
    lines.append("}")
    return "\n".join(lines)


def main():
    parts = [
        "// GENERATED by dolfin_b200/codegen/gen_facet_rows.py -- do not edit.",
        "//",
        "// Canonical rows of the exterior-facet mass and load tensors, divided by",
        "// the facet measure |F| (see the generator's docstring).",
        "#pragma once",
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
    for fd in (1, 2):
        for p in (1, 2):
            for kind in (("v",) if p == 1 else ("v", "e")):
                for what in ("mass", "load"):
                    for with_w in (False, True):
                        parts.append(gen(fd, p, kind, with_w, what))
                        parts.append("")
    parts += ["}  // namespace gen", "}  // namespace db2", ""]
    with open(OUT, "w") as fh:
        fh.write("\n".join(parts))
    print("wrote", os.path.relpath(OUT))


if __name__ == "__main__":
    main()

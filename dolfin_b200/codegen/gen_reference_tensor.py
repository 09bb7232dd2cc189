#!/usr/bin/env python3
"""Generates ``csrc/generated/ref_tensor.h``: the whole reference tensor of
kappa*inner(grad(u), grad(v))*dx on P2 tetrahedra with a P1 kappa, as the
B operand of a tensor-core contraction.

With the barycentric gradients g_a of the affine tetrahedron T and the P1
kappa = sum_m kappa_m lambda_m (Kirby & Logg's reference tensor x geometry
tensor factorisation, as in gen_element_rows.py):

    A_ij = sum_m sum_{a<=b} G_(m,ab) R_(m,ab),ij / DEN
    G_(m,ab) = kappa_m W_ab,   W_ab = |T| g_a.g_b       (the geometry tensor)
    R_(m,ab),ij = DEN (1/|T|) int_T lambda_m (dphi_i/dlambda_a dphi_j/dlambda_b
                                             + [a<b] dphi_i/dlambda_b dphi_j/dlambda_a)

R is an integer matrix (40 features x 100 entries of the 10 x 10 element
matrix, row-major): DEN is the least common denominator of the exact
rationals, so R is exact in half precision (|R| < 2048) and the only
rounding of the contraction is in the geometry operand and the FP32 sums.

Run:  python dolfin_b200/codegen/gen_reference_tensor.py   (rewrites the header)
"""
from __future__ import annotations

import os
from math import lcm

import sympy as sp

from gen_element_rows import basis, integrate, lam_symbols

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "..", "csrc", "generated", "ref_tensor.h")

PAIRS = [(a, b) for a in range(4) for b in range(a, 4)]  # the 10 symmetric (a, b)


def reference_tensor_p2tet():
    """(R as a list of 40 rows of 100 ints, DEN)."""
    L = lam_symbols(3)
    phi = basis(3, 2)
    dphi = [[sp.diff(f, L[a]) for a in range(4)] for f in phi]
    rows = []
    for m in range(4):
        for a, b in PAIRS:
            row = []
            for i in range(10):
                for j in range(10):
                    e = dphi[i][a] * dphi[j][b]
                    if a != b:
                        e += dphi[i][b] * dphi[j][a]
                    row.append(integrate(L[m] * e, 3))
            rows.append(row)
    den = 1
    for row in rows:
        for v in row:
            den = lcm(den, int(sp.Rational(v).q))
    R = [[int(v * den) for v in row] for row in rows]
    return R, den


def b_operand_text(R, nrows=64):
    """The tensor-core B operand, ready to copy to shared memory: row n =
    entry (i <= j) of the 10 x 10 element matrix (row-major over i <= j,
    padded to 64 rows), K = 80 = two limbs of the 40 features (the second
    limb's R scaled by 2^-11, exact), in the canonical K-major layout
    without swizzle -- 16-byte cells [k / 8][n] of 8 halves -- as uint4."""
    import numpy as np
    pairs = [(i, j) for i in range(10) for j in range(i, 10)]
    B = np.zeros((nrows, 80), np.float16)
    for n, (i, j) in enumerate(pairs):
        for k in range(80):
            v = R[k % 40][10 * i + j] * (1.0 if k < 40 else 2.0 ** -11)
            B[n, k] = np.float16(v)
            assert float(B[n, k]) == v  # exact in half precision
    words = B.view(np.uint16).astype(np.uint32)
    out = ["// B operand of the tensor-core action (see gen_reference_tensor.py)",
           f"__device__ const uint4 kRefP2TetB[10][{nrows}] = {{"]
    for c in range(10):
        cells = []
        for n in range(nrows):
            w = words[n, 8 * c:8 * c + 8]
            u = [int(w[2 * q]) | (int(w[2 * q + 1]) << 16) for q in range(4)]
            cells.append("{" + ", ".join(f"0x{x:08x}u" for x in u) + "}")
        out.append("    {" + ", ".join(cells) + "},")
    out.append("};")
    return out


def main():
    R, den = reference_tensor_p2tet()
    big = max(abs(v) for row in R for v in row)
    assert big < 2048, big
    lines = [
        "// Generated by dolfin_b200/codegen/gen_reference_tensor.py -- do not edit.",
        "// Reference tensor of kappa*inner(grad(u), grad(v))*dx, P2 tetrahedra, P1",
        "// kappa: A_ij = sum_f G_f R[f][10 i + j] / DEN, f = 10 m + pair(a, b),",
        "// G_f = kappa_m |T| g_a.g_b, pairs (a <= b) in the order",
        "// " + " ".join(f"({a},{b})" for a, b in PAIRS) + ".",
        "#pragma once",
        "",
        "namespace db2 {",
        "namespace gen {",
        "",
        f"constexpr int kRefP2TetFeatures = {len(R)};",
        f"constexpr int kRefP2TetEntries = {len(R[0])};",
        f"constexpr double kRefP2TetDen = {den}.0;",
        f"constexpr int kRefP2TetMaxAbs = {big};",
        "#ifdef __CUDACC__",
        "// the tensor itself, in constant memory (read once per CTA)",
        "__constant__ short kRefP2Tet[40][100] = {",
    ]
    for row in R:
        lines.append("    {" + ", ".join(str(v) for v in row) + "},")
    lines += ["};", ""]
    lines += b_operand_text(R)
    lines += ["#endif", "", "}  // namespace gen", "}  // namespace db2", ""]
    with open(OUT, "w") as fh:
        fh.write("\n".join(lines))
    print(f"wrote {OUT}: DEN = {den}, max |R| = {big}")


if __name__ == "__main__":
    main()

"""The row-block parallel oracle driver (used by the full-size parity tests)
reproduces the whole-mesh oracle bit for bit: CSR columns, values and the
load vector, for scalar P1/P2 and vector P2 spaces."""
import numpy as np
import pytest

from dolfin_b200 import synthetic


@pytest.mark.parametrize("kind,n", [("p1", 7), ("p2", 5), ("elas", 3)])
def test_row_blocks_equal_whole_mesh(orc, kind, n):
    from oracle import parallel
    om = orc.unit_cube_mesh(n, n, n)
    om.coords = synthetic.jitter_interior(om.coords, n, 0.15, 3)
    deg = 1 if kind == "p1" else 2
    bs = 3 if kind == "elas" else 1
    od, N = orc.dofmap(om, deg, bs)
    rp, cols = orc.sparsity(N, N, od, od)
    if kind == "elas":
        a = dict(kind=orc.ELASTICITY, tdim=3, degree0=deg, vsize0=3, mu=0.4, lmbda=0.7)
        L = dict(kind=orc.LOAD, tdim=3, degree0=deg, vsize0=3, coeff=orc.COEFF_CONST, c=(0.0, 0.0, -1.0))
        wa = wL = None
    else:
        a = dict(kind=orc.DIFFUSION, tdim=3, degree0=deg, coeff=orc.COEFF_P1)
        L = dict(kind=orc.LOAD, tdim=3, degree0=deg, coeff=orc.COEFF_P1)
        wa = synthetic.uniform_field(om.nv, 0.5, 2.0, 4)
        wL = synthetic.uniform_field(om.nv, -1.0, 1.0, 5)
    fa = orc.form(a.pop("kind"), a.pop("tdim"), **a)
    fl = orc.form(L.pop("kind"), L.pop("tdim"), **L)
    ref = orc.assemble_matrix(fa, om, od, od, rp, cols, w=wa)
    bref = orc.assemble_vector(fl, om, od, N, w=wL)
    a = dict(kind=orc.ELASTICITY, tdim=3, degree0=deg, vsize0=3, mu=0.4, lmbda=0.7) if kind == "elas" \
        else dict(kind=orc.DIFFUSION, tdim=3, degree0=deg, coeff=orc.COEFF_P1)
    L = dict(kind=orc.LOAD, tdim=3, degree0=deg, vsize0=3, coeff=orc.COEFF_CONST, c=(0.0, 0.0, -1.0)) \
        if kind == "elas" else dict(kind=orc.LOAD, tdim=3, degree0=deg, coeff=orc.COEFF_P1)
    k_node = 4 if deg == 1 else 10
    c2, v2, b2, bad, visited = parallel.assemble_rows(
        om, od, N, bs, k_node, rp, a=a, L=L, wa=wa, wL=wL, nvert=om.nv if deg == 2 else None, procs=3)
    assert bad == 0 and visited >= om.nc
    assert np.array_equal(c2, cols)
    assert np.array_equal(v2, ref)
    assert np.array_equal(b2, bref)

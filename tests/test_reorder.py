"""reorder_dofs_serial = True: the reverse Cuthill-McKee numbering of
DofMapBuilder (dof_ordering_library "Boost") -- engine (host C++) against
the oracle's independent restatement; patterns bit-exact.  Host only."""
import numpy as np
import pytest

import dolfin_b200 as d2


@pytest.fixture
def reordered():
    old = d2.parameters["reorder_dofs_serial"]
    d2.parameters["reorder_dofs_serial"] = True
    yield
    d2.parameters["reorder_dofs_serial"] = old


@pytest.mark.parametrize("tdim,n,deg,vs", [(2, 6, 1, 1), (2, 5, 2, 1), (3, 3, 1, 1), (3, 3, 2, 1),
                                           (3, 2, 2, 3), (2, 4, 2, 2)])
def test_reordered_dofmap_and_pattern_match_oracle(orc, reordered, tdim, n, deg, vs):
    m = d2.UnitSquareMesh(n, n) if tdim == 2 else d2.UnitCubeMesh(n, n, n)
    om = orc.unit_square_mesh(n, n) if tdim == 2 else orc.unit_cube_mesh(n, n, n)
    V = d2.FunctionSpace(m, "Lagrange", deg, value_size=vs)
    od, N, nnew = orc.dofmap_reordered(om, deg, vs)
    assert V.reordered() and V.dim() == N
    assert np.array_equal(V.node_numbers(), nnew)
    assert np.array_equal(V.dofmap().cell_dofs_all(), od)
    rp, cols = V.pattern().csr_host()
    orp, ocols = orc.sparsity(N, N, od, od)
    assert np.array_equal(rp, orp) and np.array_equal(cols, ocols)


def test_rcm_is_a_bandwidth_reducing_permutation(orc, reordered):
    m = d2.UnitCubeMesh(4, 4, 4)
    V = d2.FunctionSpace(m, "Lagrange", 2)
    p = V.node_numbers()
    assert np.array_equal(np.sort(p), np.arange(p.size))
    rp, cols = V.pattern().csr_host()
    rows = np.repeat(np.arange(rp.size - 1), np.diff(rp))
    bw = np.max(np.abs(cols - rows))
    d2.parameters["reorder_dofs_serial"] = False
    rp0, cols0 = d2.FunctionSpace(m, "Lagrange", 2).pattern().csr_host()
    rows0 = np.repeat(np.arange(rp0.size - 1), np.diff(rp0))
    assert bw < np.max(np.abs(cols0 - rows0))

"""The C++-frontend drop-in (qdsim_b200.frontend) on the host: Mesh follows
qdsim_cpp.Mesh's constructor and accessors (backend/src/bindings.cpp:761-778)
in SI units."""
import numpy as np
import pytest


def test_mesh_accessors_and_node_layout():
    from qdsim_b200 import frontend as F
    from oracle import fem as O
    m = F.Mesh(60e-9, 40e-9, 12, 8, 2)
    om = O.structured_mesh(2, 12, 8, 60.0, 40.0)
    assert m.get_num_nodes() == om.num_nodes == (2 * 12 + 1) * (2 * 8 + 1)
    assert m.get_num_elements() == om.num_elements == 2 * 12 * 8
    assert m.getNumNodes() == m.get_num_nodes() and m.getElementOrder() == 2
    assert (m.get_lx(), m.get_ly(), m.get_nx(), m.get_ny()) == (60e-9, 40e-9, 12, 8)
    assert np.allclose(m.get_nodes(), om.nodes * 1e-9, rtol=0, atol=1e-21)
    assert np.array_equal(m.get_elements(), om.elems)


def test_mesh_rejects_bad_order_and_solver_checks_order():
    from qdsim_b200 import frontend as F
    with pytest.raises(ValueError):
        F.Mesh(1e-8, 1e-8, 4, 4, 4)
    m = F.Mesh(1e-8, 1e-8, 4, 4, 1)
    with pytest.raises(ValueError):
        F.FEMSolver(m, lambda x, y: 0.067 * 9.1093837015e-31, lambda x, y: 0.0,
                    lambda x, y: 0.0, None, 2)
    fs = F.FEMSolver(m, lambda x, y: 1.0, lambda x, y: 0.0, lambda x, y: 0.0, None, 1)
    with pytest.raises(RuntimeError):
        fs.get_H()                      # not assembled yet
    assert fs.is_using_mpi() is False

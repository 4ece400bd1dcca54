"""Assembly and eigensolve on a refined (unstructured) mesh on the GPU: the
C++-frontend drop-in's ``FEMSolver.adapt_mesh`` (backend/src/fem.cpp:470-542,
flags of backend/src/adaptive_mesh.cpp:431-494) refines where the ground state
varies fastest, reassembles on the GPU, and ``EigenSolver`` solves the refined
pencil.  Both are checked against the oracle on the same refined mesh: H and
M at 1e-12, the levels at 1e-9.  Refined meshes have no lattice, so the solve
runs without the DST preconditioner."""
import numpy as np
import pytest

from oracle import adapt as OA, fem as O

pytestmark = pytest.mark.gpu

M_E = 9.1093837015e-31
Q_E = 1.602176634e-19


def _callbacks():
    def m_star(x, y):
        r2 = (x - 30e-9) ** 2 + (y - 20e-9) ** 2
        return np.where(r2 < (8e-9) ** 2, 0.041, 0.067) * M_E

    def V(x, y):
        r2 = (x - 30e-9) ** 2 + (y - 20e-9) ** 2
        return -0.25 * Q_E * np.exp(-r2 / (2 * (7e-9) ** 2))

    def cap(x, y):
        return 0.0 * x

    return m_star, V, cap


@pytest.mark.parametrize("order", [1, 2])
def test_refined_mesh_assembly_and_levels(cuda, order):
    from qdsim_b200 import frontend as F
    m_star, V, cap = _callbacks()
    mesh = F.Mesh(60e-9, 40e-9, 24, 16, order)
    fem = F.FEMSolver(mesh, m_star, V, cap, None, order)
    fem.assemble_matrices()
    es = F.EigenSolver(fem)
    es.solve(4)
    psi0 = np.real(es.get_eigenvectors()[0])
    si = mesh._si
    g = OA.element_gradients(si.nodes, si.elems, psi0)
    thr = float(np.quantile(np.hypot(g[:, 0], g[:, 1]), 0.85))
    n_before = mesh.get_num_elements()
    fem.adapt_mesh(psi0, thr)
    assert mesh._si is not si and mesh.get_num_elements() > n_before
    H, M = fem.get_H(), fem.get_M()
    # oracle on the refined mesh (nm / eV), natural boundaries
    nm = mesh._nm
    om = O.Mesh(nm.order, nm.nx, nm.ny, nm.Lx, nm.Ly, nm.nodes, nm.elems, nm.boundary)
    cen = mesh._si.centroids()
    c = O.C0_EV_NM2 * (M_E / m_star(cen[:, 0], cen[:, 1]))
    Vn = V(mesh._si.nodes[:, 0], mesh._si.nodes[:, 1]) / Q_E
    a = O.assemble(om, c, Vn, None, dirichlet=False)
    assert abs(H.real - a.H * Q_E).max() <= 1e-12 * abs(a.H).max() * Q_E
    assert abs(H.imag).max() == 0.0
    assert abs(M - a.M * 1e-18).max() <= 1e-12 * abs(a.M).max() * 1e-18
    es2 = F.EigenSolver(fem)
    es2.solve(4)
    E = np.array(es2.get_eigenvalues()).real
    E0 = O.eig_lowest(a.H, a.M, 4, O.sigma_below(Vn))[0] * Q_E
    assert np.abs(E - E0).max() <= 1e-9 * np.abs(E0).max()

"""The C++-frontend drop-in on the GPU: FEMSolver's H and M and EigenSolver's
levels against the oracle on the same pencil (all nodes, natural boundaries,
SI units), with the reference's semantics: +i eta for the CAP in H, the
eigensolve on the Hermitian part."""
import numpy as np
import pytest

from oracle import fem as O

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
        return 0.01 * Q_E * (np.clip(5e-9 - np.minimum(x, 60e-9 - x), 0, None) / 5e-9) ** 2

    return m_star, V, cap


def test_fem_solver_matrices_and_levels(cuda):
    from qdsim_b200 import frontend as F
    m_star, V, cap = _callbacks()
    mesh = F.Mesh(60e-9, 40e-9, 30, 20, 2)
    fem = F.FEMSolver(mesh, m_star, V, cap, None, 2)
    fem.assemble_matrices()
    H, M = fem.get_H(), fem.get_M()
    # oracle on the same mesh in nm / eV
    om = O.structured_mesh(2, 30, 20, 60.0, 40.0)
    si = mesh.get_nodes()
    cen = om.nodes[om.elems[:, :3]].mean(axis=1) * 1e-9
    c = O.C0_EV_NM2 * (M_E / m_star(cen[:, 0], cen[:, 1]))
    Vn = V(si[:, 0], si[:, 1]) / Q_E
    eta = cap(si[:, 0], si[:, 1]) / Q_E
    a = O.assemble(om, c, Vn, eta, dirichlet=False)
    Href = (a.H + 1j * a.Wm) * Q_E
    assert abs(H - Href).max() <= 1e-12 * abs(Href).max()
    assert abs(M - a.M * 1e-18).max() <= 1e-12 * abs(a.M).max() * 1e-18
    es = F.EigenSolver(fem)
    es.solve(8)
    E = np.array(es.get_eigenvalues())
    assert np.all(E.imag == 0.0)
    E0 = O.eig_lowest(a.H, a.M, 8, O.sigma_below(Vn))[0] * Q_E
    assert np.abs(E.real - E0).max() <= 1e-9 * np.abs(E0).max()
    X = np.stack(es.get_eigenvectors(), axis=1)
    assert X.shape == (mesh.get_num_nodes(), 8)
    assert np.abs(np.einsum("ij,ij->j", X, (M @ X).real) - 1.0).max() < 1e-8
    # the CAP does not enter the eigensolve (Hermitian part, as in the reference)
    fem0 = F.FEMSolver(mesh, m_star, V, lambda x, y: 0.0 * x, None, 2)
    fem0.assemble_matrices()
    es0 = F.EigenSolver(fem0)
    es0.solve(8)
    assert np.allclose(np.array(es0.get_eigenvalues()).real, E.real, rtol=1e-10, atol=0)

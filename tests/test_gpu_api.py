"""The drop-in solver classes (qdsim_b200.solvers) in SI units, against the
oracle and the compiled reference's outputs."""
import os

import numpy as np
import pytest

from oracle import fem as O, refcompat as RC

pytestmark = pytest.mark.gpu
QE = 1.602176634e-19
M0 = 9.1093837015e-31


def _c1_funcs(cx=50e-9, cy=25e-9):
    def V(x, y):
        return -0.3 * QE * np.exp(-((x - cx) ** 2 + (y - cy) ** 2) / (2 * (8e-9) ** 2))

    def m(x, y):
        return np.where(V(x, y) < -0.15 * QE, 0.041, 0.067) * M0
    return m, V


def test_schrodinger_solver_si_api(cuda):
    from qdsim_b200.solvers import CythonSchrodingerSolver, SimpleMesh
    m_func, V_func = _c1_funcs()
    mesh = SimpleMesh(101, 51, 100e-9, 50e-9)
    s = CythonSchrodingerSolver(mesh, m_func, V_func)
    E, psis = s.solve(10)
    assert E.shape == (10,) and len(psis) == 10 and psis[0].shape == (mesh.num_nodes,)
    om = O.structured_mesh(1, 100, 50, 100.0, 50.0)
    cen = O.centroids(om)
    c = O.C0_EV_NM2 * M0 / m_func(cen[:, 0] * 1e-9, cen[:, 1] * 1e-9)
    Vn = V_func(om.nodes[:, 0] * 1e-9, om.nodes[:, 1] * 1e-9) / QE
    a = O.assemble(om, c, Vn)
    E0 = O.eig_lowest(a.H, a.M, 10, O.sigma_below(Vn))[0]
    assert np.abs(E / QE - E0).max() <= 1e-9 * np.abs(E0).max()
    assert np.allclose(s.get_eigenvalues_eV(), E / QE)
    # M-normalised in SI: psi^T M_SI psi = 1 with M_SI = 1e-18 M_nm
    full = O.assemble(om, c, Vn, dirichlet=False)
    for psi in psis[:3]:
        assert abs(psi @ (full.M @ psi) * 1e-18 - 1.0) < 1e-8
        assert np.all(psi[om.boundary] == 0.0)
    info = s.get_matrix_info()
    assert info["matrix_size"] == a.n


def test_fixed_solver_reference_mode(cuda):
    from qdsim_b200.solvers import FixedOpenSystemSolver

    def V(x, y):
        return -0.2 * QE * np.exp(-((x - 50e-9) ** 2 + (y - 30e-9) ** 2) / (2 * (15e-9) ** 2))

    def m(x, y):
        return (0.041 if V(x, y) < -0.1 * QE else 0.067) * M0

    s = FixedOpenSystemSolver(21, 13, 100e-9, 60e-9, m, V, assembly_mode="reference_fixed")
    E, psis = s.solve(4)
    om = O.structured_mesh(1, 20, 12, 100e-9, 60e-9)
    H, Mm = RC.fixed_assembly(om.nodes, om.elems, m, V)
    fixed = np.zeros(om.num_nodes, bool)
    fixed[[0, om.num_nodes - 1]] = True
    import scipy.linalg as sl
    ev = sl.eigh(H[~fixed][:, ~fixed].toarray(), Mm[~fixed][:, ~fixed].toarray(),
                 eigvals_only=True)[:4]
    assert np.allclose(E, ev, rtol=1e-8, atol=0)


def test_poisson_solver_matches_compiled_reference(cuda):
    from qdsim_b200.solvers import CythonPoissonSolver, SimpleMesh
    G = np.load(os.path.join(os.path.dirname(__file__), "golden", "ref_cython.npz"))

    def eps(x, y):
        return 12.9 if x < 4e-6 else 11.7

    def rho(x, y, n, p):
        return QE * 1e21 * (1.0 if x < 4e-6 else -1.0) * (1.0 + 0.3 * np.sin(y / 1e-6))

    ps = CythonPoissonSolver(SimpleMesh(9, 6, 8e-6, 5e-6), eps, rho)
    ps.solve(0.0, 0.5)
    phi = ps.get_potential()
    assert np.abs(phi - G["poisson_phi"]).max() <= 1e-10 * np.abs(G["poisson_phi"]).max()
    ex, ey = ps.get_electric_field()
    assert np.abs(ex - G["poisson_Ex"]).max() <= 1e-9 * np.abs(G["poisson_Ex"]).max()
    assert np.abs(ey - G["poisson_Ey"]).max() <= 1e-8 * np.abs(G["poisson_Ey"]).max()
    K = ps.stiffness_matrix
    import scipy.sparse as sp
    Kr = sp.csr_matrix((G["poisson_K_data"], G["poisson_K_indices"], G["poisson_K_indptr"]),
                       shape=K.shape)
    assert abs(K - Kr).max() <= 1e-12 * abs(Kr).max()


def test_self_consistent_loop_runs(cuda):
    from qdsim_b200.solvers import CythonSelfConsistentSolver, SimpleMesh
    m_func, V_func = _c1_funcs(cx=30e-9, cy=15e-9)
    mesh = SimpleMesh(31, 16, 60e-9, 30e-9)
    sc = CythonSelfConsistentSolver(mesh, lambda x, y: 12.9, m_func, V_func, temperature=300.0)
    sc.set_solver_parameters(max_iterations=3, tolerance=1e-12, mixing=0.5)
    out = sc.solve_self_consistent(0.0, 0.1, num_quantum_states=4, N_A=1e22, N_D=1e22)
    assert out["iterations"] == 3 and len(out["convergence_history"]) == 3
    assert np.all(np.isfinite(out["potential"])) and out["eigenvalues"].shape == (4,)
    assert np.isclose(out["electron_density"].mean(), 1e22)

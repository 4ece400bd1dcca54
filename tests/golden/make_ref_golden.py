"""Record outputs of the compiled reference Cython modules as fixtures
(tests/golden/ref_cython.npz).  Needs the reference tree and
``python oracle/build_ref.py`` (modules in oracle/_ref/); the fixture is
committed so the tests run without either.

Cases (SI units, as the reference uses them):
  mesh      SimpleMesh(7, 5, 3e-6, 2e-6): node coordinates and elements
  fixed     FixedOpenSystemSolver(11, 7, 100e-9, 60e-9, m*, V)
            ._assemble_matrices_robust() CSR of H and M, and solve(4)
  cython    CythonSchrodingerSolver on SimpleMesh(9, 6, 8e-6, 5e-6) (micrometre
            cells, so its 1e-15 m^2 area test keeps every element): solve(4),
            and the CSR of the H and M that solve() hands to eigsh (the
            assembled pencil after the boundary-row replacement; the class
            keeps them private, so they are captured at that call by giving
            the module a scipy.sparse.linalg stand-in whose eigsh records its
            arguments and then runs scipy's)
  poisson   CythonPoissonSolver on SimpleMesh(9, 6, 8e-6, 5e-6): stiffness and
            mass CSR, solve(0.0, 0.5) potential and electric field
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

M0 = 9.1093837015e-31
QE = 1.602176634e-19


def m_func(x, y):
    return (0.041 if (x * x + y * y) ** 0.5 < 0.5 * 8e-6 else 0.067) * M0 if x > 1e-6 else 0.067 * M0


def v_func_nm(x, y):
    return -0.2 * QE * np.exp(-((x - 50e-9) ** 2 + (y - 30e-9) ** 2) / (2 * (15e-9) ** 2))


def v_func_um(x, y):
    return -0.2 * QE * np.exp(-((x - 4e-6) ** 2 + (y - 2.5e-6) ** 2) / (2 * (1.5e-6) ** 2))


def m_func_nm(x, y):
    return (0.041 if v_func_nm(x, y) < -0.1 * QE else 0.067) * M0


def m_func_um(x, y):
    return (0.041 if v_func_um(x, y) < -0.1 * QE else 0.067) * M0


def eps_func(x, y):
    return 12.9 if x < 4e-6 else 11.7


def rho_func(x, y, n, p):
    return QE * 1e21 * (1.0 if x < 4e-6 else -1.0) * (1.0 + 0.3 * np.sin(y / 1e-6))


def csr_parts(prefix, m, out):
    m = m.tocsr()
    m.sort_indices()
    out[prefix + "_data"] = m.data
    out[prefix + "_indices"] = m.indices
    out[prefix + "_indptr"] = m.indptr


def main():
    from oracle import build_ref as R
    if not R.built() and not R.build():
        raise SystemExit("reference modules unavailable")
    mm = R.import_ref("mesh_minimal")
    fos = R.import_ref("fixed_open_system_solver")
    ss = R.import_ref("schrodinger_solver")
    ps = R.import_ref("poisson_solver")
    out = {}
    mesh = mm.SimpleMesh(7, 5, 3e-6, 2e-6)
    x, y = mesh.get_nodes()
    out["mesh_x"], out["mesh_y"], out["mesh_elems"] = x, y, mesh.get_elements()

    fs = fos.FixedOpenSystemSolver(11, 7, 100e-9, 60e-9, m_func_nm, v_func_nm)
    H, M = fs._assemble_matrices_robust()
    csr_parts("fixed_H", H, out)
    csr_parts("fixed_M", M, out)
    E, _ = fs.solve(4)
    out["fixed_E"] = np.sort(np.real(E))

    um = mm.SimpleMesh(9, 6, 8e-6, 5e-6)
    cs = ss.CythonSchrodingerSolver(um, m_func_um, v_func_um)
    captured = {}
    real_spla = ss.spla

    class _RecordingLinalg:
        def __getattr__(self, name):
            return getattr(real_spla, name)

        def eigsh(self, A, *args, **kw):
            captured.setdefault("H", A.copy())
            captured.setdefault("M", kw["M"].copy())
            return real_spla.eigsh(A, *args, **kw)

    ss.spla = _RecordingLinalg()
    try:
        E, _ = cs.solve(4)
    finally:
        ss.spla = real_spla
    csr_parts("cython_H", captured["H"], out)
    csr_parts("cython_M", captured["M"], out)
    out["cython_E"] = np.sort(np.real(E))
    out["cython_nnz"] = cs.get_matrix_info()["hamiltonian_nnz"]

    pso = ps.CythonPoissonSolver(um, eps_func, rho_func)
    csr_parts("poisson_K", pso.stiffness_matrix, out)
    csr_parts("poisson_M", pso.mass_matrix, out)
    pso.solve(0.0, 0.5)
    out["poisson_phi"] = pso.get_potential()
    ex, ey = pso.get_electric_field()
    out["poisson_Ex"], out["poisson_Ey"] = ex, ey
    np.savez_compressed(os.path.join(os.path.dirname(os.path.abspath(__file__)), "ref_cython.npz"),
                        **out)
    print("wrote", sorted(out))


if __name__ == "__main__":
    main()

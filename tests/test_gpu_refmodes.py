"""The assembly kernel's reference-compatible modes vs the compiled reference
(fixtures in tests/golden/ref_cython.npz) and the oracle's restatement."""
import os

import numpy as np
import pytest
import scipy.sparse as sp

from oracle import fem as O, poisson as OP, refcompat as RC

pytestmark = pytest.mark.gpu
G = np.load(os.path.join(os.path.dirname(__file__), "golden", "ref_cython.npz"))
HBAR = 1.054571817e-34
M0 = 9.1093837015e-31
QE = 1.602176634e-19


def _csr(prefix, n):
    return sp.csr_matrix((G[prefix + "_data"], G[prefix + "_indices"], G[prefix + "_indptr"]),
                         shape=(n, n))


def _rel(a, b):
    return abs(a - b).max() / abs(b).max()


def v_nm(x, y):
    return -0.2 * QE * np.exp(-((x - 50e-9) ** 2 + (y - 30e-9) ** 2) / (2 * (15e-9) ** 2))


def v_um(x, y):
    return -0.2 * QE * np.exp(-((x - 4e-6) ** 2 + (y - 2.5e-6) ** 2) / (2 * (1.5e-6) ** 2))


def _elem_inputs(mesh, vf):
    cen = mesh.centroids()
    V = np.array([vf(x, y) for x, y in cen])
    mstar = np.where(V < -0.1 * QE, 0.041, 0.067) * M0
    return HBAR * HBAR / (2 * mstar), V


def test_ref_fixed_mode_matches_compiled_reference(cuda):
    from qdsim_b200 import _native as N, fem as F, mesh as Mh
    m = Mh.StructuredMesh(1, 10, 6, 100e-9, 60e-9)
    c, V = _elem_inputs(m, v_nm)
    prob = F.FEMProblem(m, dirichlet=False, device=cuda)
    out = prob.assemble(c, V, mode=N.QD_ASM_REF_FIXED)
    H, M = prob.to_scipy(out["H"]), prob.to_scipy(out["M"])
    n = m.num_nodes
    assert _rel(H, _csr("fixed_H", n)) < 1e-12
    assert _rel(M, _csr("fixed_M", n)) < 1e-12


def test_ref_cython_mode_matches_oracle(cuda):
    from qdsim_b200 import _native as N, fem as F, mesh as Mh
    m = Mh.StructuredMesh(1, 8, 5, 8e-6, 5e-6)
    c, V = _elem_inputs(m, v_um)
    prob = F.FEMProblem(m, dirichlet=False, device=cuda)
    out = prob.assemble(c, V, mode=N.QD_ASM_REF_CYTHON)
    mstar = HBAR * HBAR / (2 * c)
    cen = m.centroids()
    lut = {tuple(p): (ms, v) for p, ms, v in zip(map(tuple, cen), mstar, V)}
    Hr, Mr = RC.cython_assembly(m.nodes, m.elems, lambda x, y: lut[(x, y)][0],
                                lambda x, y: lut[(x, y)][1])
    assert _rel(prob.to_scipy(out["H"]), Hr) < 1e-12
    assert _rel(prob.to_scipy(out["M"]), Mr) < 1e-12


def test_ref_cython_mode_matches_compiled_reference(cuda):
    """GPU assembly in the Cython solver's element formulas, with the
    reference's boundary-row replacement applied on the host, equals the H and
    M the compiled CythonSchrodingerSolver passes to eigsh (fixture captured
    from the compiled module) at 1e-12."""
    from qdsim_b200 import _native as N, fem as F, mesh as Mh
    m = Mh.StructuredMesh(1, 8, 5, 8e-6, 5e-6)
    c, V = _elem_inputs(m, v_um)
    prob = F.FEMProblem(m, dirichlet=False, device=cuda)
    out = prob.assemble(c, V, mode=N.QD_ASM_REF_CYTHON)
    fixed = RC.boundary_nodes(m.nodes, 8e-6, 5e-6)
    H = RC.replace_boundary_rows(prob.to_scipy(out["H"]), fixed)
    M = RC.replace_boundary_rows(prob.to_scipy(out["M"]), fixed)
    n = m.num_nodes
    Hr, Mr = _csr("cython_H", n), _csr("cython_M", n)
    assert np.array_equal(H.indices, Hr.indices) and np.array_equal(M.indices, Mr.indices)
    assert _rel(H, Hr) < 1e-12
    assert _rel(M, Mr) < 1e-12


def test_poisson_stiffness_matches_compiled_reference(cuda):
    from qdsim_b200 import mesh as Mh, poisson as P
    m = Mh.StructuredMesh(1, 8, 5, 8e-6, 5e-6)
    eps = np.where(m.centroids()[:, 0] < 4e-6, 12.9, 11.7)
    prob = P.PoissonProblem(m, eps, device=cuda)
    n = m.num_nodes
    assert _rel(prob.fem.to_scipy(prob.K) * OP.EPS0, _csr("poisson_K", n)) < 1e-12
    assert _rel(prob.fem.to_scipy(prob.M), _csr("poisson_M", n)) < 1e-12


def test_ref_cpp_mode_matches_oracle(cuda):
    """The C++ SchrodingerSolver's element formulas (QD_ASM_REF_CPP: P1
    stiffness, potential and mass by the centroid rule) on the GPU equal the
    oracle's restatement at 1e-12."""
    from qdsim_b200 import _native as N, fem as F, mesh as Mh
    m = Mh.StructuredMesh(1, 20, 12, 60e-9, 40e-9)
    c, V = _elem_inputs(m, v_nm)
    prob = F.FEMProblem(m, dirichlet=False, device=cuda)
    out = prob.assemble(c, V, mode=N.QD_ASM_REF_CPP)
    mstar = HBAR * HBAR / (2 * c)
    cen = m.centroids()
    lut = {tuple(p): (ms, v) for p, ms, v in zip(map(tuple, cen), mstar, V)}
    Hr, Mr = RC.cpp_assembly(m.nodes, m.elems, lambda x, y: lut[(x, y)][0],
                             lambda x, y: lut[(x, y)][1])
    assert _rel(prob.to_scipy(out["H"]), Hr) < 1e-12
    assert _rel(prob.to_scipy(out["M"]), Mr) < 1e-12

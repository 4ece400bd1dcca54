"""The reference Cython solvers' own element formulas, restated in numpy.
TEST INFRASTRUCTURE ONLY.  Pinned against the compiled reference modules by
the fixtures in tests/golden/ref_cython.npz (tests/golden/make_ref_golden.py).

All quantities in SI, as the reference uses them.

* ``fixed_assembly`` -- FixedOpenSystemSolver._assemble_matrices_robust
  (qdsim_cython/solvers/fixed_open_system_solver.pyx:197-271): per element,
  centroid m* and V; H_ii = hbar^2/(2m*) A/3 + V A/3, H_ij = hbar^2/(2m*) A/6
  (no shape-function gradients), consistent mass A/12 (2 on the diagonal);
  elements with area < 1e-20 m^2 skipped.
* ``cython_assembly`` -- CythonSchrodingerSolver._assemble_matrices
  (qdsim_cython/solvers/schrodinger_solver.pyx:120-251): P1 stiffness with
  gradients, V A/3 on the diagonal, added a second time at local nodes 1 and 2
  (:224-236); area < 1e-15 m^2 skipped (:151).
* ``cpp_assembly`` -- SchrodingerSolver::assemble_matrices_cpu
  (backend/src/schrodinger.cpp:92-230): P1 stiffness with gradients, the
  potential and the mass by the one-point centroid rule (every entry of the
  element matrices V A/9 and A/9).  That mass matrix is singular (each
  element adds a rank-one term), which is why the reference's dense solve
  (:699-724) falls back to adding reg I to it.
* Boundary handling: the reference replaces boundary rows by identity rows
  (:253-283; fixed solver: nodes 0 and N-1 only, :273-291).  The physical
  eigenpairs of that pencil are those of the pencil restricted to the free
  nodes, which ``eig_free`` returns.
"""
import numpy as np
import scipy.sparse as sp

from . import fem as F

HBAR = 1.054571817e-34


def _tri(nodes, elems):
    P0, P1, P2 = nodes[elems[:, 0]], nodes[elems[:, 1]], nodes[elems[:, 2]]
    det = (P1[:, 0] - P0[:, 0]) * (P2[:, 1] - P0[:, 1]) - (P2[:, 0] - P0[:, 0]) * (P1[:, 1] - P0[:, 1])
    return P0, P1, P2, det, 0.5 * np.abs(det)


def _csr(elems, Ae, n):
    rows = np.repeat(elems, 3, axis=1).ravel()
    cols = np.tile(elems, (1, 3)).ravel()
    m = sp.coo_matrix((Ae.ravel(), (rows, cols)), shape=(n, n)).tocsr()
    m.sum_duplicates()
    m.sort_indices()
    return m


def element_centroid_values(nodes, elems, m_func, V_func):
    cen = nodes[elems].mean(axis=1)
    m = np.array([m_func(x, y) for x, y in cen], dtype=float)
    V = np.array([V_func(x, y) for x, y in cen], dtype=float)
    return m, V


def fixed_assembly(nodes, elems, m_func, V_func):
    _, _, _, det, A = _tri(nodes, elems)
    keep = A >= 1e-20
    m, V = element_centroid_values(nodes, elems, m_func, V_func)
    kin = HBAR * HBAR / (2.0 * m) * A / 3.0
    pot = V * A / 3.0
    He = np.empty((len(A), 3, 3))
    He[:] = (kin * 0.5)[:, None, None]
    for i in range(3):
        He[:, i, i] = kin + pot
    Me = np.empty((len(A), 3, 3))
    Me[:] = (A / 12.0)[:, None, None]
    for i in range(3):
        Me[:, i, i] = 2.0 * A / 12.0
    n = nodes.shape[0]
    return _csr(elems[keep], He[keep], n), _csr(elems[keep], Me[keep], n)


def cython_assembly(nodes, elems, m_func, V_func):
    P0, P1, P2, det, A = _tri(nodes, elems)
    keep = A >= 1e-15
    m, V = element_centroid_values(nodes, elems, m_func, V_func)
    inv = 1.0 / det
    g = np.stack([np.stack([(P1[:, 1] - P2[:, 1]) * inv, (P2[:, 0] - P1[:, 0]) * inv], 1),
                  np.stack([(P2[:, 1] - P0[:, 1]) * inv, (P0[:, 0] - P2[:, 0]) * inv], 1),
                  np.stack([(P0[:, 1] - P1[:, 1]) * inv, (P1[:, 0] - P0[:, 0]) * inv], 1)], 1)
    kin = HBAR * HBAR / (2.0 * m) * A
    He = kin[:, None, None] * np.einsum('eid,ejd->eij', g, g)
    pot = V * A / 3.0
    He[:, 0, 0] += pot
    He[:, 1, 1] += 2.0 * pot
    He[:, 2, 2] += 2.0 * pot
    Me = np.empty((len(A), 3, 3))
    Me[:] = (A / 12.0)[:, None, None]
    for i in range(3):
        Me[:, i, i] = 2.0 * A / 12.0
    n = nodes.shape[0]
    return _csr(elems[keep], He[keep], n), _csr(elems[keep], Me[keep], n)


def cpp_assembly(nodes, elems, m_func, V_func):
    P0, P1, P2, det, A = _tri(nodes, elems)
    m, V = element_centroid_values(nodes, elems, m_func, V_func)
    inv = 1.0 / det
    g = np.stack([np.stack([(P1[:, 1] - P2[:, 1]) * inv, (P2[:, 0] - P1[:, 0]) * inv], 1),
                  np.stack([(P2[:, 1] - P0[:, 1]) * inv, (P0[:, 0] - P2[:, 0]) * inv], 1),
                  np.stack([(P0[:, 1] - P1[:, 1]) * inv, (P1[:, 0] - P0[:, 0]) * inv], 1)], 1)
    kin = HBAR * HBAR / (2.0 * m) * A
    He = kin[:, None, None] * np.einsum('eid,ejd->eij', g, g) + (V * A / 9.0)[:, None, None]
    Me = np.broadcast_to((A / 9.0)[:, None, None], He.shape).copy()
    n = nodes.shape[0]
    return _csr(elems, He, n), _csr(elems, Me, n)


def boundary_nodes(nodes, Lx, Ly):
    x, y = nodes[:, 0], nodes[:, 1]
    return (np.abs(x) < 1e-12) | (np.abs(x - Lx) < 1e-12) | (np.abs(y) < 1e-12) | (np.abs(y - Ly) < 1e-12)


def replace_boundary_rows(A, fixed):
    """The reference's Dirichlet treatment of CythonSchrodingerSolver
    (qdsim_cython/solvers/schrodinger_solver.pyx:253-283): every boundary row
    of H and of M becomes the identity row (row zeroed, diagonal 1)."""
    L = A.tolil()
    for i in np.where(fixed)[0]:
        L[i, :] = 0
        L[i, i] = 1
    out = L.tocsr()
    out.sort_indices()
    return out


def eig_free_sm(H, M, fixed, k):
    """The k eigenvalues of smallest magnitude (the reference calls
    eigsh(..., which='SM'), schrodinger_solver.pyx:447-453) of the physical
    part of the row-replaced pencil, i.e. of the pencil on the free nodes
    (dense solve; test meshes only)."""
    import scipy.linalg as sl
    free = ~fixed
    Hf = H[free][:, free].toarray()
    Mf = M[free][:, free].toarray()
    E = sl.eigh(0.5 * (Hf + Hf.T), 0.5 * (Mf + Mf.T), eigvals_only=True)
    return np.sort(E[np.argsort(np.abs(E))[:k]])

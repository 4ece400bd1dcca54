"""FP64 reference gradients of L = sum_s w_s E_s (TEST INFRASTRUCTURE ONLY).

Hellmann-Feynman with M-normalised eigenvectors (M depends on neither V nor c):
  dL/dV_g = sum_s w_s psi_s^T (dH/dV_g) psi_s,  dH/dV_g = sum_{e, l: node g} A_e T_l
  dL/dc_e = sum_s w_s psi_{s,e}^T Khat_e psi_{s,e}
with the same quadrature tables as ``fem.element_matrices``.  Checked against
central finite differences of the oracle's eigenvalues in the tests.
"""
import numpy as np

from . import fem as F


def gradients(mesh, psi_nodal, weights):
    """psi_nodal [N, ns] (zeros on Dirichlet nodes), weights [ns]."""
    tab = F.ref_tables(mesh.order)
    A, g00, g01, g11 = F.element_geometry(mesh.nodes, mesh.elems)
    Pe = psi_nodal[mesh.elems]                                   # [E, k, ns]
    U = np.einsum('eis,ejs,s->eij', Pe, Pe, np.asarray(weights, float))
    Khat = (g00[:, None, None] * tab.Sxx + g01[:, None, None] * tab.Sxy
            + g11[:, None, None] * tab.Syy) * A[:, None, None]
    dLdc = np.einsum('eij,eij->e', Khat, U)
    Gl = A[:, None] * np.einsum('lij,eij->el', tab.T, U)          # [E, k]
    dLdV = np.zeros(mesh.num_nodes)
    np.add.at(dLdV, mesh.elems.ravel(), Gl.ravel())
    return dLdV, dLdc

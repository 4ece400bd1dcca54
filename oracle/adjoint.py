"""FP64 reference gradients of L = Re sum_s w_s E_s (TEST INFRASTRUCTURE ONLY).

Hellmann-Feynman with normalised eigenvectors (M depends on neither V nor c):
  dL/dV_g = Re sum_s w_s psi_s^T (dH/dV_g) psi_s,  dH/dV_g = sum_{e, l: node g} A_e T_l
  dL/dc_e = Re sum_s w_s psi_{s,e}^T Khat_e psi_{s,e}
with the same quadrature tables as ``fem.element_matrices``.  Real psi
(Hermitian pencil, psi^T M psi = 1) or complex psi of the complex-symmetric
open-system pencil H - i Wm (bilinear psi^T M psi = 1, no conjugation: the
left eigenvector of a complex-symmetric pencil is psi itself), with complex
weights w_s = dL/dRe E_s - i dL/dIm E_s.  Checked against central finite
differences of the oracle's eigenvalues in the tests.
"""
import numpy as np

from . import fem as F


def gradients(mesh, psi_nodal, weights):
    """psi_nodal [N, ns] real or complex (zeros on Dirichlet nodes), weights [ns]."""
    tab = F.ref_tables(mesh.order)
    A, g00, g01, g11 = F.element_geometry(mesh.nodes, mesh.elems)
    Pe = psi_nodal[mesh.elems]                                   # [E, k, ns]
    U = np.real(np.einsum('eis,ejs,s->eij', Pe, Pe, np.asarray(weights)))
    Khat = (g00[:, None, None] * tab.Sxx + g01[:, None, None] * tab.Sxy
            + g11[:, None, None] * tab.Syy) * A[:, None, None]
    dLdc = np.einsum('eij,eij->e', Khat, U)
    Gl = A[:, None] * np.einsum('lij,eij->el', tab.T, U)          # [E, k]
    dLdV = np.zeros(mesh.num_nodes)
    np.add.at(dLdV, mesh.elems.ravel(), Gl.ravel())
    return dLdV, dLdc


def bilinear_normalise(X, M):
    """Columns scaled so that x^T M x = 1 (complex-symmetric pencils)."""
    s = np.sqrt(np.einsum('is,is->s', X, M @ X))
    return X / s[None, :]

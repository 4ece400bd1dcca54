"""FP64 restatement of the P1 Poisson step (TEST INFRASTRUCTURE ONLY).

Follows ``qdsim_cython/solvers/poisson_solver.pyx``:
  * stiffness K_ij = sum_e eps_r(e) eps0 |T| grad(phi_i).grad(phi_j) with eps_r at
    the element centroid (:114-167, :169-196) -- without the m^2-scale area skip
    at :126 that drops every element of a nanometre mesh;
  * mass M_ij = |T|/12 (2 on the diagonal) (:198-211);
  * RHS = M (-rho_nodal) (:254-274, the reference's sign convention);
  * Dirichlet phi = V_p on x = 0 and V_n on x = Lx, natural (Neumann) elsewhere
    (:276-308); the reference replaces those rows by identity rows and calls
    spsolve (:240), which has the same solution as eliminating them;
  * electric field by one-sided / central differences on the node grid (:310-335).

Lengths in nm; eps0 = 8.854187817e-12 F/m (:28); rho in C/m^3; phi in V.
"""
import numpy as np
import scipy.sparse.linalg as spla

from . import fem as F

EPS0 = 8.854187817e-12
Q_E = 1.602176634e-19


def assemble(mesh, eps_r_elem):
    """K (eps_r weighted, dimensionless) and M (nm^2) on the full P1 pattern."""
    dm = F.dof_map(mesh, dirichlet=False)
    n = mesh.num_nodes
    Ke, Me, _, _ = F.element_matrices(mesh, np.asarray(eps_r_elem, float), None, None)
    K, M = F.assemble_csr(mesh.elems, dm, [Ke, Me], n)
    return K, M


def dirichlet_mask(mesh):
    x = mesh.nodes[:, 0]
    left = np.abs(x) < 1e-9 * mesh.Lx
    right = np.abs(x - mesh.Lx) < 1e-9 * mesh.Lx
    return left, right


def solve(mesh, eps_r_elem, rho_nodal, V_p, V_n, length_scale=1e-9):
    """phi (V) at every node.  rho_nodal in C/m^3 ([N] or [N, nrhs]);
    ``length_scale`` is the mesh unit in metres (1e-9 for nm, 1 for SI)."""
    K, M = assemble(mesh, eps_r_elem)
    rho = np.asarray(rho_nodal, float)
    one = rho.ndim == 1
    rho = rho.reshape(mesh.num_nodes, -1)
    # K_r phi = (l^2 / eps0) M (-rho), M in mesh units^2
    b = (length_scale ** 2 / EPS0) * (M @ (-rho))
    left, right = dirichlet_mask(mesh)
    fixed = left | right
    vp = np.broadcast_to(np.asarray(V_p, float), (rho.shape[1],))
    vn = np.broadcast_to(np.asarray(V_n, float), (rho.shape[1],))
    phi = np.zeros_like(b)
    phi[left] = vp
    phi[right] = vn
    free = ~fixed
    Kff = K[free][:, free].tocsc()
    rhs = b[free] - K[free][:, fixed] @ phi[fixed]
    phi[free] = spla.splu(Kff).solve(rhs)
    return phi[:, 0] if one else phi


def electric_field(phi, nx_pts, ny_pts, dx, dy):
    """Reference finite differences on the (ny_pts x nx_pts) node grid."""
    P = phi.reshape(ny_pts, nx_pts)
    Ex = np.empty_like(P)
    Ey = np.empty_like(P)
    Ex[:, 1:-1] = -(P[:, 2:] - P[:, :-2]) / (2 * dx)
    Ex[:, 0] = -(P[:, 1] - P[:, 0]) / dx
    Ex[:, -1] = -(P[:, -1] - P[:, -2]) / dx
    Ey[1:-1, :] = -(P[2:, :] - P[:-2, :]) / (2 * dy)
    Ey[0, :] = -(P[1, :] - P[0, :]) / dy
    Ey[-1, :] = -(P[-1, :] - P[-2, :]) / dy
    return Ex.ravel(), Ey.ravel()

"""FP64 restatement of QDSim's P1/P2/P3 finite-element Schrodinger assembly and
eigensolve.  TEST INFRASTRUCTURE ONLY (the checker, never the product path).

Units: lengths in nm, energies in eV.  The kinetic coefficient of an element is
``c_e = hbar^2 / (2 m*_e)`` in eV nm^2; ``C0 = hbar^2/(2 m0)`` = 0.0380998 eV nm^2.

Weak form (``backend/src/fem.cpp:924-989``), per element ``T``::

    H_ij = sum_q w_q |T| [ c_e grad(phi_i).grad(phi_j) + (V_h(x_q) - i W_h(x_q)) phi_i phi_j ]
    M_ij = sum_q w_q |T| phi_i phi_j

``V_h`` / ``W_h`` are the finite-element interpolants of nodal values, which is
what ``fem.cpp:930-934`` does when ``use_interpolation`` is set
(``interpolator->interpolate(x, y, potential_values)``).  The quadrature rules
are the full-precision tables the reference carries: P1 3-point
(``fem.cpp:843-847``), P2 7-point (``fem.cpp:787-803``), P3 12-point
(``fem.cpp:807-832``); weights are normalised to sum to one and multiplied by
the element area.  The CAP enters with the sign ``-iW`` so that decaying states
have Im E < 0 (``fem.cpp:974`` adds ``+i eta``).

Meshes follow ``backend/src/mesh.cpp:66-115`` (nx, ny are cells; each cell
(n0, n1, n2, n3) is split into (n0, n1, n2) and (n1, n3, n2)).  Local node
order follows ``backend/src/fe_interpolator.cpp:474-518``.  The reference's P3
mesh aliases both edge nodes onto one midpoint (``mesh.cpp:130-153``); here the
two edge nodes sit at 1/3 and 2/3 and the interior node at the centroid, and
all nodes are numbered row-major on the refined (p nx + 1) x (p ny + 1) lattice.
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np
import scipy.sparse as sp
import scipy.sparse.linalg as spla

# CODATA values as in qdsim_cython/solvers/schrodinger_solver.pyx:26-28
HBAR = 1.054571817e-34
M_E = 9.1093837015e-31
Q_E = 1.602176634e-19
K_B = 1.380649e-23
EPS0_REF = 8.854187817e-12          # qdsim_cython/solvers/poisson_solver.pyx:28
C0_EV_NM2 = HBAR * HBAR / (2.0 * M_E) / Q_E * 1e18

# ---------------------------------------------------------------------------
# Quadrature (barycentric lambda0, lambda1, lambda2; weights sum to 1)
# ---------------------------------------------------------------------------


def _rule_from_xi_eta(pts, wts):
    pts = np.asarray(pts, dtype=np.float64)
    lam = np.stack([1.0 - pts[:, 0] - pts[:, 1], pts[:, 0], pts[:, 1]], axis=1)
    w = np.asarray(wts, dtype=np.float64)
    return lam, w / w.sum()


def quadrature(order: int):
    """Quadrature points (barycentric) and area-fraction weights.

    P1: ``fem.cpp:843-847`` (interior 3-point rule, weight area/3).
    P2: ``fem.cpp:787-803`` (7-point, degree 5).
    P3: ``fem.cpp:807-832`` (12-point, degree 6).
    """
    if order == 1:
        lam = np.array([[1 / 6, 1 / 6, 2 / 3], [1 / 6, 2 / 3, 1 / 6], [2 / 3, 1 / 6, 1 / 6]])
        return lam, np.full(3, 1.0 / 3.0)
    if order == 2:
        pts = [(1 / 3, 1 / 3),
               (0.059715871789770, 0.470142064105115),
               (0.470142064105115, 0.059715871789770),
               (0.470142064105115, 0.470142064105115),
               (0.797426985353087, 0.101286507323456),
               (0.101286507323456, 0.797426985353087),
               (0.101286507323456, 0.101286507323456)]
        wts = [0.225000000000000] + [0.132394152788506] * 3 + [0.125939180544827] * 3
        return _rule_from_xi_eta(pts, wts)
    if order == 3:
        a, b = 0.249286745170910, 0.501426509658179
        c, d = 0.063089014491502, 0.873821971016996
        e, f, g = 0.310352451033785, 0.636502499121399, 0.053145049844816
        pts = [(a, a), (a, b), (b, a), (c, c), (c, d), (d, c),
               (e, f), (f, g), (g, e), (f, e), (e, g), (g, f)]
        wts = [0.116786275726379] * 3 + [0.050844906370207] * 3 + [0.082851075618374] * 6
        return _rule_from_xi_eta(pts, wts)
    raise ValueError(f"unsupported element order {order}")


def nodes_per_element(order: int) -> int:
    return {1: 3, 2: 6, 3: 10}[order]


# ---------------------------------------------------------------------------
# Shape functions in barycentric form (fe_interpolator.cpp:474-613)
# ---------------------------------------------------------------------------


def shape(order: int, lam: np.ndarray):
    """Values phi[i] and barycentric partials dphi[m][i] = d phi_i / d lambda_m."""
    l0, l1, l2 = lam
    if order == 1:
        phi = np.array([l0, l1, l2])
        d = np.zeros((3, 3))
        d[0, 0] = d[1, 1] = d[2, 2] = 1.0
        return phi, d
    if order == 2:
        phi = np.array([l0 * (2 * l0 - 1), l1 * (2 * l1 - 1), l2 * (2 * l2 - 1),
                        4 * l0 * l1, 4 * l1 * l2, 4 * l2 * l0])
        d = np.zeros((3, 6))
        d[0, 0] = 4 * l0 - 1
        d[1, 1] = 4 * l1 - 1
        d[2, 2] = 4 * l2 - 1
        d[0, 3], d[1, 3] = 4 * l1, 4 * l0
        d[1, 4], d[2, 4] = 4 * l2, 4 * l1
        d[2, 5], d[0, 5] = 4 * l0, 4 * l2
        return phi, d
    if order == 3:
        phi = np.array([
            0.5 * l0 * (3 * l0 - 1) * (3 * l0 - 2),
            0.5 * l1 * (3 * l1 - 1) * (3 * l1 - 2),
            0.5 * l2 * (3 * l2 - 1) * (3 * l2 - 2),
            4.5 * l0 * l1 * (3 * l0 - 1), 4.5 * l0 * l1 * (3 * l1 - 1),
            4.5 * l1 * l2 * (3 * l1 - 1), 4.5 * l1 * l2 * (3 * l2 - 1),
            4.5 * l2 * l0 * (3 * l2 - 1), 4.5 * l2 * l0 * (3 * l0 - 1),
            27 * l0 * l1 * l2])
        d = np.zeros((3, 10))
        for m, l in enumerate((l0, l1, l2)):
            d[m, m] = 0.5 * (27 * l * l - 18 * l + 2)
        # edge node pairs (i, j, node near i, node near j)
        for (i, j, ni, nj) in ((0, 1, 3, 4), (1, 2, 5, 6), (2, 0, 7, 8)):
            li, lj = lam[i], lam[j]
            # phi_ni = 4.5 li lj (3 li - 1)
            d[i, ni] = 4.5 * lj * (6 * li - 1)
            d[j, ni] = 4.5 * li * (3 * li - 1)
            # phi_nj = 4.5 li lj (3 lj - 1)
            d[i, nj] = 4.5 * lj * (3 * lj - 1)
            d[j, nj] = 4.5 * li * (6 * lj - 1)
        d[0, 9], d[1, 9], d[2, 9] = 27 * l1 * l2, 27 * l0 * l2, 27 * l0 * l1
        return phi, d
    raise ValueError(order)


# barycentric coordinates of the local nodes, times the order (integers)
LOCAL_NODES = {
    1: [(1, 0, 0), (0, 1, 0), (0, 0, 1)],
    2: [(2, 0, 0), (0, 2, 0), (0, 0, 2), (1, 1, 0), (0, 1, 1), (1, 0, 1)],
    3: [(3, 0, 0), (0, 3, 0), (0, 0, 3), (2, 1, 0), (1, 2, 0), (0, 2, 1), (0, 1, 2),
        (1, 0, 2), (2, 0, 1), (1, 1, 1)],
}


@dataclass
class RefTables:
    """Reference-element tables (area-fraction weighted sums over quadrature)."""
    order: int
    k: int
    Mr: np.ndarray      # [k,k]   sum_q w phi_i phi_j
    Sxx: np.ndarray     # [k,k]   sum_q w dxi_i dxi_j
    Sxy: np.ndarray     # [k,k]   sum_q w (dxi_i deta_j + deta_i dxi_j)
    Syy: np.ndarray     # [k,k]   sum_q w deta_i deta_j
    T: np.ndarray       # [k,k,k] sum_q w phi_l phi_i phi_j   (index l, i, j)
    Phi: np.ndarray     # [Q,k]
    w: np.ndarray       # [Q]


def ref_tables(order: int) -> RefTables:
    lam, w = quadrature(order)
    k = nodes_per_element(order)
    Q = len(w)
    Phi = np.zeros((Q, k))
    Dxi = np.zeros((Q, k))
    Deta = np.zeros((Q, k))
    for q in range(Q):
        phi, d = shape(order, lam[q])
        Phi[q] = phi
        Dxi[q] = d[1] - d[0]       # xi = lambda1, eta = lambda2, lambda0 = 1 - xi - eta
        Deta[q] = d[2] - d[0]
    Mr = np.einsum('q,qi,qj->ij', w, Phi, Phi)
    Sxx = np.einsum('q,qi,qj->ij', w, Dxi, Dxi)
    Sxy = np.einsum('q,qi,qj->ij', w, Dxi, Deta) + np.einsum('q,qi,qj->ij', w, Deta, Dxi)
    Syy = np.einsum('q,qi,qj->ij', w, Deta, Deta)
    T = np.einsum('q,ql,qi,qj->lij', w, Phi, Phi, Phi)
    return RefTables(order, k, Mr, Sxx, Sxy, Syy, T, Phi, w)


# ---------------------------------------------------------------------------
# Meshes
# ---------------------------------------------------------------------------


@dataclass
class Mesh:
    order: int
    nx: int            # cells
    ny: int
    Lx: float          # nm
    Ly: float
    nodes: np.ndarray  # [N,2] float64 (nm)
    elems: np.ndarray  # [E,k] int32
    boundary: np.ndarray  # [N] bool

    @property
    def num_nodes(self):
        return self.nodes.shape[0]

    @property
    def num_elements(self):
        return self.elems.shape[0]


def structured_mesh(order: int, nx: int, ny: int, Lx: float, Ly: float) -> Mesh:
    """Structured triangulation (``backend/src/mesh.cpp:66-115``) with P2/P3
    nodes on the refined lattice; P3 edge nodes at 1/3 and 2/3 (corrected)."""
    p = order
    NX, NY = p * nx + 1, p * ny + 1
    ix, iy = np.meshgrid(np.arange(NX), np.arange(NY))
    nodes = np.stack([ix.ravel() * (Lx / (p * nx)), iy.ravel() * (Ly / (p * ny))], axis=1)
    boundary = ((ix == 0) | (ix == NX - 1) | (iy == 0) | (iy == NY - 1)).ravel()
    # vertex lattice coordinates of the two triangles of every cell
    ci, cj = np.meshgrid(np.arange(nx), np.arange(ny))
    ci = ci.ravel()
    cj = cj.ravel()
    v00 = np.stack([ci, cj], 1) * p
    v10 = np.stack([ci + 1, cj], 1) * p
    v01 = np.stack([ci, cj + 1], 1) * p
    v11 = np.stack([ci + 1, cj + 1], 1) * p
    tri0 = (v00, v10, v01)          # (n0, n1, n2)
    tri1 = (v10, v11, v01)          # (n1, n3, n2)
    k = nodes_per_element(p)
    E = 2 * nx * ny
    elems = np.zeros((E, k), dtype=np.int64)
    for t, tri in enumerate((tri0, tri1)):
        for a, bc in enumerate(LOCAL_NODES[p]):
            lat = (bc[0] * tri[0] + bc[1] * tri[1] + bc[2] * tri[2]) // p
            elems[t::2, a] = lat[:, 1] * NX + lat[:, 0]
    return Mesh(p, nx, ny, float(Lx), float(Ly), nodes, elems.astype(np.int32), boundary)


# ---------------------------------------------------------------------------
# Element matrices and global assembly
# ---------------------------------------------------------------------------


def element_geometry(nodes, elems):
    """Area A and inverse metric J^-1 J^-T (g00, g01, g11) per element."""
    P0 = nodes[elems[:, 0]]
    P1 = nodes[elems[:, 1]]
    P2 = nodes[elems[:, 2]]
    a = P1[:, 0] - P0[:, 0]
    b = P2[:, 0] - P0[:, 0]
    c = P1[:, 1] - P0[:, 1]
    d = P2[:, 1] - P0[:, 1]
    det = a * d - b * c
    A = 0.5 * np.abs(det)
    # J = [[a, b], [c, d]];  J^-1 = [[d, -b], [-c, a]] / det
    # Ginv = J^-1 J^-T
    g00 = (d * d + b * b) / (det * det)
    g01 = -(d * c + b * a) / (det * det)
    g11 = (c * c + a * a) / (det * det)
    return A, g00, g01, g11


def element_matrices(mesh: Mesh, c_elem, V_nodal=None, W_nodal=None):
    """Element matrices Ke (with c), Me, Ve, We, each [E,k,k] float64."""
    tab = ref_tables(mesh.order)
    A, g00, g01, g11 = element_geometry(mesh.nodes, mesh.elems)
    cA = np.asarray(c_elem, dtype=np.float64) * A
    Ke = cA[:, None, None] * (g00[:, None, None] * tab.Sxx + g01[:, None, None] * tab.Sxy
                              + g11[:, None, None] * tab.Syy)
    Me = A[:, None, None] * tab.Mr
    Ve = None
    We = None
    if V_nodal is not None:
        Vl = np.asarray(V_nodal, dtype=np.float64)[mesh.elems]            # [E,k]
        Ve = A[:, None, None] * np.einsum('el,lij->eij', Vl, tab.T)
    if W_nodal is not None:
        Wl = np.asarray(W_nodal, dtype=np.float64)[mesh.elems]
        We = A[:, None, None] * np.einsum('el,lij->eij', Wl, tab.T)
    return Ke, Me, Ve, We


def dof_map(mesh: Mesh, dirichlet: bool = True):
    """Reduced DOF index per node (-1 for eliminated Dirichlet nodes)."""
    keep = ~mesh.boundary if dirichlet else np.ones(mesh.num_nodes, bool)
    dm = np.full(mesh.num_nodes, -1, dtype=np.int64)
    dm[keep] = np.arange(int(keep.sum()))
    return dm


def csr_pattern(elems, dm, n):
    """Sorted CSR pattern over reduced DOFs and the slot of every element
    entry (-1 where a row or column is eliminated)."""
    k = elems.shape[1]
    rows = np.repeat(dm[elems], k, axis=1).reshape(-1)
    cols = np.tile(dm[elems], (1, k)).reshape(-1)
    ok = (rows >= 0) & (cols >= 0)
    keys = rows[ok].astype(np.int64) * n + cols[ok]
    uniq, inv = np.unique(keys, return_inverse=True)
    indptr = np.zeros(n + 1, dtype=np.int64)
    np.add.at(indptr, (uniq // n) + 1, 1)
    indptr = np.cumsum(indptr)
    indices = (uniq % n).astype(np.int64)
    slot = np.full(rows.size, -1, dtype=np.int64)
    slot[ok] = inv
    return indptr, indices, slot.reshape(elems.shape[0], k, k)


def assemble_csr(elems, dm, Ae_list, n):
    """Sum element matrices into CSR matrices over the reduced DOFs ``dm``
    (``fem.cpp:116-151``: triplets + setFromTriplets).  Returns scipy CSR
    matrices with sorted indices on one common pattern (zeros kept)."""
    indptr, indices, slot = csr_pattern(elems, dm, n)
    s = slot.reshape(-1)
    ok = s >= 0
    nnz = indices.size
    out = []
    for Ae in Ae_list:
        v = Ae.reshape(-1)[ok]
        if np.iscomplexobj(v):
            data = (np.bincount(s[ok], weights=v.real, minlength=nnz)
                    + 1j * np.bincount(s[ok], weights=v.imag, minlength=nnz))
        else:
            data = np.bincount(s[ok], weights=v, minlength=nnz)
        out.append(sp.csr_matrix((data, indices.copy(), indptr.copy()), shape=(n, n)))
    return out


@dataclass
class Assembled:
    H: sp.csr_matrix      # real part of H (K + V)
    M: sp.csr_matrix
    Wm: sp.csr_matrix | None   # CAP matrix (H = H - i Wm)
    K: sp.csr_matrix
    dm: np.ndarray
    n: int


def assemble(mesh: Mesh, c_elem, V_nodal, W_nodal=None, dirichlet=True) -> Assembled:
    Ke, Me, Ve, We = element_matrices(mesh, c_elem, V_nodal, W_nodal)
    dm = dof_map(mesh, dirichlet)
    n = int(dm.max()) + 1
    mats = [Ke + Ve, Me, Ke] + ([We] if We is not None else [])
    out = assemble_csr(mesh.elems, dm, mats, n)
    H, M, K = out[0], out[1], out[2]
    Wm = out[3] if We is not None else None
    return Assembled(H, M, Wm, K, dm, n)


# ---------------------------------------------------------------------------
# Coefficient fields used by the benchmark configurations
# ---------------------------------------------------------------------------


def cap_profile(x, y, Lx, Ly, W0, L):
    """CAP amplitude W0 (d/L)^2 where d is the penetration depth into the
    layer of width L along the domain edge (zero in the interior).  The
    reference's ``physics.cpp:244-254`` ``cap()`` assumes centred coordinates;
    this profile is the [0,Lx]x[0,Ly] form used by the CAP configuration."""
    dist = np.minimum(np.minimum(x, Lx - x), np.minimum(y, Ly - y))
    d = np.clip(L - dist, 0.0, None)
    return W0 * (d / L) ** 2


def centroids(mesh: Mesh):
    P = mesh.nodes[mesh.elems[:, :3]]
    return P.mean(axis=1)


# ---------------------------------------------------------------------------
# Eigen solve (scipy shift-invert ARPACK + FP64 Rayleigh-Ritz refinement)
# ---------------------------------------------------------------------------


def eig_lowest(H, M, k, sigma=None, tol=1e-14):
    """k lowest eigenpairs of H x = E M x (real symmetric H, SPD M).

    The reference's Python path calls ``spla.eigsh(H, k, M=M, which='SM')``
    (``qdsim_cython/solvers/schrodinger_solver.pyx:447-453``); shift-invert
    around a point below the spectrum returns the same pairs far faster.  The
    converged block is refined by a dense FP64 Rayleigh-Ritz.  Eigenvectors
    are M-orthonormal (``schrodinger_solver.pyx:461-468``)."""
    H = sp.csr_matrix(H)
    M = sp.csr_matrix(M)
    if sigma is None:
        raise ValueError("pass sigma below the lowest eigenvalue (see sigma_below)")
    ncv = min(H.shape[0] - 1, max(2 * k + 1, 40))
    w, X = spla.eigsh(H, k=k, M=M, sigma=sigma, which='LM', tol=tol, ncv=ncv)
    # Rayleigh-Ritz refinement in FP64
    A = X.T @ (H @ X)
    B = X.T @ (M @ X)
    A = 0.5 * (A + A.T)
    B = 0.5 * (B + B.T)
    import scipy.linalg as sl
    w2, Y = sl.eigh(A, B)
    X = X @ Y
    idx = np.argsort(w2)
    w2 = w2[idx]
    X = X[:, idx]
    nrm = np.sqrt(np.einsum('ij,ij->j', X, M @ X))
    X = X / nrm
    # deterministic sign: largest-magnitude component positive
    s = np.sign(X[np.argmax(np.abs(X), axis=0), np.arange(X.shape[1])])
    s[s == 0] = 1
    return w2, X * s


def sigma_below(V_nodal, margin=0.05):
    """A shift below the spectrum of H = K + V: the interpolant of nodal V
    undershoots min(V) by at most a quarter of the range for P1-P3."""
    V = np.asarray(V_nodal)
    return float(V.min() - 0.25 * (V.max() - V.min()) - margin)


def eig_nearest_complex(H, M, k, sigma, tol=1e-13):
    """k eigenvalues of the complex-symmetric pencil (H, M) nearest ``sigma``
    by shift-invert ARPACK; bilinear normalisation x^T M x = 1."""
    H = sp.csc_matrix(H)
    M = sp.csc_matrix(M).astype(np.complex128)
    w, X = spla.eigs(H, k=k, M=M, sigma=sigma, which='LM', tol=tol)
    idx = np.argsort(np.abs(w - sigma))
    w = w[idx]
    X = X[:, idx]
    nrm = np.sqrt(np.einsum('ij,ij->j', X, M @ X))
    return w, X / nrm


def residuals(H, M, E, X):
    """Relative residual ||H x - E M x|| / (|E| ||M x||) per pair."""
    R = H @ X - (M @ X) * E
    return np.linalg.norm(R, axis=0) / (np.abs(E) * np.linalg.norm(M @ X, axis=0))


def subspace_angles(X, Y, M):
    """Largest principal angle between span(X) and span(Y) in the M inner product."""
    import scipy.linalg as sl
    L = np.linalg.cholesky(X.T @ (M @ X))
    Qx = X @ np.linalg.inv(L).T
    L = np.linalg.cholesky(Y.T @ (M @ Y))
    Qy = Y @ np.linalg.inv(L).T
    s = sl.svdvals(Qx.T @ (M @ Qy))
    return np.arccos(np.clip(s, -1.0, 1.0))


# ---------------------------------------------------------------------------
# Benchmark configurations (seeded synthetic inputs)
# ---------------------------------------------------------------------------


def dot_config_c1(seed=0, nx=100, ny=50, Lx=100.0, Ly=50.0):
    """Single Gaussian dot on P1: V = -0.3 exp(-r^2/(2 8^2)), centre within
    +-10 nm of the middle; m* = 0.041 m0 where V(centroid) < -0.15 eV else 0.067 m0."""
    rng = np.random.default_rng(seed)
    cx = Lx / 2 + rng.uniform(-10, 10)
    cy = Ly / 2 + rng.uniform(-10, 10)
    mesh = structured_mesh(1, nx, ny, Lx, Ly)

    def V(x, y):
        return -0.3 * np.exp(-((x - cx) ** 2 + (y - cy) ** 2) / (2 * 8.0 ** 2))

    Vn = V(mesh.nodes[:, 0], mesh.nodes[:, 1])
    cen = centroids(mesh)
    mstar = np.where(V(cen[:, 0], cen[:, 1]) < -0.15, 0.041, 0.067)
    c = C0_EV_NM2 / mstar
    return mesh, c, Vn


SWEEP_SEED = 20261203


def dot_config_sweep(i, base_seed=SWEEP_SEED, order=2, nx=None):
    """Dot i of the batched sweep: P2, nx ~ U{40..240}, ny = nx // 2, 1 nm cells,
    circular well of radius U[5,20] nm and depth U[0.1,0.5] eV centred within
    +-5 nm of the middle, m* 0.041 m0 inside (element centroid) / 0.067 outside."""
    rng = np.random.default_rng([base_seed, i])
    n = int(rng.integers(40, 241))
    if nx is not None:
        n = int(nx)
    ny = n // 2
    Lx, Ly = float(n), float(ny)
    R = rng.uniform(5.0, 20.0)
    depth = rng.uniform(0.1, 0.5)
    cx = Lx / 2 + rng.uniform(-5.0, 5.0)
    cy = Ly / 2 + rng.uniform(-5.0, 5.0)
    mesh = structured_mesh(order, n, ny, Lx, Ly)
    x, y = mesh.nodes[:, 0], mesh.nodes[:, 1]
    Vn = np.where((x - cx) ** 2 + (y - cy) ** 2 < R * R, -depth, 0.0)
    cen = centroids(mesh)
    inside = (cen[:, 0] - cx) ** 2 + (cen[:, 1] - cy) ** 2 < R * R
    mstar = np.where(inside, 0.041, 0.067)
    return mesh, C0_EV_NM2 / mstar, Vn

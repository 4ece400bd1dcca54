"""Drop-in for the C++ backend classes the reference's Python frontend drives.

``frontend/qdsim/simulator.py`` builds ``qdsim_cpp.Mesh(Lx, Ly, nx, ny,
element_order)`` (:228-232), ``qdsim_cpp.FEMSolver(mesh, m_star, V, cap,
sc_solver, order, use_mpi)`` with ``assemble_matrices``, ``get_H``, ``get_M``
(:746-766) and ``qdsim_cpp.EigenSolver(fem_solver)`` with ``solve``,
``get_eigenvalues``, ``get_eigenvectors`` (:808-818); the bindings are
backend/src/bindings.cpp:761-985, ``FEInterpolator(mesh)`` among them
(:779-809).  Importing this module as ``qdsim_cpp`` points that path at the
GPU library:

    from qdsim_b200 import frontend as qdsim_cpp

Semantics kept from the C++ classes (SI units in and out):
 - ``FEMSolver`` assembles every node (backend/src/fem.cpp:116-151 applies no
   boundary condition: natural boundaries), H = K + V + i int eta phi phi
   with the CAP callback as +i eta (fem.cpp:974), M the consistent mass.
 - ``EigenSolver`` solves the Hermitian part of the pencil: the C++ solver
   symmetrises L^-1 H L^-H and calls SelfAdjointEigenSolver
   (backend/src/solver.cpp:118-128), which drops the CAP term.  It returns the
   k lowest eigenvalues as complex numbers with zero imaginary part and the
   real parts of the M-normalised eigenvectors (solver.cpp:141-163).
 - ``FEMSolver.set_potential_values`` / ``use_interpolated_potential`` make the
   assembly use the finite-element interpolant of the given nodal potential
   (J) instead of the ``V`` callback (fem.cpp:441-462, :930-937).
 - ``FEInterpolator`` evaluates nodal fields at points on the GPU
   (``qd_fe_interpolate``): the reference's element scan becomes an O(1)
   cell lookup with the same containing element, and points outside the mesh
   take the nearest node's value and the reference's gradient estimate.
 - ``FEMSolver.adapt_mesh`` refines the mesh where the eigenvector varies
   fastest (``qdsim_b200.adapt``: the reference's gradient flags, red-green
   refinement) and reassembles on the refined, unstructured mesh.
 - ``potential``, ``charge_density``, ``effective_mass``, ``epsilon_r`` and
   ``cap`` are the callbacks of backend/src/physics.cpp the frontend hands to
   its solvers; ``potential`` and ``charge_density`` resample nodal fields
   through the ``FEInterpolator`` (one launch for all points when given
   arrays).
Internally the mesh is scaled to nm and energies to eV (c = hbar^2/(2 m*) in
eV nm^2), as the other drop-in solvers do; eigenvalues come back in J and
eigenvectors are M-normalised in m^2.
"""
from __future__ import annotations

import os

import numpy as np
import torch

from .batch import DeviceBatch, HostBatch
from .fem import C0_EV_NM2, FEMProblem, M_E, Q_E
from .adapt import TriMesh, refine, refinement_flags
from .interp import FieldInterpolator
from .mesh import StructuredMesh
from .solvers import _block_for, _eval
from .workloads import Dot


class Mesh:
    """Structured triangular mesh of [0, Lx] x [0, Ly] (meters) with nx x ny
    cells and P1/P2/P3 elements, in the node order of backend/src/mesh.cpp."""

    def __init__(self, Lx: float, Ly: float, nx: int, ny: int, element_order: int = 1):
        if element_order not in (1, 2, 3):
            raise ValueError("element_order must be 1, 2 or 3")
        self._Lx, self._Ly = float(Lx), float(Ly)
        self._si = StructuredMesh(int(element_order), int(nx), int(ny), self._Lx, self._Ly)
        self._nm = StructuredMesh(int(element_order), int(nx), int(ny), self._Lx * 1e9,
                                  self._Ly * 1e9)

    def get_nodes(self):
        return self._si.nodes.copy()

    def get_elements(self):
        return self._si.elems.copy()

    def get_num_nodes(self) -> int:
        return int(self._si.num_nodes)

    def get_num_elements(self) -> int:
        return int(self._si.num_elements)

    def get_element_order(self) -> int:
        return int(self._si.order)

    def get_lx(self) -> float:
        return self._Lx

    def get_ly(self) -> float:
        return self._Ly

    def get_nx(self) -> int:
        return int(self._si.nx)

    def get_ny(self) -> int:
        return int(self._si.ny)

    def is_refined(self) -> bool:
        """True once ``FEMSolver.adapt_mesh`` has replaced the structured mesh."""
        return isinstance(self._si, TriMesh)

    def _replace(self, si, nm):
        self._si, self._nm = si, nm

    getNumNodes = get_num_nodes
    getNumElements = get_num_elements
    getElementOrder = get_element_order


class FEMSolver:
    """H and M of a ``Mesh`` from the reference's callbacks: ``m_star(x, y)``
    in kg (element centroids), ``V(x, y)`` and ``cap(x, y)`` in J (nodes)."""

    def __init__(self, mesh: Mesh, m_star, V, cap, sc_solver=None, order=None,
                 use_mpi: bool = False, device="cuda"):
        if order is not None and int(order) != mesh.get_element_order():
            raise ValueError("order must match the mesh's element order")
        self.mesh = mesh
        self.m_star, self.V, self.cap = m_star, V, cap
        self.sc_solver = sc_solver
        self.device = torch.device(device)
        self._prob = None
        self._mats = None
        self._coef = None
        self._potential = np.zeros(mesh.get_num_nodes())
        self._use_interp = False
        self._interp = None

    def is_using_mpi(self) -> bool:
        return False

    def assemble_matrices(self):
        si, nm = self.mesh._si, self.mesh._nm
        cen = si.centroids()
        mstar = _eval(self.m_star, cen[:, 0], cen[:, 1])
        c = C0_EV_NM2 * (M_E / mstar)
        # the interpolated potential applies while it matches the mesh
        # (fem.cpp:934); after a refinement the V callback is used again
        if self._use_interp and self._potential.size == si.num_nodes:
            V_eV = self._potential / Q_E
        else:
            V_eV = _eval(self.V, si.nodes[:, 0], si.nodes[:, 1]) / Q_E
        eta_eV = _eval(self.cap, si.nodes[:, 0], si.nodes[:, 1]) / Q_E
        self._coef = (c, V_eV)
        self._prob = FEMProblem(nm, dirichlet=False, device=self.device)
        # Himag = -int W phi phi, so W = -eta gives the reference's +i eta
        self._mats = self._prob.assemble(c, V_eV, -eta_eV)

    def _need(self):
        if self._mats is None:
            raise RuntimeError("call assemble_matrices() first")

    def get_H(self):
        """Complex H (J) as a scipy CSR matrix over all nodes."""
        self._need()
        Hr = self._prob.to_scipy(self._mats["H"])
        Hi = self._prob.to_scipy(self._mats["Himag"])
        return ((Hr + 1j * Hi) * Q_E).tocsr()

    def get_M(self):
        """M (m^2) as a scipy CSR matrix over all nodes."""
        self._need()
        return (self._prob.to_scipy(self._mats["M"]) * 1e-18).tocsr()

    def adapt_mesh(self, eigenvector, threshold, cache_dir=""):
        """Refine the mesh where the nodal ``eigenvector`` varies fastest and
        reassemble (fem.cpp:470-542): elements whose least-squares gradient
        (in the mesh's units) exceeds ``threshold`` are red-refined, with a
        conforming red-green closure (``qdsim_b200.adapt``).  With a
        ``cache_dir`` the refined mesh is stored as mesh_<norm>.npz (<norm> the
        eigenvector's 2-norm, six decimals) and reused when that file exists.
        The refined mesh is unstructured: the interpolator locates points
        through a bucket grid over the original cells (qd_fe_interpolate_tri),
        and the eigensolve takes the Jacobi preconditioner instead of the DST
        one, which needs the lattice."""
        psi = np.real(np.asarray(eigenvector)).astype(np.float64).reshape(-1)
        si, nm = self.mesh._si, self.mesh._nm
        cache = (os.path.join(cache_dir, f"mesh_{np.linalg.norm(psi):.6f}.npz")
                 if cache_dir else None)
        if cache is not None and os.path.exists(cache):
            z = np.load(cache)
            args = (int(z["order"]), z["nodes"], z["elems"], z["boundary"])
            green = dict(green_pair=z["green_pair"], green_parent=z["green_parent"])
            si2 = TriMesh(*args, float(z["Lx"]), float(z["Ly"]), int(z["nx"]), int(z["ny"]),
                          **green)
            nm2 = TriMesh(args[0], args[1] * 1e9, args[2], args[3], si2.Lx * 1e9,
                          si2.Ly * 1e9, si2.nx, si2.ny, **green)
        else:
            flags = refinement_flags(si, psi, threshold)
            si2, nm2 = refine(si, flags), refine(nm, flags)
            if cache is not None:
                os.makedirs(cache_dir, exist_ok=True)
                np.savez(cache, order=si2.order, nodes=si2.nodes, elems=si2.elems,
                         boundary=si2.boundary, Lx=si2.Lx, Ly=si2.Ly, nx=si2.nx, ny=si2.ny,
                         green_pair=si2.green_pair, green_parent=si2.green_parent)
        self.mesh._replace(si2, nm2)
        self._interp = None
        self.assemble_matrices()

    def get_interpolator(self):
        if self._interp is None:
            self._interp = FEInterpolator(self.mesh, device=self.device)
        return self._interp

    def set_potential_values(self, potential_values):
        """Nodal potential (J) for the interpolated-potential assembly; the
        length must be the number of nodes (fem.cpp:441-449)."""
        v = np.asarray(potential_values, dtype=np.float64).reshape(-1)
        if v.size != self.mesh.get_num_nodes():
            raise ValueError("potential_values must have one value per mesh node")
        self._potential = v.copy()

    def use_interpolated_potential(self, enable):
        self._use_interp = bool(enable)


class FEInterpolator:
    """Field evaluation on a ``Mesh`` (backend/src/fe_interpolator.cpp) with the
    reference's method names; coordinates are in the mesh's units.  Every
    evaluation is one ``qd_fe_interpolate`` launch, and a host field is
    copied to the device on each call: the per-point methods suit a few
    points, while ``interpolate_vector`` / ``interpolate_points`` take whole
    arrays of points (and device fields) in one launch."""

    def __init__(self, mesh: Mesh, device="cuda"):
        self.mesh = mesh
        self._fi = FieldInterpolator(mesh._si, device=device)
        self._fz = FieldInterpolator(mesh._si, device=device, outside="zero")
        self._zeros = None

    def _one(self, x, y, field, gradient=False, element=False):
        return self._fi.evaluate([float(x)], [float(y)], field, gradient=gradient,
                                 element=element)

    def interpolate(self, x, y, field) -> float:
        return float(self._one(x, y, field)["value"][0])

    def interpolate_with_gradient(self, x, y, field):
        r = self._one(x, y, field, gradient=True)
        return (float(r["value"][0]), float(r["grad_x"][0]), float(r["grad_y"][0]))

    def interpolate_complex(self, x, y, values, component="real"):
        """A complex nodal field at (x, y), as the Cython wrapper's
        ``interpolate_complex`` (qdsim_cython/core/interpolator.pyx:107-150):
        ``"real"`` / ``"imag"`` interpolate that part, ``"abs"`` gives the
        modulus of the interpolated value.  Both parts are evaluated in one
        launch (two fields)."""
        if component not in ("real", "imag", "abs"):
            raise ValueError(f"Unknown component: {component}")
        z = np.asarray(values, dtype=np.complex128).reshape(-1)
        parts = np.stack([z.real, z.imag])
        v = self._fi.evaluate([float(x)], [float(y)], parts)["value"]
        re, im = float(v[0, 0]), float(v[1, 0])
        if component == "real":
            return re
        if component == "imag":
            return im
        return float(np.hypot(re, im))

    def interpolate_gradient(self, x, y, field):
        _, gx, gy = self.interpolate_with_gradient(x, y, field)
        return (gx, gy)

    def find_element(self, x, y) -> int:
        if self._zeros is None:
            self._zeros = torch.zeros(self.mesh.get_num_nodes(), dtype=torch.float64,
                                      device=self._fz.device)
        r = self._fz.evaluate([float(x)], [float(y)], self._zeros, element=True)
        return int(r["element"][0])

    find_containing_element = find_element

    def is_inside_domain(self, x, y) -> bool:
        return self.find_element(x, y) >= 0

    def interpolate_vector(self, x_points, y_points, field):
        """Values at many points (numpy array), one launch."""
        x = np.asarray(x_points, dtype=np.float64).reshape(-1)
        y = np.asarray(y_points, dtype=np.float64).reshape(-1)
        if x.size != y.size:
            raise ValueError("x_points and y_points must have same length")
        return self._fi.evaluate(x, y, field)["value"].cpu().numpy()

    def interpolate_points(self, x_points, y_points, field, gradient=False, zero_outside=False):
        """Values (and gradients) of one or more fields at many points as
        device tensors, one launch (``FieldInterpolator.evaluate``)."""
        fi = self._fz if zero_outside else self._fi
        return fi.evaluate(x_points, y_points, field, gradient=gradient, element=True)

    @staticmethod
    def compute_barycentric_coordinates(x, y, vertices):
        """(inside, [l0, l1, l2]) of (x, y) in the triangle ``vertices``
        (fe_interpolator.cpp:433-472): signed-area formula, inside when every
        coordinate is >= -1e-10."""
        (x0, y0), (x1, y1), (x2, y2) = [(float(v[0]), float(v[1])) for v in vertices[:3]]
        area = 0.5 * ((x1 - x0) * (y2 - y0) - (x2 - x0) * (y1 - y0))
        lam = [0.5 * ((x1 * y2 - x2 * y1) + (y1 - y2) * x + (x2 - x1) * y) / area,
               0.5 * ((x2 * y0 - x0 * y2) + (y2 - y0) * x + (x0 - x2) * y) / area,
               0.5 * ((x0 * y1 - x1 * y0) + (y0 - y1) * x + (x1 - x0) * y) / area]
        return (all(v >= -1e-10 for v in lam), lam)


class AdaptiveMesh:
    """The static refinement helpers bound as ``qdsim_cpp.AdaptiveMesh``
    (backend/src/bindings.cpp:1590-1608) on this module's ``Mesh``."""

    @staticmethod
    def compute_refinement_flags(mesh: Mesh, psi, threshold):
        """Elements whose least-squares gradient of the nodal ``psi`` (per
        metre) exceeds ``threshold`` (adaptive_mesh.cpp:431-494)."""
        return [bool(f) for f in refinement_flags(mesh._si, psi, threshold)]

    @staticmethod
    def refine_mesh(mesh: Mesh, refine_flags):
        """Refine the flagged elements of ``mesh`` in place (conforming
        red-green refinement, ``qdsim_b200.adapt.refine``)."""
        flags = np.asarray(refine_flags, dtype=bool)
        mesh._replace(refine(mesh._si, flags), refine(mesh._nm, flags))

    @staticmethod
    def compute_triangle_quality(mesh: Mesh, elem_idx: int) -> float:
        """4 sqrt(3) area / (sum of squared edge lengths): 1 for an
        equilateral triangle (adaptive_mesh.cpp:1323-1337)."""
        p = mesh._si.nodes[mesh._si.elems[int(elem_idx), :3]]
        l1 = float(np.linalg.norm(p[1] - p[0]))
        l2 = float(np.linalg.norm(p[2] - p[1]))
        l3 = float(np.linalg.norm(p[0] - p[2]))
        sp = 0.5 * (l1 + l2 + l3)
        area = np.sqrt(max(sp * (sp - l1) * (sp - l2) * (sp - l3), 0.0))
        return float(4.0 * np.sqrt(3.0) * area / (l1 * l1 + l2 * l2 + l3 * l3))

    @staticmethod
    def is_mesh_conforming(mesh: Mesh) -> bool:
        """False when an edge is shared by more than two triangles, the test
        the reference makes (adaptive_mesh.cpp:1339-1362)."""
        tri = mesh._si.elems[:, :3].astype(np.int64)
        a, b = tri, np.roll(tri, -1, axis=1)
        n = int(tri.max()) + 1
        keys = (np.minimum(a, b) * n + np.maximum(a, b)).ravel()
        return bool(np.unique(keys, return_counts=True)[1].max() <= 2)


# the elementary charge and the potential cap of backend/src/physics.cpp:69-141
_PHYS_Q = 1.602e-19
_MAX_POTENTIAL_EV = 100.0


def _field(mat, name):
    """A material property from a Material-like object or a mapping."""
    if isinstance(mat, dict):
        return float(mat[name])
    return float(getattr(mat, name))


def _out(v, scalar):
    return float(v) if scalar else v


def effective_mass(x, y, qd_mat, matrix_mat, R):
    """m_e of the dot inside the disc x^2 + y^2 <= R^2, of the matrix outside
    (physics.cpp:39-43); arrays are evaluated elementwise."""
    xa, ya = np.asarray(x, dtype=float), np.asarray(y, dtype=float)
    v = np.where(xa * xa + ya * ya <= R * R, _field(qd_mat, "m_e"), _field(matrix_mat, "m_e"))
    return _out(v, xa.ndim == 0)


def epsilon_r(x, y, p_mat, n_mat):
    """p-side permittivity for x < 0, n-side otherwise (physics.cpp:143-147)."""
    xa = np.asarray(x, dtype=float)
    v = np.where(xa < 0, _field(p_mat, "epsilon_r"), _field(n_mat, "epsilon_r"))
    return _out(v, xa.ndim == 0)


def cap(x, y, eta, Lx, Ly, d):
    """Absorbing-potential amplitude, quadratic in the distance past
    |x| = Lx/2 - d or |y| = Ly/2 - d, the larger of the two
    (physics.cpp:244-254)."""
    xa, ya = np.abs(np.asarray(x, dtype=float)), np.abs(np.asarray(y, dtype=float))
    ex = np.where(xa > Lx / 2 - d, eta * ((xa - Lx / 2) / d) ** 2, 0.0)
    ey = np.where(ya > Ly / 2 - d, eta * ((ya - Ly / 2) / d) ** 2, 0.0)
    return _out(np.maximum(ex, ey), xa.ndim == 0)


def potential(x, y, qd_mat, matrix_mat, R, type, phi, interpolator=None):
    """Dot potential plus the electrostatic potential phi resampled at (x, y)
    (physics.cpp:69-141), in J.  The dot term is -min(Delta_E_c, 100 eV)
    inside the disc ("square") or as a Gaussian of width R ("gaussian"); the
    electrostatic term is the finite-element interpolation of the nodal phi
    (volts, read as eV), clipped to +-100, or phi[0] clipped when there is no
    interpolator.  With a ``FEInterpolator`` of this module, arrays of points
    are resampled in one GPU launch."""
    xa, ya = np.asarray(x, dtype=float), np.asarray(y, dtype=float)
    scalar = xa.ndim == 0
    xa, ya = np.atleast_1d(xa), np.atleast_1d(ya)
    depth = min(_field(qd_mat, "Delta_E_c"), _MAX_POTENTIAL_EV)
    r2 = xa * xa + ya * ya
    if type == "square":
        v_qd = np.where(r2 <= R * R, -depth, 0.0)
    elif type == "gaussian":
        v_qd = -depth * np.exp(-r2 / (2 * R * R))
    else:
        v_qd = np.zeros_like(xa)
    ph = np.asarray(phi, dtype=float).reshape(-1)
    v_el = np.zeros_like(xa)
    first = (min(abs(ph[0]), _MAX_POTENTIAL_EV) * (1.0 if ph[0] >= 0 else -1.0)
             if ph.size else 0.0)
    if ph.size and interpolator is not None:
        try:
            v_el = _resample(interpolator, xa, ya, ph)
            v_el = np.where(np.abs(v_el) > _MAX_POTENTIAL_EV,
                            np.where(v_el >= 0, _MAX_POTENTIAL_EV, -_MAX_POTENTIAL_EV), v_el)
        except Exception:
            v_el = np.full_like(xa, first)
    elif ph.size:
        v_el = np.full_like(xa, first)
    v = v_qd * _PHYS_Q + v_el * _PHYS_Q
    return float(v[0]) if scalar else v


def _resample(interpolator, xa, ya, field):
    """``field`` at the points through ``interpolator``: one launch for all
    points with this module's FEInterpolator, point by point otherwise."""
    if isinstance(interpolator, FEInterpolator):
        return np.asarray(interpolator.interpolate_vector(xa, ya, field), dtype=float)
    return np.array([interpolator.interpolate(a, b, field) for a, b in zip(xa, ya)],
                    dtype=float)


def charge_density(x, y, n, p, n_interpolator=None, p_interpolator=None):
    """q (p - n) at (x, y) (physics.cpp:184-216): each carrier density is
    resampled through its interpolator, or is its first entry when there is
    no interpolator (or the interpolation fails), or 0 when empty."""
    xa, ya = np.asarray(x, dtype=float), np.asarray(y, dtype=float)
    scalar = xa.ndim == 0
    xa, ya = np.atleast_1d(xa), np.atleast_1d(ya)

    def density(field, interp):
        f = np.asarray(field, dtype=float).reshape(-1)
        if f.size == 0:
            return np.zeros_like(xa)
        if interp is not None:
            try:
                return _resample(interp, xa, ya, f)
            except Exception:
                pass
        return np.full_like(xa, f[0])

    v = _PHYS_Q * (density(p, p_interpolator) - density(n, n_interpolator))
    return float(v[0]) if scalar else v


class EigenSolver:
    """The k lowest levels of a ``FEMSolver``'s Hermitian pencil (K + V, M)."""

    def __init__(self, fem_solver: FEMSolver):
        self.fem = fem_solver
        self.eigenvalues = []
        self.eigenvectors = []

    def solve(self, num_eigenpairs: int = 10):
        fem = self.fem
        fem._need()
        nm = fem.mesh._nm
        c, V_eV = fem._coef
        k = int(min(num_eigenpairs, nm.num_nodes - 1))
        hb = HostBatch([Dot(nm, c, V_eV)], dirichlet=False)
        db = DeviceBatch(hb, fem.device)
        db.upload(non_blocking=False)
        db.assemble()
        db.check_status()
        # natural boundaries: the lowest level can sit at zero energy, so
        # errors are measured relative to max(|E|, 0.01 eV)
        E, X, _, _, _, _ = db.solve(k, b=_block_for(k), precision="mixed", tol=1e-9,
                                    max_iter=4000, allow_not_converged=False,
                                    eig_scale=0.01)
        E_J = E.cpu().numpy()[0] * Q_E
        psi = X.cpu().numpy() * 1e9          # M-normalised in nm^2 -> m^2
        self.eigenvalues = [complex(e, 0.0) for e in E_J]
        self.eigenvectors = [np.ascontiguousarray(psi[:, i]) for i in range(k)]

    def get_eigenvalues(self):
        return list(self.eigenvalues)

    def get_eigenvectors(self):
        return [v.copy() for v in self.eigenvectors]


__all__ = ["Mesh", "FEMSolver", "EigenSolver", "FEInterpolator", "AdaptiveMesh", "potential",
           "charge_density", "effective_mass", "epsilon_r", "cap"]

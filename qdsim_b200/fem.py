"""Finite-element problems on the GPU: CSR pattern (host C++), device-resident
mesh and coefficient arrays, and the warp-per-row assembly kernel.

Units are the library's scaled ones: lengths in nm, energies in eV, kinetic
coefficient ``c = hbar^2/(2 m*)`` in eV nm^2.  ``C0_EV_NM2`` converts a mass
ratio: ``c = C0_EV_NM2 * (m0 / m*)``.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np
import torch

from . import _native as N
from .mesh import StructuredMesh

HBAR = 1.054571817e-34
M_E = 9.1093837015e-31
Q_E = 1.602176634e-19
C0_EV_NM2 = HBAR * HBAR / (2.0 * M_E) / Q_E * 1e18


@dataclass
class Pattern:
    n: int
    nnz: int
    rowptr: np.ndarray
    col: np.ndarray
    adjptr: np.ndarray
    adj: np.ndarray
    cptr: np.ndarray
    contrib: np.ndarray
    slotcnt: np.ndarray


def build_pattern(elems: np.ndarray, dof_map: np.ndarray, n_dofs: int, num_nodes: int) -> Pattern:
    """CSR pattern over reduced DOFs plus the assembly plan (``qd_pattern_build``)."""
    L = N.lib()
    elems = np.ascontiguousarray(elems, dtype=np.int32)
    dof_map = np.ascontiguousarray(dof_map, dtype=np.int32)
    E, k = elems.shape
    nnz, nadj, ncon = C.c_int64(), C.c_int64(), C.c_int64()
    N.check(L.qd_pattern_build(num_nodes, E, k, N.ptr(elems), N.ptr(dof_map), n_dofs,
                               C.byref(nnz), C.byref(nadj), C.byref(ncon),
                               None, None, None, None, None, None, None), "qd_pattern_build")
    P = Pattern(n_dofs, nnz.value,
                np.empty(n_dofs + 1, np.int32), np.empty(nnz.value, np.int32),
                np.empty(n_dofs + 1, np.int32), np.empty(nadj.value, np.int32),
                np.empty(n_dofs + 1, np.int32), np.empty(ncon.value, np.uint8),
                np.empty(nnz.value, np.uint8))
    N.check(L.qd_pattern_build(num_nodes, E, k, N.ptr(elems), N.ptr(dof_map), n_dofs,
                               C.byref(nnz), C.byref(nadj), C.byref(ncon),
                               N.ptr(P.rowptr), N.ptr(P.col), N.ptr(P.adjptr), N.ptr(P.adj),
                               N.ptr(P.cptr), N.ptr(P.contrib), N.ptr(P.slotcnt)),
            "qd_pattern_build")
    return P


def node_adjacency(elems: np.ndarray, num_nodes: int):
    L = N.lib()
    elems = np.ascontiguousarray(elems, dtype=np.int32)
    E, k = elems.shape
    nadj = C.c_int64()
    N.check(L.qd_node_adjacency(num_nodes, E, k, N.ptr(elems), C.byref(nadj), None, None),
            "qd_node_adjacency")
    ptr = np.empty(num_nodes + 1, np.int32)
    adj = np.empty(nadj.value, np.int32)
    N.check(L.qd_node_adjacency(num_nodes, E, k, N.ptr(elems), C.byref(nadj), N.ptr(ptr),
                                N.ptr(adj)), "qd_node_adjacency")
    return ptr, adj


_PATTERN_CACHE: dict = {}


def dof_map_for(mesh, dirichlet: bool):
    keep = ~mesh.boundary if dirichlet else np.ones(mesh.num_nodes, bool)
    dm = np.full(mesh.num_nodes, -1, dtype=np.int32)
    dm[keep] = np.arange(int(keep.sum()), dtype=np.int32)
    return dm, int(keep.sum())


def stream_ptr(stream=None):
    s = stream if stream is not None else torch.cuda.current_stream()
    return C.c_void_p(s.cuda_stream)


class FEMProblem:
    """One mesh on the device with its CSR pattern and assembly plan.

    ``dirichlet=True`` eliminates the boundary nodes (homogeneous Dirichlet by
    symmetric elimination); ``False`` keeps every node (Poisson uses a row
    mask for inhomogeneous Dirichlet values instead).
    """

    def __init__(self, mesh: StructuredMesh, dirichlet: bool = True, device="cuda",
                 eliminate=None):
        """``eliminate`` (bool per node) overrides ``dirichlet`` with an explicit
        set of eliminated nodes."""
        self.mesh = mesh
        self.order = mesh.order
        self.device = torch.device(device)
        key = None
        if eliminate is not None:
            keep = ~np.asarray(eliminate, bool)
            self.dof_map = np.full(mesh.num_nodes, -1, dtype=np.int32)
            self.dof_map[keep] = np.arange(int(keep.sum()), dtype=np.int32)
            self.n = int(keep.sum())
        else:
            self.dof_map, self.n = dof_map_for(mesh, dirichlet)
            if isinstance(mesh, StructuredMesh):
                key = (mesh.shape_key(), dirichlet)
        if key is not None and key in _PATTERN_CACHE:
            self.pattern = _PATTERN_CACHE[key]
        else:
            self.pattern = build_pattern(mesh.elems, self.dof_map, self.n, mesh.num_nodes)
            if key is not None:
                _PATTERN_CACHE[key] = self.pattern
        dev = self.device
        t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)  # noqa: E731
        self.d_nodes = t(mesh.nodes.astype(np.float64))
        self.d_elems = t(mesh.elems)
        self.d_dofmap = t(self.dof_map)
        P = self.pattern
        self.d_rowptr, self.d_col = t(P.rowptr), t(P.col)
        self.d_adjptr, self.d_adj = t(P.adjptr), t(P.adj)
        self.d_cptr, self.d_contrib, self.d_slotcnt = t(P.cptr), t(P.contrib), t(P.slotcnt)
        self.d_status = torch.zeros(1, dtype=torch.int32, device=dev)
        self._nadj = None

    @property
    def nnz(self) -> int:
        return self.pattern.nnz

    def assemble(self, c_elem, V, W=None, mode: int = N.QD_ASM_FEM, out=None, stream=None,
                 check: bool = True):
        """Assemble H (real), M and optionally Himag on the device.

        ``c_elem`` is per element; ``V`` / ``W`` are nodal in FEM mode and ``V``
        is per element in the reference-compatible modes.  Returns a dict of
        device tensors sharing this problem's CSR pattern.
        """
        dev = self.device
        as_dev = lambda a: (a if isinstance(a, torch.Tensor) else torch.from_numpy(  # noqa: E731
            np.ascontiguousarray(a, dtype=np.float64))).to(dev, torch.float64).contiguous()
        c = as_dev(c_elem)
        v = as_dev(V)
        w = as_dev(W) if W is not None else None
        E = self.mesh.num_elements
        if c.numel() != E:
            raise ValueError("c_elem must have one value per element")
        if mode == N.QD_ASM_FEM and v.numel() != self.mesh.num_nodes:
            raise ValueError("V must be nodal in FEM mode")
        if mode != N.QD_ASM_FEM and v.numel() != E:
            raise ValueError("V must be per element in the reference-compatible modes")
        if out is None:
            out = {"H": torch.empty(self.nnz, dtype=torch.float64, device=dev),
                   "M": torch.empty(self.nnz, dtype=torch.float64, device=dev)}
            if w is not None:
                out["Himag"] = torch.empty(self.nnz, dtype=torch.float64, device=dev)
        self.d_status.zero_()
        N.check(N.lib().qd_assemble(
            self.order, mode, self.mesh.num_nodes, E, self.n,
            N.ptr(self.d_nodes), N.ptr(self.d_elems), N.ptr(c), N.ptr(v), N.ptr(w),
            N.ptr(self.d_rowptr), N.ptr(self.d_adjptr), N.ptr(self.d_adj), N.ptr(self.d_cptr),
            N.ptr(self.d_contrib), N.ptr(self.d_slotcnt), N.ptr(out["H"]), N.ptr(out["M"]),
            N.ptr(out.get("Himag")), N.ptr(self.d_status), stream_ptr(stream)), "qd_assemble")
        if check:
            flag = int(self.d_status.item())
            if flag:
                raise N.QDError(N.QD_ERR_DEGENERATE, f"qd_assemble (flag {flag})")
        return out

    def node_adjacency(self):
        if self._nadj is None:
            ptr, adj = node_adjacency(self.mesh.elems, self.mesh.num_nodes)
            self._nadj = (torch.from_numpy(ptr).to(self.device), torch.from_numpy(adj).to(self.device))
        return self._nadj

    def to_scipy(self, vals):
        """Host scipy CSR of a device value array on this pattern (tests/debug)."""
        import scipy.sparse as sp
        v = vals.detach().cpu().numpy() if isinstance(vals, torch.Tensor) else vals
        P = self.pattern
        return sp.csr_matrix((v, P.col.copy(), P.rowptr.copy()), shape=(self.n, self.n))

    def expand(self, x_reduced):
        """Reduced DOF vector(s) -> nodal (zeros on eliminated nodes)."""
        x = np.asarray(x_reduced)
        out = np.zeros((self.mesh.num_nodes,) + x.shape[1:], dtype=x.dtype)
        keep = self.dof_map >= 0
        out[keep] = x[self.dof_map[keep]]
        return out

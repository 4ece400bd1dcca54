"""Poisson step of the self-consistent loop on the GPU.

Same weak form and boundary conditions as
``qdsim_cython/solvers/poisson_solver.pyx`` (P1 stiffness with eps_r per
element, RHS = M (-rho), phi = V_p on x = 0 and V_n on x = Lx, natural
elsewhere), without its m^2-scale degenerate-area test that skips every
element of a nanometre mesh (:126).  Assembly uses the warp-per-row kernel
(c = eps_r, V = 0); the solve is the batched Jacobi-PCG over any number of
right-hand sides (bias points) sharing the stiffness matrix.

Units: node coordinates in nm, rho in C/m^3, phi in V.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from . import _native as N
from .fem import FEMProblem, stream_ptr

EPS0 = 8.854187817e-12     # qdsim_cython/solvers/poisson_solver.pyx:28


class PoissonProblem:
    def __init__(self, mesh, eps_r_elem, device="cuda"):
        if mesh.order != 1:
            raise ValueError("the Poisson step is P1")
        self.mesh = mesh
        self.fem = FEMProblem(mesh, dirichlet=False, device=device)
        self.device = self.fem.device
        out = self.fem.assemble(np.asarray(eps_r_elem, float), np.zeros(mesh.num_nodes))
        self.K = out["H"]
        self.M = out["M"]
        x = mesh.nodes[:, 0]
        self.left = np.abs(x) < 1e-9 * mesh.Lx
        self.right = np.abs(x - mesh.Lx) < 1e-9 * mesh.Lx
        self.d_fixed = torch.from_numpy((self.left | self.right).astype(np.int32)).to(self.device)
        self._ws = None
        self.last_iters = 0
        self.last_relres = 0.0

    def rhs(self, rho):
        """(1e-18/eps0) M (-rho) on the device; rho [N] or [N, nrhs] (C/m^3)."""
        r = rho if isinstance(rho, torch.Tensor) else torch.from_numpy(np.asarray(rho, np.float64))
        r = r.to(self.device, torch.float64).reshape(self.mesh.num_nodes, -1).contiguous()
        b = torch.empty_like(r)
        n, nrhs = r.shape
        N.check(N.lib().qd_csr_spmv(n, nrhs, N.ptr(self.fem.d_rowptr), N.ptr(self.fem.d_col),
                                    N.ptr(self.M), N.ptr(r), N.ptr(b), -1e-18 / EPS0,
                                    stream_ptr()), "qd_csr_spmv")
        return b

    def solve(self, rho, V_p, V_n, tol=1e-12, max_iter=20000, x0=None):
        """phi (V) at every node, [N] or [N, nrhs] (device tensor)."""
        b = self.rhs(rho)
        n, nrhs = b.shape
        vp = torch.as_tensor(np.broadcast_to(np.asarray(V_p, float), (nrhs,)).copy(),
                             device=self.device)
        vn = torch.as_tensor(np.broadcast_to(np.asarray(V_n, float), (nrhs,)).copy(),
                             device=self.device)
        X = (torch.zeros_like(b) if x0 is None
             else x0.to(self.device, torch.float64).reshape(n, nrhs).clone())
        X[torch.from_numpy(self.left).to(self.device)] = vp
        X[torch.from_numpy(self.right).to(self.device)] = vn
        L = N.lib()
        nbytes = C.c_size_t()
        N.check(L.qd_pcg_workspace_size(n, nrhs, C.byref(nbytes)), "qd_pcg_workspace_size")
        if self._ws is None or self._ws.numel() < nbytes.value:
            self._ws = torch.empty(nbytes.value, dtype=torch.uint8, device=self.device)
        iters = C.c_int32()
        relres = C.c_double()
        N.check(L.qd_pcg_solve(n, nrhs, N.ptr(self.fem.d_rowptr), N.ptr(self.fem.d_col),
                               N.ptr(self.K), N.ptr(b), N.ptr(X), N.ptr(self.d_fixed), float(tol),
                               int(max_iter), C.byref(iters), C.byref(relres), N.ptr(self._ws),
                               self._ws.numel(), stream_ptr()), "qd_pcg_solve")
        self.last_iters = iters.value
        self.last_relres = relres.value
        return X if nrhs > 1 else X[:, 0]

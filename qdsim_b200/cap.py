"""Open-system eigensolve with a complex absorbing potential (CAP).

The pencil is complex symmetric: A = H + i Himag with H = K + V and
Himag = -int W phi_i phi_j (W >= 0 the CAP amplitude), M real SPD; the
eigenvalues E - i Gamma lie in the lower half plane.  The reference has no
sparse solver for it: backend/src/schrodinger.cpp:699-818 (a12) factorises the
dense pencil and calls Eigen's ComplexEigenSolver, and its Python path only
appends a constant imaginary part to real eigenvalues
(qdsim_cython/solvers/schrodinger_solver.pyx:528-557).  The oracle is scipy's
shift-invert eigs on the same assembled pencil.

Method: block LOBPCG on the complex pencil for the ``nev`` eigenvalues of
smallest real part, then the ``k`` of them nearest the shift ``sigma``, in
``qd_cap_lobpcg_solve`` (qdsim_b200/csrc/cap_lobpcg.cu), every step on the
device:
 - Products AX, MX from ``qd_cap_spmm`` (one CSR pass for H, Himag, M).
 - Preconditioner: the tensor-core DST preconditioner of the real kinetic
   operator, applied to the real and imaginary parts as separate columns.
 - Rayleigh-Ritz with a Hermitian M-orthonormal basis of [X P W] (Cholesky of
   the diagonally scaled Gram matrix while it is well conditioned, else SVQB);
   the projected non-Hermitian 3b x 3b eigenproblem goes to Schur form by a
   Jacobi-like method on an 8-CTA cluster; the b Ritz pairs of smallest real
   part are kept.
 - Mixed form: FP32 vectors and products until the relative residuals reach
   ``tol32`` (or stop improving), then FP64 vectors warm-started from them.
   Plain form: FP64 throughout.  Gram sums and the projected problem are FP64.
 - Final eigenvalues are the bilinear Rayleigh quotients x^T A x / x^T M x
   (stationary for complex-symmetric pencils), eigenvectors are normalised
   x^T M x = 1 as the oracle does.
 - Completeness: the k selected eigenvalues are certified nearest sigma only if
   every unconverged Ritz value (all of real part above the converged ones)
   lies farther from sigma than the k-th selected one; ``info['complete']``.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np
import torch

from . import _native as N
from .eigen import DSTPreconditioner
from .fem import FEMProblem, stream_ptr


@dataclass
class CAPResult:
    E: np.ndarray            # complex [k], nearest sigma first
    X: torch.Tensor          # complex128 [n, k] (device), x^T M x = 1
    residual: np.ndarray     # [k] ||A x - E M x|| / (|E| ||M x||)
    info: dict


def _real_view(Z):
    """[n, m] complex (row-major) -> [n, 2m] real view."""
    return torch.view_as_real(Z).reshape(Z.shape[0], 2 * Z.shape[1])


class CAPProblem:
    """Device pencil (H, Himag, M) of one structured mesh with Dirichlet
    elimination, its FP32 copies and the DST preconditioner."""

    def __init__(self, mesh, c_elem, V, W, device="cuda", shift_ev: float = 0.02):
        self.device = torch.device(device)
        self.fem = FEMProblem(mesh, dirichlet=True, device=self.device)
        mats = self.fem.assemble(c_elem, V, W)
        self.H, self.M = mats["H"], mats["M"]
        self.G = mats.get("Himag")
        self.H32, self.M32 = self.H.float(), self.M.float()
        self.G32 = self.G.float() if self.G is not None else None
        self.n = self.fem.n
        spec = DSTPreconditioner.spec_for(mesh, c_elem, V, shift_ev)
        self.prec = DSTPreconditioner([spec], self.device) if spec is not None else None
        self._pws = None
        self._work = None

    def workspace(self, nbytes):
        """Solver workspace of at least nbytes (kept between solves)."""
        if self._work is None or self._work.numel() < nbytes:
            self._work = None
            self._work = torch.empty(max(nbytes, 256), dtype=torch.uint8, device=self.device)
        return self._work

    # -- kernels ---------------------------------------------------------------
    def spmm(self, X, AX, MX):
        """AX = A X, MX = M X for complex column blocks (views allowed: the
        innermost stride must be 1)."""
        b = X.shape[1]
        fp32 = X.dtype == torch.complex64
        for T in (X, AX, MX):
            if T.stride(1) != 1 or T.shape[0] != self.n:
                raise ValueError("cap spmm operands must be [n, b] with unit column stride")
        H, G, M = (self.H32, self.G32, self.M32) if fp32 else (self.H, self.G, self.M)
        N.check(N.lib().qd_cap_spmm(self.n, b, 1 if fp32 else 0, N.ptr(self.fem.d_rowptr),
                                    N.ptr(self.fem.d_col), N.ptr(H), N.ptr(G), N.ptr(M),
                                    N.ptr(X), X.stride(0), N.ptr(AX), N.ptr(MX), AX.stride(0),
                                    stream_ptr()), "qd_cap_spmm")

    def precondition(self, R):
        """W = T R (real and imaginary parts as separate columns)."""
        if self.prec is None:
            return R.clone()
        Rr = _real_view(R.contiguous())
        cols = Rr.shape[1]
        if cols < 4:
            pad = torch.zeros(self.n, 4, dtype=Rr.dtype, device=Rr.device)
            pad[:, :cols] = Rr
            return torch.view_as_complex(
                self._apply(pad, 4)[:, :cols].contiguous().view(self.n, -1, 2))
        out = self._apply(Rr.contiguous(), cols)
        return torch.view_as_complex(out.view(self.n, -1, 2))

    def _apply(self, Rr, cols):
        import ctypes as C
        L = N.lib()
        ro = np.array([0, self.n], np.int32)
        nb = C.c_size_t()
        N.check(L.qd_dst_precond_workspace_size(1, N.ptr(ro), cols, N.ptr(self.prec.desc),
                                                C.byref(nb)), "qd_dst_precond_workspace_size")
        if self._pws is None or self._pws.numel() < nb.value:
            self._pws = torch.empty(max(nb.value, 256), dtype=torch.uint8, device=self.device)
        out = torch.empty_like(Rr)
        N.check(L.qd_dst_precond_apply(1, N.ptr(ro), cols, 1 if Rr.dtype == torch.float32 else 0,
                                       N.ptr(self.prec.desc), N.ptr(self.prec.d_mats), N.ptr(Rr),
                                       N.ptr(out), N.ptr(self._pws), self._pws.numel(),
                                       stream_ptr()), "qd_dst_precond_apply")
        return out


def solve_nearest(prob: CAPProblem, k: int = 20, sigma: float = -0.05, nev: int = 40,
                  b: int = 48, precision: str = "mixed", tol: float = 1e-9, tol32: float = 1e-4,
                  max_iter: int = 2000, seed: int = 1234, eig_scale: float = 0.01,
                  X0: torch.Tensor | None = None) -> CAPResult:
    """The k eigenvalues nearest sigma from the nev lowest (by real part),
    by ``qd_cap_lobpcg_solve`` on the device (block b, even, <= 48)."""
    if precision not in ("mixed", "fp64"):
        raise ValueError("precision must be 'mixed' or 'fp64'")
    if X0 is not None and precision != "fp64":
        raise ValueError("a start block is taken by the FP64 form only")
    L = N.lib()
    pm = N.QD_PREC_MIXED if precision == "mixed" else N.QD_PREC_FP64
    desc = prob.prec.desc if prob.prec is not None else None
    nb = C.c_size_t()
    N.check(L.qd_cap_lobpcg_workspace_size(prob.n, b, pm, N.ptr(desc), C.byref(nb)),
            "qd_cap_lobpcg_workspace_size")
    work = prob.workspace(nb.value)
    E = np.zeros(2 * k)
    res = np.zeros(k)
    info = np.zeros(1, dtype=N.CAP_INFO_DTYPE)
    Xout = torch.empty(prob.n, k, dtype=torch.complex128, device=prob.device)
    x0 = None
    if X0 is not None:
        x0 = X0.to(prob.device, torch.complex128).contiguous()
        if tuple(x0.shape) != (prob.n, b):
            raise ValueError("X0 must be [n, b]")
    st = L.qd_cap_lobpcg_solve(
        prob.n, N.ptr(prob.fem.d_rowptr), N.ptr(prob.fem.d_col), N.ptr(prob.H), N.ptr(prob.G),
        N.ptr(prob.M), N.ptr(prob.H32), N.ptr(prob.G32), N.ptr(prob.M32), N.ptr(desc),
        N.ptr(prob.prec.d_mats) if prob.prec is not None else None, b, nev, k, sigma, tol, tol32,
        max_iter, pm, eig_scale, seed, N.ptr(x0), N.ptr(E), N.ptr(Xout), N.ptr(res),
        N.ptr(info), N.ptr(work), work.numel(), stream_ptr())
    N.check(st, "qd_cap_lobpcg_solve", allow=(N.QD_ERR_NOT_CONVERGED,))
    f = info[0]
    sel = int(f["selected"])
    out = {"block": b, "nev": nev, "precision": precision,
           "iters_fp32": int(f["iters_fp32"]), "iters_fp64": int(f["iters_fp64"]),
           "iterations": int(f["iters_fp32"] + f["iters_fp64"]),
           "converged": int(f["converged"]), "complete": bool(f["complete"]),
           "kth_distance": float(f["kth_distance"]),
           "unconverged_bound": float(f["unconverged_bound"]),
           "max_residual": float(f["max_residual"]),
           "schur_sweeps_max": int(f["schur_sweeps_max"]),
           "schur_unconverged": int(f["schur_unconverged"]),
           "status": N.status_string(st)}
    if precision == "mixed":
        out["fp32_residual"] = float(f["fp32_residual"])
    Ec = E[0::2] + 1j * E[1::2]
    return CAPResult(Ec[:sel].copy(), Xout[:, :sel], res[:sel].copy(), out)


class CAPSolver:
    """The ``k`` eigenvalues of the CAP pencil nearest ``sigma`` (device
    assembly, ``qd_cap_spmm`` products, tensor-core DST preconditioner)."""

    def __init__(self, mesh, c_elem, V, W, device="cuda", shift_ev: float = 0.02):
        self.prob = CAPProblem(mesh, c_elem, V, W, device=device, shift_ev=shift_ev)

    def solve(self, k: int = 20, sigma: float = -0.05, **kw) -> CAPResult:
        return solve_nearest(self.prob, k, sigma, **kw)

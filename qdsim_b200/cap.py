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
smallest real part, then the ``k`` of them nearest the shift ``sigma``.
 - Products AX, MX from ``qd_cap_spmm`` (one CSR pass for H, Himag, M).
 - Preconditioner: the tensor-core DST preconditioner of the real kinetic
   operator, applied to the real and imaginary parts as separate columns.
 - Rayleigh-Ritz with a Hermitian M-orthonormal basis of [X P W] (Cholesky of
   the diagonally scaled Gram matrix while it is well conditioned, else SVQB)
   and the projected non-Hermitian eigenproblem solved in FP64 on the host
   (3b x 3b, LAPACK); the b Ritz pairs of smallest real part are kept.
 - Mixed form: FP32 vectors and products until the relative residuals reach
   ``tol32`` (or stop improving), then FP64 vectors warm-started from them.
   Plain form: FP64 throughout.
 - Final eigenvalues are the bilinear Rayleigh quotients x^T A x / x^T M x
   (stationary for complex-symmetric pencils), eigenvectors are normalised
   x^T M x = 1 as the oracle does.
 - Completeness: the k selected eigenvalues are certified nearest sigma only if
   every unconverged Ritz value (all of real part above the converged ones)
   lies farther from sigma than the k-th selected one; ``info['complete']``.
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np
import torch
from scipy.linalg import solve_triangular
from threadpoolctl import threadpool_limits

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


def _orthonormaliser(GM, drop):
    """B with B^H GM B = I: Cholesky of the diagonally scaled Gram matrix when
    its smallest pivot shows the basis is well conditioned (condition number
    below ~1e6), else SVQB, which also drops dependent directions."""
    d = np.sqrt(np.maximum(GM.diagonal().real, 0.0))
    if np.all(d > 0.0):
        Gs = GM / d[:, None] / d[None, :]
        try:
            L = np.linalg.cholesky(0.5 * (Gs + Gs.conj().T))
        except np.linalg.LinAlgError:
            L = None
        if L is not None and np.min(np.abs(L.diagonal())) ** 2 > 1e-6:
            Linv = solve_triangular(L, np.eye(L.shape[0]), lower=True)
            return Linv.conj().T / d[:, None]
    return _svqb(GM, drop)


def _svqb(GM, drop):
    """Hermitian M-orthonormalising transform of a basis from its Gram
    matrix: B with B^H GM B = I on the numerically independent directions."""
    d = np.sqrt(np.maximum(GM.diagonal().real, 0.0))
    ok = d > 0.0
    dinv = np.where(ok, 1.0 / np.where(ok, d, 1.0), 0.0)
    Gs = GM * dinv[:, None] * dinv[None, :]
    Gs = 0.5 * (Gs + Gs.conj().T)
    lam, U = np.linalg.eigh(Gs)
    keep = lam > drop * max(lam[-1], 1e-300)
    return (dinv[:, None] * U[:, keep]) / np.sqrt(lam[keep])[None, :]


class _Block:
    """Basis buffers S = [X P W], AS, MS (complex, [n, 3b]) of one precision."""

    def __init__(self, n, b, dtype, device):
        z = lambda: torch.zeros(n, 3 * b, dtype=dtype, device=device)  # noqa: E731
        self.S, self.AS, self.MS = z(), z(), z()


def lobpcg_cap(prob: CAPProblem, b: int, nev: int, tol: float, max_iter: int,
               dtype=torch.complex128, X0=None, seed: int = 1234, eig_scale: float = 0.01,
               stall: int = 0, on_iter=None):
    """Block LOBPCG on (A, M) for the nev eigenvalues of smallest real part.

    Returns (theta [b] complex numpy sorted by real part, X [n, b], AX, MX,
    residuals [b], iterations).  With ``stall`` > 0 the iteration also stops
    when the largest of the first nev residuals has not decreased for that
    many iterations (the FP32 phase's hand-over)."""
    n, dev = prob.n, prob.device
    drop = 1e-6 if dtype == torch.complex64 else 1e-14
    cur, nxt = _Block(n, b, dtype, dev), _Block(n, b, dtype, dev)
    if X0 is None:
        g = torch.Generator(device="cpu").manual_seed(seed)
        X0 = torch.view_as_complex(torch.randn(n, b, 2, generator=g, dtype=torch.float64))
    cur.S[:, :b] = X0.to(dev, dtype)
    X, AX, MX = cur.S[:, :b], cur.AS[:, :b], cur.MS[:, :b]
    prob.spmm(X, AX, MX)
    # initial Rayleigh-Ritz on span(X)
    Y, theta = _rr(cur, b, b, 0, drop)
    _combine(cur, nxt, Y, b, b, 0, with_p=False)
    cur, nxt = nxt, cur
    prob.spmm(cur.S[:, :b], cur.AS[:, :b], cur.MS[:, :b])
    npc = 0
    best, since = math.inf, 0
    res = np.full(b, np.inf)
    it = 0
    for it in range(1, max_iter + 1):
        X, AX, MX = cur.S[:, :b], cur.AS[:, :b], cur.MS[:, :b]
        th = torch.from_numpy(theta).to(dev, dtype)
        R = AX - MX * th[None, :]
        rn = torch.linalg.vector_norm(R, dim=0).double().cpu().numpy()
        mn = torch.linalg.vector_norm(MX, dim=0).double().cpu().numpy()
        res = rn / (np.maximum(mn, 1e-300) * np.maximum(np.abs(theta), eig_scale))
        if on_iter is not None:
            on_iter(it, theta, res)
        worst = float(res[:nev].max())
        if worst <= tol:
            break
        if stall:
            if worst < 0.9 * best:
                best, since = worst, 0
            else:
                since += 1
                if since >= stall:
                    break
        act = np.nonzero(res > tol)[0]
        act = act if act.size >= 2 else np.arange(b - 2, b)
        m = int(act.size)
        Wc = prob.precondition(R[:, torch.from_numpy(act).to(dev)])
        w0 = b + npc
        cur.S[:, w0:w0 + m] = Wc
        prob.spmm(cur.S[:, w0:w0 + m], cur.AS[:, w0:w0 + m], cur.MS[:, w0:w0 + m])
        Y, theta = _rr(cur, b, b + npc + m, npc, drop)
        _combine(cur, nxt, Y, b, b + npc + m, npc, with_p=True)
        cur, nxt = nxt, cur
        npc = b
        # explicit products of the new X (P's products are combined)
        prob.spmm(cur.S[:, :b], cur.AS[:, :b], cur.MS[:, :b])
    X, AX, MX = cur.S[:, :b], cur.AS[:, :b], cur.MS[:, :b]
    return theta, X.clone(), AX.clone(), MX.clone(), res, it


def _rr(blk: _Block, b, used, npc, drop):
    """Ritz pairs of (A, M) on span S[:, :used]: (Y [used, b] device, theta)."""
    S = blk.S[:, :used]
    GM = (S.mH @ blk.MS[:, :used]).to(torch.complex128).cpu().numpy()
    GA = (S.mH @ blk.AS[:, :used]).to(torch.complex128).cpu().numpy()
    # the projected problem is at most 3b x 3b: one BLAS thread (a threaded
    # BLAS on matrices this small only contends with the host's other work)
    with threadpool_limits(limits=1, user_api="blas"):
        return _rr_small(GM, GA, b, drop, blk.S)


def _rr_small(GM, GA, b, drop, like):
    Bm = _orthonormaliser(0.5 * (GM + GM.conj().T), drop)
    C = Bm.conj().T @ GA @ Bm
    w, V = np.linalg.eig(C)
    order = np.argsort(w.real, kind="stable")[:b]
    Y = Bm @ V[:, order]
    # Hermitian M-normalise the Ritz vectors (x^H M x = 1)
    nrm = np.sqrt(np.maximum(np.sum(Y.conj() * (GM @ Y), axis=0).real, 1e-300))
    Y = Y / nrm[None, :]
    return torch.from_numpy(Y).to(like.device, like.dtype), w[order]


def _combine(cur: _Block, nxt: _Block, Y, b, used, npc, with_p):
    """nxt.X = cur.S Y; nxt.P = cur.S[:, b:] Y[b:] (and the same for AS, MS)."""
    for src, dst in ((cur.S, nxt.S), (cur.AS, nxt.AS), (cur.MS, nxt.MS)):
        dst[:, :b].copy_(src[:, :used] @ Y)
        if with_p:
            dst[:, b:2 * b].copy_(src[:, b:used] @ Y[b:])


def solve_nearest(prob, k: int = 20, sigma: float = -0.05, nev: int = 40, b: int = 48,
                  precision: str = "mixed", tol: float = 1e-9, tol32: float = 1e-4,
                  max_iter: int = 2000, seed: int = 1234, eig_scale: float = 0.01) -> CAPResult:
    """The k eigenvalues nearest sigma from the nev lowest (by real part) of a
    problem exposing ``n``, ``device``, ``spmm`` and ``precondition``."""
    info = {"block": b, "nev": nev, "precision": precision}
    X0 = None
    it32 = 0
    if precision == "mixed":
        _, X, _, _, res32, it32 = lobpcg_cap(prob, b, nev, tol32, max_iter, dtype=torch.complex64,
                                             seed=seed, eig_scale=eig_scale, stall=8)
        X0 = X.to(torch.complex128)
        info["fp32_residual"] = float(res32[:nev].max())
    elif precision != "fp64":
        raise ValueError("precision must be 'mixed' or 'fp64'")
    th, X, AX, MX, res, it64 = lobpcg_cap(prob, b, nev, tol, max_iter, dtype=torch.complex128,
                                          X0=X0, seed=seed, eig_scale=eig_scale)
    info.update(iters_fp32=int(it32), iters_fp64=int(it64), iterations=int(it32 + it64))
    E, Xn, rres, sel = nearest_from_block(th, X, AX, MX, res, k, sigma, nev, tol)
    info.update(sel)
    return CAPResult(E, Xn, rres, info)


def nearest_from_block(theta, X, AX, MX, res, k, sigma, nev, tol):
    """Bilinear Rayleigh quotients of the converged block columns, x^T M x = 1
    normalisation, the k nearest sigma and the completeness check."""
    xtax = (X * AX).sum(dim=0)
    xtmx = (X * MX).sum(dim=0)
    E = (xtax / xtmx).cpu().numpy()
    s = torch.sqrt(xtmx)
    Xn, AXn, MXn = X / s[None, :], AX / s[None, :], MX / s[None, :]
    Et = torch.from_numpy(E).to(X.device)
    R = AXn - MXn * Et[None, :]
    rres = (torch.linalg.vector_norm(R, dim=0) /
            (torch.linalg.vector_norm(MXn, dim=0) * torch.abs(Et))).cpu().numpy()
    conv = np.asarray(res) <= tol
    conv[nev:] = False
    idx_c = np.nonzero(conv)[0]
    pick = idx_c[np.argsort(np.abs(E[idx_c] - sigma), kind="stable")[:k]]
    dk = float(np.abs(E[pick] - sigma).max()) if pick.size else math.inf
    unconv = np.nonzero(~conv)[0]
    bound = float(np.asarray(theta)[unconv].real.min() - sigma) if unconv.size else math.inf
    sel = dict(converged=int(conv.sum()), complete=bool(pick.size == k and dk < bound),
               kth_distance=dk, unconverged_bound=bound,
               max_residual=float(rres[pick].max()) if pick.size else math.inf)
    return E[pick], Xn[:, torch.from_numpy(pick).to(X.device)], rres[pick], sel


class CAPSolver:
    """The ``k`` eigenvalues of the CAP pencil nearest ``sigma`` (device
    assembly, ``qd_cap_spmm`` products, tensor-core DST preconditioner)."""

    def __init__(self, mesh, c_elem, V, W, device="cuda", shift_ev: float = 0.02):
        self.prob = CAPProblem(mesh, c_elem, V, W, device=device, shift_ev=shift_ev)

    def solve(self, k: int = 20, sigma: float = -0.05, **kw) -> CAPResult:
        return solve_nearest(self.prob, k, sigma, **kw)

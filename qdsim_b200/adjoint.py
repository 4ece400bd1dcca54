"""Adjoint gradients of eigenvalue losses (``qd_adjoint``) and
``torch.autograd.Function``s that make eigenvalues differentiable with
respect to nodal V and per-element inverse effective mass.

Closed system (``lowest_eigenvalues``): for L = sum_s w_s E_s with
M-normalised eigenvectors (M depends on neither V nor m*),
dE_s/dV = psi_s^T (dH/dV) psi_s and dE_s/dc_e = psi_s^T Khat_e psi_s,
c_e = C0 (m0/m*_e).

Open system with a complex absorbing potential (``nearest_eigenvalues``): the
pencil A = H + i Himag is complex symmetric, its eigenvectors are normalised
bilinearly (x^T M x = 1, no conjugation), the left eigenvector is x itself and
dE_s/dp = x_s^T (dH/dp) x_s.  A real loss of the complex eigenvalues has
dL/dp = Re sum_s w_s dE_s/dp with w_s = dL/dRe E_s - i dL/dIm E_s (the
conjugate of torch's complex gradient).

Degenerate levels: a single E_s of a degenerate cluster is not
differentiable, but any sum over the whole cluster is, and its gradient is
the same for every normalised basis of the cluster's eigenspace.  The
weights inside a cluster (levels within ``degenerate_rtol`` of each other,
relative to the largest |E|) are replaced by their mean, which leaves
cluster sums unchanged and is the basis-independent choice otherwise.  The
solves return one level beyond those asked for, so a cluster cut by the
last requested level is detected: its gradient would depend on the basis
the solver returned, and a ``RuntimeWarning`` says so.
"""
from __future__ import annotations

import warnings

import numpy as np
import torch

from . import _native as N
from .batch import DeviceBatch, HostBatch
from .fem import C0_EV_NM2, FEMProblem, stream_ptr
from .workloads import Dot


def clusters(E, degenerate_rtol=1e-8):
    """Groups of (real or complex) levels within degenerate_rtol * max|E| of
    one another, transitively closed; a list of index arrays."""
    E = np.asarray(E)
    n = len(E)
    scale = max(1e-12, float(np.abs(E).max())) if n else 1.0
    parent = list(range(n))

    def find(i):
        while parent[i] != i:
            parent[i] = parent[parent[i]]
            i = parent[i]
        return i

    for i in range(n):
        for j in range(i + 1, n):
            if abs(E[i] - E[j]) <= degenerate_rtol * scale:
                parent[find(i)] = find(j)
    groups = {}
    for i in range(n):
        groups.setdefault(find(i), []).append(i)
    return [np.array(g) for g in groups.values()]


def cluster_weights(E, w, degenerate_rtol=1e-8, E_next=None):
    """Weights averaged over each degenerate cluster of E.  ``E_next``: the
    level(s) just beyond E; when one of them belongs to a cluster of E whose
    weights are not all zero, the cluster is cut and a RuntimeWarning is
    issued."""
    E = np.asarray(E)
    w = np.asarray(w).copy()
    allE = E if E_next is None else np.concatenate([E, np.atleast_1d(E_next)])
    for g in clusters(allE, degenerate_rtol):
        inside = g[g < len(E)]
        if inside.size == 0:
            continue
        if inside.size < g.size and np.any(w[inside] != 0):
            warnings.warn("a degenerate cluster extends past the last requested level; its "
                          "gradient depends on the eigenvector basis (request more levels)",
                          RuntimeWarning, stacklevel=3)
        if inside.size > 1:
            w[inside] = w[inside].mean()
    return w


class _Outputs:
    """Preallocated gradient arrays and the element-pass scratch of one
    problem (reused between calls)."""

    def __init__(self):
        self.key = None
        self.dV = self.dc = self.work = None

    def get(self, m, dev):
        key = (m.num_nodes, m.num_elements, str(dev))
        if self.key != key:
            self.dV = torch.empty(m.num_nodes, dtype=torch.float64, device=dev)
            self.dc = torch.empty(m.num_elements, dtype=torch.float64, device=dev)
            self.work = torch.empty(m.elems.size, dtype=torch.float64, device=dev)
            self.key = key
        return self.dV, self.dc, self.work


def energy_gradients(prob: FEMProblem, psi_reduced: torch.Tensor, weights, stream=None,
                     out=None):
    """dL/dV (nodal) and dL/dc (per element) on the device (an element pass
    and a node gather).

    ``psi_reduced``: [n_dofs, ns] real (Hermitian pencil, M-normalised) or
    complex (complex-symmetric pencil, x^T M x = 1); ``weights``: ns real or
    complex values (w_s of L = Re sum_s w_s E_s).  ``out``: optional
    (dV, dc) float64 device tensors to write into; by default arrays cached
    on ``prob`` are reused, so the returned tensors are overwritten by the
    next call for the same problem."""
    dev = prob.device
    psi = psi_reduced.to(dev)
    cplx = torch.is_complex(psi)
    psi = psi.to(torch.complex128 if cplx else torch.float64).contiguous()
    ns = psi.shape[1]
    w = np.asarray(weights)
    if cplx:
        wv = np.empty(2 * ns)
        wv[0::2], wv[1::2] = np.real(w), np.imag(w)
    else:
        if np.iscomplexobj(w) and np.any(np.imag(w) != 0):
            raise ValueError("complex weights need complex eigenvectors")
        wv = np.real(w).astype(np.float64)
    wt = torch.as_tensor(wv, dtype=torch.float64, device=dev)
    nptr, nadj = prob.node_adjacency()
    m = prob.mesh
    if not hasattr(prob, "_adj_out"):
        prob._adj_out = _Outputs()
    dV, dc, work = prob._adj_out.get(m, dev)
    if out is not None:
        dV, dc = out
    N.check(N.lib().qd_adjoint(m.order, m.num_nodes, m.num_elements, ns, 1 if cplx else 0,
                               N.ptr(prob.d_nodes), N.ptr(prob.d_elems), N.ptr(prob.d_dofmap),
                               N.ptr(psi), N.ptr(wt), N.ptr(nptr), N.ptr(nadj), N.ptr(dV),
                               N.ptr(dc), N.ptr(work), stream_ptr(stream)), "qd_adjoint")
    return dV, dc


class LowestEigenvalues(torch.autograd.Function):
    """E[:k] of (H(V, 1/m*), M) for one structured mesh; differentiable in V
    (nodal, eV) and inv_mstar (per element, units of 1/m0).  Solves k + 1
    levels so that a degenerate cluster at the last level can be detected."""

    @staticmethod
    def forward(ctx, V, inv_mstar, mesh, k, solve_kw):
        prob = FEMProblem(mesh, device=V.device)
        c = (C0_EV_NM2 * inv_mstar.detach()).double()
        dot = Dot(mesh, c.cpu().numpy(), V.detach().double().cpu().numpy())
        hb = HostBatch([dot])
        db = DeviceBatch(hb, V.device)
        db.upload(non_blocking=False)
        db.assemble()
        db.check_status()
        kw = dict(solve_kw or {})
        if "b" in kw and kw["b"] < k + 1:
            kw["b"] = ((k + 1 + 3) // 4) * 4
        E, X, _, _, info, _ = db.solve(k + 1, **kw)
        ctx.save_for_backward(X[:, :k].clone(), E[0, :k].clone())
        ctx.E_next = float(E[0, k].item())
        ctx.prob = prob
        return E[0, :k].to(V.dtype)

    @staticmethod
    def backward(ctx, gE):
        X, E = ctx.saved_tensors
        w = cluster_weights(E.cpu().numpy(), gE.detach().cpu().numpy(), E_next=ctx.E_next)
        dV, dc = energy_gradients(ctx.prob, X, w, out=(
            torch.empty(ctx.prob.mesh.num_nodes, dtype=torch.float64, device=X.device),
            torch.empty(ctx.prob.mesh.num_elements, dtype=torch.float64, device=X.device)))
        return dV, dc * C0_EV_NM2, None, None, None


def lowest_eigenvalues(V, inv_mstar, mesh, k, **solve_kw):
    return LowestEigenvalues.apply(V, inv_mstar, mesh, k, solve_kw)


class NearestEigenvalues(torch.autograd.Function):
    """The k complex eigenvalues nearest ``sigma`` of the open-system pencil
    (H(V, 1/m*) + i Himag(W), M) (``qdsim_b200.cap``), differentiable in V
    (nodal, eV) and inv_mstar (per element, units of 1/m0).  The CAP
    amplitude W is a fixed input.  Returns complex128 [k], nearest first."""

    @staticmethod
    def forward(ctx, V, inv_mstar, mesh, W, k, sigma, solve_kw):
        from .cap import CAPSolver
        c = (C0_EV_NM2 * inv_mstar.detach()).double().cpu().numpy()
        solver = CAPSolver(mesh, c, V.detach().double().cpu().numpy(),
                           np.asarray(W, np.float64), device=V.device)
        kw = dict(solve_kw or {})
        res = solver.solve(k=k + 1, sigma=sigma, **kw)
        if not res.info.get("complete", False):
            warnings.warn("the open-system solve could not certify that the returned "
                          "eigenvalues are the nearest to sigma", RuntimeWarning, stacklevel=2)
        ctx.save_for_backward(res.X[:, :k].clone())
        ctx.E = res.E[:k].copy()
        ctx.E_next = res.E[k:k + 1].copy()
        ctx.prob = solver.prob.fem
        return torch.as_tensor(res.E[:k], dtype=torch.complex128, device=V.device)

    @staticmethod
    def backward(ctx, gE):
        (X,) = ctx.saved_tensors
        w = np.conj(gE.detach().cpu().numpy().astype(np.complex128))
        w = cluster_weights(ctx.E, w, E_next=ctx.E_next)
        m = ctx.prob.mesh
        dV, dc = energy_gradients(ctx.prob, X, w, out=(
            torch.empty(m.num_nodes, dtype=torch.float64, device=X.device),
            torch.empty(m.num_elements, dtype=torch.float64, device=X.device)))
        return dV, dc * C0_EV_NM2, None, None, None, None, None


def nearest_eigenvalues(V, inv_mstar, mesh, W, k, sigma, **solve_kw):
    return NearestEigenvalues.apply(V, inv_mstar, mesh, W, k, sigma, solve_kw)

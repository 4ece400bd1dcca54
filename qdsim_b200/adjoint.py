"""Adjoint gradients of eigenvalue losses (``qd_adjoint``) and a
``torch.autograd.Function`` that makes the lowest eigenvalues differentiable
with respect to nodal V and per-element inverse effective mass.

For L = sum_s w_s E_s with M-normalised eigenvectors (M depends on neither V
nor m*): dE_s/dV = psi_s^T (dH/dV) psi_s and dE_s/dc_e = psi_s^T Khat_e psi_s,
c_e = C0 (m0/m*_e).  Degenerate levels: a single E_s of a degenerate cluster is
not differentiable, but any sum over the whole cluster is; the weights inside a
cluster (relative spacing below ``degenerate_rtol``) are replaced by their mean,
which leaves cluster sums unchanged and gives the symmetric choice otherwise.
"""
from __future__ import annotations

import numpy as np
import torch

from . import _native as N
from .batch import DeviceBatch, HostBatch
from .fem import C0_EV_NM2, FEMProblem, stream_ptr
from .workloads import Dot


def cluster_weights(E, w, degenerate_rtol=1e-8):
    E = np.asarray(E, float)
    w = np.asarray(w, float).copy()
    scale = max(1e-12, float(np.abs(E).max()))
    i = 0
    while i < len(E):
        j = i + 1
        while j < len(E) and abs(E[j] - E[j - 1]) <= degenerate_rtol * scale:
            j += 1
        if j - i > 1:
            w[i:j] = w[i:j].mean()
        i = j
    return w


def energy_gradients(prob: FEMProblem, psi_reduced: torch.Tensor, weights, stream=None):
    """dL/dV (nodal) and dL/dc (per element) on the device."""
    dev = prob.device
    psi = psi_reduced.to(dev, torch.float64).contiguous()
    ns = psi.shape[1]
    w = torch.as_tensor(np.asarray(weights, float), device=dev)
    nptr, nadj = prob.node_adjacency()
    m = prob.mesh
    dV = torch.empty(m.num_nodes, dtype=torch.float64, device=dev)
    dc = torch.empty(m.num_elements, dtype=torch.float64, device=dev)
    N.check(N.lib().qd_adjoint(m.order, m.num_nodes, m.num_elements, ns, N.ptr(prob.d_nodes),
                               N.ptr(prob.d_elems), N.ptr(prob.d_dofmap), None, N.ptr(psi),
                               N.ptr(w), N.ptr(nptr), N.ptr(nadj), N.ptr(dV), N.ptr(dc),
                               stream_ptr(stream)), "qd_adjoint")
    return dV, dc


class LowestEigenvalues(torch.autograd.Function):
    """E[:k] of (H(V, 1/m*), M) for one structured mesh; differentiable in V
    (nodal, eV) and inv_mstar (per element, units of 1/m0)."""

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
        E, X, _, _, info, _ = db.solve(k, **(solve_kw or {}))
        ctx.save_for_backward(X.clone(), E[0].clone())
        ctx.prob = prob
        return E[0].to(V.dtype)

    @staticmethod
    def backward(ctx, gE):
        X, E = ctx.saved_tensors
        w = cluster_weights(E.cpu().numpy(), gE.detach().cpu().numpy())
        dV, dc = energy_gradients(ctx.prob, X, w)
        return dV, dc * C0_EV_NM2, None, None, None


def lowest_eigenvalues(V, inv_mstar, mesh, k, **solve_kw):
    return LowestEigenvalues.apply(V, inv_mstar, mesh, k, solve_kw)

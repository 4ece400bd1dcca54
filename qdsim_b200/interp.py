"""Finite-element field evaluation at arbitrary points, on the GPU.

``FieldInterpolator`` evaluates nodal fields of a ``StructuredMesh`` (values,
gradients, containing elements) for a whole batch of points and fields in one
launch of ``qd_fe_interpolate``, and of a refined (unstructured) ``TriMesh``
in one launch of ``qd_fe_interpolate_tri``, which locates points through a
bucket grid over the cells of the mesh the refinement started from.  It is the batched form of the reference's
``FEInterpolator`` (backend/src/fe_interpolator.cpp, bound at
backend/src/bindings.cpp:779-809) and of ``interpolate_field_kernel``
(backend/src/gpu_kernels.cu:352-423); ``qdsim_b200.frontend.FEInterpolator``
wraps it with the reference's per-point method names.

Outside every element the value is the nearest node's with the reference's
neighbour-difference gradient estimate (``outside="nearest"``, FEInterpolator)
or zero (``outside="zero"``, interpolate_field_kernel).
"""
from __future__ import annotations

import numpy as np
import torch

from . import _native as N
from .adapt import TriMesh
from .fem import node_adjacency, stream_ptr
from .mesh import StructuredMesh


def element_buckets(nodes, elems, gx: int, gy: int, Lx: float, Ly: float):
    """Bucket grid of a triangular mesh: gx x gy cells over [0, Lx] x [0, Ly];
    cell (i, j) lists, in ascending element order, every element whose
    bounding box (vertices only: the P2/P3 nodes lie inside the triangle),
    padded by 1e-6 of a cell, meets the cell.  The pad is far wider than the
    -1e-10 barycentric acceptance band, so an element that can accept a point
    is in the bucket of the point's cell.  Returns (cell_ptr int32[gx gy + 1],
    cell_elems int32[...])."""
    v = np.asarray(nodes, np.float64)[np.asarray(elems)[:, :3]]      # (E, 3, 2)
    hx, hy = Lx / gx, Ly / gy
    pad = 1e-6 * max(hx, hy)
    i0 = np.clip(np.floor((v[:, :, 0].min(1) - pad) / hx), 0, gx - 1).astype(np.int64)
    i1 = np.clip(np.floor((v[:, :, 0].max(1) + pad) / hx), 0, gx - 1).astype(np.int64)
    j0 = np.clip(np.floor((v[:, :, 1].min(1) - pad) / hy), 0, gy - 1).astype(np.int64)
    j1 = np.clip(np.floor((v[:, :, 1].max(1) + pad) / hy), 0, gy - 1).astype(np.int64)
    ni, nj = i1 - i0 + 1, j1 - j0 + 1
    count = ni * nj
    e_rep = np.repeat(np.arange(len(v), dtype=np.int64), count)
    k = np.arange(int(count.sum())) - np.repeat(np.cumsum(count) - count, count)
    ci = np.repeat(i0, count) + k % np.repeat(ni, count)
    cj = np.repeat(j0, count) + k // np.repeat(ni, count)
    cell = cj * gx + ci
    order = np.lexsort((e_rep, cell))          # by cell, then element ascending
    cell_elems = e_rep[order].astype(np.int32)
    ptr = np.zeros(gx * gy + 1, np.int64)
    np.add.at(ptr, cell + 1, 1)
    return np.cumsum(ptr).astype(np.int32), cell_elems


def _points(a, device) -> torch.Tensor:
    t = torch.as_tensor(a, dtype=torch.float64)
    return t.reshape(-1).to(device).contiguous()


class FieldInterpolator:
    """Point evaluation of nodal fields of one structured mesh."""

    def __init__(self, mesh: StructuredMesh, device="cuda", outside: str = "nearest"):
        if outside not in ("nearest", "zero"):
            raise ValueError("outside must be 'nearest' or 'zero'")
        self.mesh = mesh
        self.device = torch.device(device)
        self.outside = outside
        self._tri = None
        if isinstance(mesh, TriMesh):
            ptr, cel = element_buckets(mesh.nodes, mesh.elems, mesh.nx, mesh.ny, mesh.Lx,
                                       mesh.Ly)
            aptr, adj = node_adjacency(mesh.elems, mesh.num_nodes)
            dev = self.device
            self._tri = {
                "nodes": torch.from_numpy(np.ascontiguousarray(mesh.nodes)).to(dev),
                "elems": torch.from_numpy(np.ascontiguousarray(mesh.elems)).to(dev),
                "cell_ptr": torch.from_numpy(ptr).to(dev),
                "cell_elems": torch.from_numpy(cel).to(dev),
                "adjptr": torch.from_numpy(aptr).to(dev),
                "adj": torch.from_numpy(adj).to(dev)}
        elif not isinstance(mesh, StructuredMesh):
            raise TypeError("FieldInterpolator needs a StructuredMesh or a TriMesh")

    @property
    def num_nodes(self) -> int:
        return int(self.mesh.num_nodes)

    def evaluate(self, x, y, field, gradient: bool = False, element: bool = False,
                 stream=None):
        """Evaluate ``field`` ((N,) or (F, N) nodal values) at the points
        ``x``, ``y`` (array-likes or device tensors, P each).

        Returns a dict of device tensors: ``value`` ((P,) or (F, P)), and with
        ``gradient`` ``grad_x`` / ``grad_y`` of the same shape, with
        ``element`` ``element`` ((P,) int32, -1 outside the mesh).

        With an explicit ``stream`` the input copies, the output allocations and
        the launch all happen on that stream, so the kernel never reads inputs
        still being copied on another stream and the caching allocator ties the
        outputs to the stream that writes them."""
        if stream is not None:
            with torch.cuda.stream(stream):
                return self._evaluate(x, y, field, gradient, element, stream)
        return self._evaluate(x, y, field, gradient, element, None)

    def _evaluate(self, x, y, field, gradient, element, stream):
        m = self.mesh
        xs, ys = _points(x, self.device), _points(y, self.device)
        if xs.numel() != ys.numel():
            raise ValueError("x and y must have the same number of points")
        f = torch.as_tensor(field, dtype=torch.float64)
        single = f.dim() == 1
        f = f.reshape(1, -1) if single else f
        if f.dim() != 2 or f.shape[1] != self.num_nodes:
            raise ValueError(f"field must have {self.num_nodes} nodal values per row")
        f = f.to(self.device).contiguous()
        P, F = xs.numel(), f.shape[0]
        val = torch.empty((F, P), dtype=torch.float64, device=self.device)
        gx = torch.empty_like(val) if gradient else None
        gy = torch.empty_like(val) if gradient else None
        el = torch.empty(P, dtype=torch.int32, device=self.device) if element else None
        if self._tri is not None:
            t = self._tri
            N.check(N.lib().qd_fe_interpolate_tri(
                m.order, m.num_nodes, m.num_elements, N.ptr(t["nodes"]), N.ptr(t["elems"]),
                m.nx, m.ny, m.Lx, m.Ly, N.ptr(t["cell_ptr"]), N.ptr(t["cell_elems"]),
                N.ptr(t["adjptr"]), N.ptr(t["adj"]), F, f.shape[1], N.ptr(f), P, N.ptr(xs),
                N.ptr(ys), N.ptr(val), N.ptr(gx), N.ptr(gy), N.ptr(el),
                int(self.outside == "zero"), stream_ptr(stream)), "qd_fe_interpolate_tri")
        else:
            N.check(N.lib().qd_fe_interpolate(
                m.order, m.nx, m.ny, m.Lx, m.Ly, F, f.shape[1], N.ptr(f), P, N.ptr(xs),
                N.ptr(ys), N.ptr(val), N.ptr(gx), N.ptr(gy), N.ptr(el),
                int(self.outside == "zero"), stream_ptr(stream)), "qd_fe_interpolate")
        out = {"value": val[0] if single else val}
        if gradient:
            out["grad_x"] = gx[0] if single else gx
            out["grad_y"] = gy[0] if single else gy
        if element:
            out["element"] = el
        return out

    def resample(self, field, target: StructuredMesh, stream=None) -> torch.Tensor:
        """``field`` on this mesh evaluated at the nodes of ``target`` (one
        launch; (N_target,) or (F, N_target))."""
        nodes = torch.as_tensor(np.ascontiguousarray(target.nodes), dtype=torch.float64)
        return self.evaluate(nodes[:, 0], nodes[:, 1], field, stream=stream)["value"]


__all__ = ["FieldInterpolator"]

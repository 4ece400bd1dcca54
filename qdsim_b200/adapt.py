"""Adaptive refinement of the triangular meshes (host side).

Restates the reference's refinement step, ``FEMSolver::adapt_mesh``
(backend/src/fem.cpp:470-542):
- ``refinement_flags`` marks the elements whose least-squares gradient of a
  nodal field exceeds a threshold (``AdaptiveMesh::computeRefinementFlags``,
  backend/src/adaptive_mesh.cpp:431-494). The gradient is fitted over the
  element's K nodes, (c, gx, gy) = pinv([1 x y]) psi_e.
- ``refine`` red-refines them (four children by the edge midpoints, in the
  reference's child order, adaptive_mesh.cpp:105-117).

The reference then tries to close the hanging nodes by refining neighbours
again, but indexes the old elements' flags with the new elements' numbers
(:354-395), so its result is not a conforming mesh. Here the closure is the
standard red-green one with green removal:
- a triangle with two or three split edges is red-refined too, until no
  triangle has more than one split edge;
- a triangle with one split edge is bisected from that edge's midpoint to the
  opposite vertex (a green pair, whose parent the mesh remembers);
- green pairs are merged back into their parents before the next refinement,
  so a green triangle is never bisected again;
- a red triangle on half of a hanging edge makes the coarse triangle across
  it red too, so neighbours differ by at most one level.
The result is conforming, every child keeps its parent's orientation, and
shapes and vertex valences stay bounded over repeated refinements.

The refined mesh is a ``TriMesh``: the vertex mesh is refined, then the P2/P3
nodes are generated on it (edge nodes at 1/2, or at 1/3 and 2/3; the P3
centroid) in the local node order of the structured meshes. Its boundary
nodes are those on edges that belong to one element only. ``TriMesh`` has the
attributes ``FEMProblem`` and ``HostBatch`` read, so the GPU assembly
(explicit coordinates) and the eigensolve run on it unchanged; the DST
preconditioner, which needs the lattice, is not used on it.
"""
from __future__ import annotations

import hashlib

import numpy as np

from .mesh import LOCAL_NODES, nodes_per_element

_EDGES = ((0, 1), (1, 2), (2, 0))


class TriMesh:
    """Unstructured triangular mesh of order 1, 2 or 3 over the rectangle
    [0, Lx] x [0, Ly]: ``nodes`` (N, 2), ``elems`` (E, K) in the local node
    order of ``StructuredMesh``, ``boundary`` (N,) flags."""

    def __init__(self, order: int, nodes, elems, boundary, Lx: float, Ly: float,
                 nx: int, ny: int, green_pair=None, green_parent=None):
        self.order = int(order)
        self.nodes = np.ascontiguousarray(nodes, dtype=np.float64)
        self.elems = np.ascontiguousarray(elems, dtype=np.int32)
        self.boundary = np.ascontiguousarray(boundary, dtype=bool)
        self.Lx, self.Ly = float(Lx), float(Ly)
        # the cell counts of the mesh this one was refined from (the
        # reference's Mesh keeps reporting them)
        self.nx, self.ny = int(nx), int(ny)
        if self.elems.shape[1] != nodes_per_element(self.order):
            raise ValueError("elems do not match the element order")
        # green pairs of the last refinement: pair id per element (-1 none)
        # and each pair's parent triangle (vertex node numbers)
        self.green_pair = (np.full(self.num_elements, -1, dtype=np.int64) if green_pair is None
                           else np.asarray(green_pair, dtype=np.int64))
        self.green_parent = (np.zeros((0, 3), dtype=np.int64) if green_parent is None
                             else np.asarray(green_parent, dtype=np.int64).reshape(-1, 3))
        if self.green_pair.shape != (self.num_elements,):
            raise ValueError("one green-pair entry per element")
        self._key = None

    @property
    def num_nodes(self) -> int:
        return int(self.nodes.shape[0])

    @property
    def num_elements(self) -> int:
        return int(self.elems.shape[0])

    def centroids(self) -> np.ndarray:
        return self.nodes[self.elems[:, :3]].mean(axis=1)

    def shape_key(self):
        if self._key is None:
            h = hashlib.sha1(self.elems.tobytes()).hexdigest()
            self._key = ("tri", self.order, self.num_nodes, self.num_elements, h)
        return self._key


def refinement_flags(mesh, psi, threshold: float) -> np.ndarray:
    """Elements whose least-squares gradient of the nodal field ``psi``
    exceeds ``threshold`` (adaptive_mesh.cpp:431-494): per element, A = [1 x y]
    over its K nodes, (c, gx, gy) = pinv(A) psi_e, flagged when
    |(gx, gy)| > threshold."""
    psi = np.asarray(psi, dtype=np.float64).reshape(-1)
    if psi.size != mesh.num_nodes:
        raise ValueError("psi must have one value per mesh node")
    el = mesh.elems
    xy = mesh.nodes[el]                                  # (E, K, 2)
    A = np.concatenate([np.ones(el.shape + (1,)), xy], axis=2)
    g = np.einsum("ejk,ek->ej", np.linalg.pinv(A)[:, 1:3, :], psi[el])
    return np.sqrt(g[:, 0] ** 2 + g[:, 1] ** 2) > threshold


def _vertex_mesh(mesh):
    """Vertex coordinates and vertex triangles of a mesh of any order, and the
    node -> vertex map (-1 for nodes that are not vertices)."""
    tri = mesh.elems[:, :3]
    verts, inv = np.unique(tri.ravel(), return_inverse=True)
    vmap = np.full(mesh.num_nodes, -1, dtype=np.int64)
    vmap[verts] = np.arange(verts.size)
    return mesh.nodes[verts], inv.reshape(tri.shape).astype(np.int64), vmap


def _edge_ids(tri, nv):
    """Unique edge ids (E, 3) of the local edges, numbered in order of first
    appearance (element order, local edge order), and each edge's vertices."""
    a = tri[:, [0, 1, 2]]
    b = tri[:, [1, 2, 0]]
    keys = (np.minimum(a, b) * nv + np.maximum(a, b)).ravel()
    uniq, first, inv = np.unique(keys, return_index=True, return_inverse=True)
    rank = np.empty(uniq.size, dtype=np.int64)
    rank[np.argsort(first, kind="stable")] = np.arange(uniq.size)
    ids = rank[inv].reshape(tri.shape)
    ends = np.empty((uniq.size, 2), dtype=np.int64)
    ends[rank] = np.stack([uniq // nv, uniq % nv], axis=1)
    return ids, ends


def _refine_vertex_mesh(V, T, flags, pair=None, parents=None, extra_hang=None):
    """Red-green refinement of the vertex mesh (V, T) for the flagged
    triangles, with green removal.

    ``pair[e]`` names the green pair triangle e belongs to (-1 for none) and
    ``parents[p]`` that pair's parent triangle (a, b, c), bisected on (a, b).

    1. Every green pair is replaced by its parent (flagged when either half
       is), which leaves a red-only mesh whose hanging edges are the parents'
       bisected edges, each with its existing midpoint.
    2. Closure, until stable:
       - a triangle is red when flagged;
       - a triangle is red when two or more of its edges are split (hanging,
         or an edge of a red triangle);
       - a red triangle lying on half of a hanging edge makes the coarse
         triangle across that edge red too, so neighbours never differ by
         more than one level.
    3. Red triangles get four children, in the reference's order. A hanging
       edge reuses its midpoint. A triangle with exactly one split edge is
       bisected to its opposite vertex (a new green pair).

    Only red triangles are ever subdivided further, so shapes and vertex
    valences stay bounded over repeated refinements.

    ``extra_hang`` adds hanging edges (edge -> existing midpoint) left by an
    earlier pass.  Returns the new vertices (old ones first, then the new
    midpoints in order of first appearance), the triangles (each parent's
    children in the parent's place), the new green pairs and parents, and
    the midpoint of every edge split in this pass."""
    V = np.asarray(V, dtype=np.float64)
    nv = V.shape[0]
    T = np.asarray(T, dtype=np.int64)
    flags = np.asarray(flags, dtype=bool)
    hang = dict(extra_hang or {})           # hanging edge -> its midpoint vertex
    if pair is not None and (np.asarray(pair) >= 0).any():
        pair = np.asarray(pair, dtype=np.int64)
        parents = np.asarray(parents, dtype=np.int64)
        nT, nF, seen = [], [], set()
        for e in range(T.shape[0]):
            pid = int(pair[e])
            if pid < 0:
                nT.append(T[e])
                nF.append(bool(flags[e]))
                continue
            if pid in seen:
                continue
            seen.add(pid)
            pa, pb, pc = (int(v) for v in parents[pid])
            m = ({int(v) for v in T[e]} - {pa, pb, pc}).pop()
            hang[(min(pa, pb), max(pa, pb))] = m
            nT.append((pa, pb, pc))
            nF.append(bool(flags[pair == pid].any()))
        T = np.asarray(nT, dtype=np.int64)
        flags = np.asarray(nF, dtype=bool)
    eid, ends = _edge_ids(T, nv)
    ne = ends.shape[0]
    keyid = {(int(u), int(v)): i for i, (u, v) in enumerate(ends)}
    is_hang = np.zeros(ne, dtype=bool)
    owner = np.full(ne, -1, dtype=np.int64)  # half of a hanging edge -> coarse triangle
    tri_of = np.full(ne, -1, dtype=np.int64)
    tri_of[eid.ravel()] = np.repeat(np.arange(T.shape[0]), 3)
    for (u, v), m in hang.items():
        h = keyid[(u, v)]
        is_hang[h] = True
        for half in ((min(u, m), max(u, m)), (min(m, v), max(m, v))):
            if half in keyid:
                owner[keyid[half]] = tri_of[h]
    red = flags.copy()
    while True:
        split = is_hang.copy()
        split[eid[red].ravel()] = True
        more = (~red) & (split[eid].sum(axis=1) >= 2)
        coarse = owner[eid[red].ravel()]
        coarse = coarse[coarse >= 0]
        more[coarse[~red[coarse]]] = True
        if not more.any():
            break
        red |= more
    green = (~red) & (split[eid].sum(axis=1) == 1)
    mid = np.full(ne, -1, dtype=np.int64)
    fresh = []
    for ed in np.flatnonzero(split):        # edge ids are first-appearance ranks
        k = (int(ends[ed, 0]), int(ends[ed, 1]))
        if k in hang:
            mid[ed] = hang[k]
        else:
            mid[ed] = nv + len(fresh)
            fresh.append(ed)
    fresh = np.asarray(fresh, dtype=np.int64)
    newV = np.concatenate([V, 0.5 * (V[ends[fresh, 0]] + V[ends[fresh, 1]])])
    mids = {(int(ends[ed, 0]), int(ends[ed, 1])): int(mid[ed]) for ed in np.flatnonzero(split)}
    out, out_pair, out_parents = [], [], []
    for e in range(T.shape[0]):
        n0, n1, n2 = T[e]
        if red[e]:
            m01, m12, m20 = mid[eid[e, 0]], mid[eid[e, 1]], mid[eid[e, 2]]
            out += [(n0, m01, m20), (n1, m12, m01), (n2, m20, m12), (m01, m12, m20)]
            out_pair += [-1] * 4
        elif green[e]:
            j = int(np.flatnonzero(split[eid[e]])[0])
            a, b, c = T[e][j], T[e][(j + 1) % 3], T[e][(j + 2) % 3]
            m = mid[eid[e, j]]
            out += [(a, m, c), (m, b, c)]
            out_pair += [len(out_parents)] * 2
            out_parents.append((a, b, c))
        else:
            out.append((n0, n1, n2))
            out_pair.append(-1)
    return (newV, np.asarray(out, dtype=np.int64), np.asarray(out_pair, dtype=np.int64),
            np.asarray(out_parents, dtype=np.int64).reshape(-1, 3), mids)


def _refine_conforming(V, T, flags, pair, parents):
    """One refinement step, then closure passes until no edge of the mesh has
    a midpoint used on its other side.  A coarse triangle and a finer one on
    half of its hanging edge can both be refined in one step; the coarse
    triangle's child then keeps a full edge that the fine side split, and the
    next pass (no new flags) closes it like any other split edge."""
    V, T, pair, parents, known = _refine_vertex_mesh(V, T, flags, pair, parents)
    while True:
        a = T[:, [0, 1, 2]]
        b = T[:, [1, 2, 0]]
        lo, hi = np.minimum(a, b).ravel(), np.maximum(a, b).ravel()
        residual = {}
        for u, v in zip(lo.tolist(), hi.tolist()):
            m = known.get((u, v))
            if m is not None:
                residual[(u, v)] = m
        if not residual:
            return V, T, pair, parents
        V, T, pair, parents, more = _refine_vertex_mesh(
            V, T, np.zeros(T.shape[0], dtype=bool), pair, parents, extra_hang=residual)
        known.update(more)


def _lift(V, T, order):
    """Elements of ``order`` on the vertex mesh (V, T): vertices first, then
    the edge nodes (per edge in order of first appearance; for P3 the node
    nearer the lower-numbered vertex first), then the P3 centroids."""
    nv = V.shape[0]
    eid, ends = _edge_ids(T, nv)
    ne = ends.shape[0]
    # boundary: edges of one element only, with all their nodes
    counts = np.bincount(eid.ravel(), minlength=ne)
    bedge = counts == 1
    if order == 1:
        bnd = np.zeros(nv, dtype=bool)
        bnd[ends[bedge].ravel()] = True
        return V, T, bnd
    p = order
    per_edge = p - 1
    u, v = V[ends[:, 0]], V[ends[:, 1]]
    edge_nodes = [((p - s) * u + s * v) / p for s in range(1, p)]   # s-th from the lower end
    E_nodes = np.stack(edge_nodes, axis=1).reshape(ne * per_edge, 2)
    nodes = [V, E_nodes]
    if p == 3:
        nodes.append(V[T].mean(axis=1))
    nodes = np.concatenate(nodes)
    K = nodes_per_element(p)
    el = np.zeros((T.shape[0], K), dtype=np.int64)
    el[:, :3] = T
    for a, bc in enumerate(LOCAL_NODES[p]):
        if a < 3:
            continue
        nz = [m for m in range(3) if bc[m] > 0]
        if len(nz) == 3:                               # P3 centroid
            el[:, a] = nv + ne * per_edge + np.arange(T.shape[0])
            continue
        i, j = nz                                      # local edge between vertices i and j
        k = {(0, 1): 0, (1, 2): 1, (0, 2): 2}[(i, j)]
        e = eid[:, k]
        lo = ends[e, 0]
        # distance (in steps of 1/p) of this node from the edge's lower end
        steps_from_i = bc[j]                          # bc[j] / p of the way from i to j
        s = np.where(T[:, i] == lo, steps_from_i, p - steps_from_i)
        el[:, a] = nv + e * per_edge + (s - 1)
    bnd = np.zeros(nodes.shape[0], dtype=bool)
    be = np.flatnonzero(bedge)
    bnd[ends[be].ravel()] = True
    for s in range(per_edge):
        bnd[nv + be * per_edge + s] = True
    return nodes, el, bnd


def refine(mesh, flags) -> TriMesh:
    """The mesh after refining the flagged elements (red-green closure, see
    the module docstring), as a ``TriMesh`` of the same order."""
    flags = np.asarray(flags, dtype=bool).reshape(-1)
    if flags.size != mesh.num_elements:
        raise ValueError("one flag per element")
    V, T, vmap = _vertex_mesh(mesh)
    pair = getattr(mesh, "green_pair", None)
    parents = getattr(mesh, "green_parent", None)
    if parents is not None:
        parents = vmap[parents]
    V2, T2, pair2, parents2 = _refine_conforming(V, T, flags, pair, parents)
    nodes, el, bnd = _lift(V2, T2, mesh.order)
    # vertices keep their numbers in the lifted mesh (they come first)
    return TriMesh(mesh.order, nodes, el, bnd, mesh.Lx, mesh.Ly, mesh.nx, mesh.ny,
                   green_pair=pair2, green_parent=parents2)


__all__ = ["TriMesh", "refinement_flags", "refine"]

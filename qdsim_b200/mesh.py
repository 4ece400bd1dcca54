"""Structured triangular meshes (host-side input preparation).

``StructuredMesh`` follows ``backend/src/mesh.cpp:66-115``: ``nx``/``ny`` are
cells, each cell (n0, n1, n2, n3) is split into (n0, n1, n2) and
(n1, n3, n2).  P2 adds edge midpoints; P3 adds two nodes per edge (at 1/3 and
2/3; the reference aliases both onto one midpoint, ``mesh.cpp:130-153``) and
the element centroid.  All nodes sit on the refined lattice of
(p nx + 1) x (p ny + 1) points and are numbered row-major on it.  Local node
order per element follows ``backend/src/fe_interpolator.cpp:474-518``:
P2 = (v0, v1, v2, m01, m12, m20); P3 = (v0, v1, v2, e01 near v0, e01 near v1,
e12 near v1, e12 near v2, e20 near v2, e20 near v0, centroid).

``SimpleMesh`` mirrors ``qdsim_cython/core/mesh_minimal.pyx:18-126`` (nx, ny
are *points*, coordinates in metres) and is the P1 special case.
"""
from __future__ import annotations

import numpy as np

LOCAL_NODES = {
    1: [(1, 0, 0), (0, 1, 0), (0, 0, 1)],
    2: [(2, 0, 0), (0, 2, 0), (0, 0, 2), (1, 1, 0), (0, 1, 1), (1, 0, 1)],
    3: [(3, 0, 0), (0, 3, 0), (0, 0, 3), (2, 1, 0), (1, 2, 0), (0, 2, 1), (0, 1, 2),
        (1, 0, 2), (2, 0, 1), (1, 1, 1)],
}


def nodes_per_element(order: int) -> int:
    return {1: 3, 2: 6, 3: 10}[order]


class StructuredMesh:
    """Rectangle [0, Lx] x [0, Ly] with nx x ny cells and elements of ``order``."""

    def __init__(self, order: int, nx: int, ny: int, Lx: float, Ly: float):
        if order not in (1, 2, 3):
            raise ValueError("order must be 1, 2 or 3")
        if nx < 1 or ny < 1:
            raise ValueError("need at least one cell in each direction")
        if not (Lx > 0 and Ly > 0):
            raise ValueError("domain lengths must be positive")
        self.order, self.nx, self.ny = int(order), int(nx), int(ny)
        self.Lx, self.Ly = float(Lx), float(Ly)
        p = self.order
        NX, NY = p * nx + 1, p * ny + 1
        self.lattice = (NX, NY)
        ix, iy = np.meshgrid(np.arange(NX), np.arange(NY))
        self.nodes = np.ascontiguousarray(
            np.stack([ix.ravel() * (self.Lx / (p * nx)), iy.ravel() * (self.Ly / (p * ny))], 1))
        self.boundary = ((ix == 0) | (ix == NX - 1) | (iy == 0) | (iy == NY - 1)).ravel()
        ci, cj = np.meshgrid(np.arange(nx), np.arange(ny))
        ci, cj = ci.ravel(), cj.ravel()
        v00 = np.stack([ci, cj], 1) * p
        v10 = np.stack([ci + 1, cj], 1) * p
        v01 = np.stack([ci, cj + 1], 1) * p
        v11 = np.stack([ci + 1, cj + 1], 1) * p
        k = nodes_per_element(p)
        elems = np.zeros((2 * nx * ny, k), dtype=np.int64)
        for t, tri in enumerate(((v00, v10, v01), (v10, v11, v01))):
            for a, bc in enumerate(LOCAL_NODES[p]):
                lat = (bc[0] * tri[0] + bc[1] * tri[1] + bc[2] * tri[2]) // p
                elems[t::2, a] = lat[:, 1] * NX + lat[:, 0]
        self.elems = np.ascontiguousarray(elems.astype(np.int32))

    @property
    def num_nodes(self) -> int:
        return self.nodes.shape[0]

    @property
    def num_elements(self) -> int:
        return self.elems.shape[0]

    @property
    def k(self) -> int:
        return self.elems.shape[1]

    def centroids(self) -> np.ndarray:
        return self.nodes[self.elems[:, :3]].mean(axis=1)

    def shape_key(self):
        return (self.order, self.nx, self.ny)


class SimpleMesh:
    """``SimpleMesh(nx, ny, Lx, Ly)`` of ``qdsim_cython/core/mesh_minimal.pyx``:
    nx x ny grid *points* on [0, Lx] x [0, Ly] (metres), P1 triangles."""

    def __init__(self, nx: int = 10, ny: int = 10, Lx: float = 100e-9, Ly: float = 100e-9):
        if nx < 2 or ny < 2:
            raise ValueError("SimpleMesh needs at least 2 points per direction")
        self.nx, self.ny = int(nx), int(ny)
        self.Lx, self.Ly = float(Lx), float(Ly)
        self.num_nodes = self.nx * self.ny
        self.num_elements = (self.nx - 1) * (self.ny - 1) * 2
        self._m = StructuredMesh(1, self.nx - 1, self.ny - 1, self.Lx, self.Ly)

    def get_nodes(self):
        return self._m.nodes[:, 0].copy(), self._m.nodes[:, 1].copy()

    def get_elements(self):
        return self._m.elems.copy()

    def get_node_at(self, node_id: int):
        return float(self._m.nodes[node_id, 0]), float(self._m.nodes[node_id, 1])

    def structured(self) -> StructuredMesh:
        return self._m

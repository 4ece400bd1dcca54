"""FP64 restatement of QDSim's finite-element field interpolation.
TEST INFRASTRUCTURE ONLY (the checker, never the product path).

Follows ``backend/src/fe_interpolator.cpp`` point by point, with its linear
search:

- ``find_element`` (:363-431): the first element, in element order, whose
  barycentric coordinates (:433-472, signed-area formula) are all >= -1e-10;
  -1 when there is none.
- ``interpolate`` (:54-138): sum of nodal values times the shape functions
  (:474-540) of that element; outside every element, the value at the
  nearest node (squared distance, first node on ties, none when no distance
  is below DBL_MAX), else 0.
- ``interpolate_with_gradient`` (:163-361): the same value, and the gradient
  sum_a f_a grad(phi_a) with grad(phi_a) = sum_m (d phi_a / d lambda_m)
  grad(lambda_m) (:542-613); outside, the inverse-distance weighted average of
  the directional differences (f_q - f_n) (x_q - x_n) / |x_q - x_n| over the
  nodes q that share an element with the nearest node n, each counted once
  in the order the element scan meets them.
- ``zero_outside`` mode: 0 outside every element, as ``interpolate_field_kernel``
  (``backend/src/gpu_kernels.cu:352-423``) does.

Parity pin: ``fe_interpolator.cpp`` needs Eigen, which this image lacks, so
it cannot be compiled here.  The restatement is pinned (``tests/test_cpu_interp.py``)
against golden vectors of the reference's own Python P1 interpolator
(``frontend/qdsim/fe_interpolator.py``; ``tests/golden/make_interp_golden.py``)
for interior values, gradients and elements and for outside-point values, and
by known answers for P2/P3 and the C++-only rules: nodal values reproduced,
polynomials of the element degree reproduced with their gradients, the first
element winning on shared edges, hand-computed outside-point estimates.

Mesh: ``oracle.fem.structured_mesh`` (lattice node order; P1 identical to
``backend/src/mesh.cpp:66-92``).
"""
from __future__ import annotations

import numpy as np

from .fem import Mesh, shape

INSIDE_EPS = 1e-10
DBL_MAX = np.finfo(np.float64).max


def barycentric(x: float, y: float, v) -> np.ndarray:
    """lambda of (x, y) in the triangle v[0..2] (fe_interpolator.cpp:433-457)."""
    (x0, y0), (x1, y1), (x2, y2) = v
    area = 0.5 * ((x1 - x0) * (y2 - y0) - (x2 - x0) * (y1 - y0))
    return np.array([
        0.5 * ((x1 * y2 - x2 * y1) + (y1 - y2) * x + (x2 - x1) * y) / area,
        0.5 * ((x2 * y0 - x0 * y2) + (y2 - y0) * x + (x0 - x2) * y) / area,
        0.5 * ((x0 * y1 - x1 * y0) + (y0 - y1) * x + (x1 - x0) * y) / area,
    ])


def lambda_gradients(v) -> np.ndarray:
    """grad(lambda_m) as rows [d/dx, d/dy] (fe_interpolator.cpp:552-566)."""
    (x0, y0), (x1, y1), (x2, y2) = v
    area = 0.5 * ((x1 - x0) * (y2 - y0) - (x2 - x0) * (y1 - y0))
    return np.array([[0.5 * (y1 - y2) / area, 0.5 * (x2 - x1) / area],
                     [0.5 * (y2 - y0) / area, 0.5 * (x0 - x2) / area],
                     [0.5 * (y0 - y1) / area, 0.5 * (x1 - x0) / area]])


class Interpolator:
    """The reference's FEInterpolator over an oracle mesh."""

    def __init__(self, mesh: Mesh):
        self.mesh = mesh
        nodes, elems = mesh.nodes, mesh.elems
        self._v = nodes[elems[:, :3]]            # (E, 3, 2) vertex coordinates

    def _bary_all(self, x, y):
        v = self._v
        x0, y0 = v[:, 0, 0], v[:, 0, 1]
        x1, y1 = v[:, 1, 0], v[:, 1, 1]
        x2, y2 = v[:, 2, 0], v[:, 2, 1]
        area = 0.5 * ((x1 - x0) * (y2 - y0) - (x2 - x0) * (y1 - y0))
        l0 = 0.5 * ((x1 * y2 - x2 * y1) + (y1 - y2) * x + (x2 - x1) * y) / area
        l1 = 0.5 * ((x2 * y0 - x0 * y2) + (y2 - y0) * x + (x0 - x2) * y) / area
        l2 = 0.5 * ((x0 * y1 - x1 * y0) + (y0 - y1) * x + (x1 - x0) * y) / area
        return l0, l1, l2

    def find_element(self, x: float, y: float) -> int:
        with np.errstate(invalid="ignore", over="ignore"):
            l0, l1, l2 = self._bary_all(x, y)
            ok = (l0 >= -INSIDE_EPS) & (l1 >= -INSIDE_EPS) & (l2 >= -INSIDE_EPS)
        hit = np.flatnonzero(ok)
        return int(hit[0]) if hit.size else -1

    def nearest_node(self, x: float, y: float) -> int:
        nodes = self.mesh.nodes
        with np.errstate(invalid="ignore", over="ignore"):
            dx = x - nodes[:, 0]
            dy = y - nodes[:, 1]
            d = dx * dx + dy * dy
            valid = d < DBL_MAX
        if not valid.any():
            return -1
        d = np.where(valid, d, np.inf)
        return int(np.argmin(d))        # first index of the minimum

    def _linked(self, node: int):
        """Nodes sharing an element with ``node``, first-seen order, unique."""
        out = []
        for e in np.flatnonzero((self.mesh.elems == node).any(axis=1)):
            row = list(self.mesh.elems[e])
            i = row.index(node)
            for j, q in enumerate(row):
                if j != i and q not in out:
                    out.append(int(q))
        return out

    def evaluate(self, x: float, y: float, field, gradient: bool = False,
                 zero_outside: bool = False):
        """(value, gx, gy, element) for one point."""
        field = np.asarray(field, dtype=np.float64)
        e = self.find_element(x, y)
        if e >= 0:
            v = self._v[e]
            lam = barycentric(x, y, v)
            phi, dphi = shape(self.mesh.order, lam)
            f = field[self.mesh.elems[e]]
            val = float(np.sum(f * phi))
            if not gradient:
                return val, 0.0, 0.0, e
            g = dphi.T @ lambda_gradients(v)      # (K, 2)
            return val, float(f @ g[:, 0]), float(f @ g[:, 1]), e
        n = -1 if zero_outside else self.nearest_node(x, y)
        if n < 0:
            return 0.0, 0.0, 0.0, -1
        if not gradient:
            return float(field[n]), 0.0, 0.0, -1
        nodes = self.mesh.nodes
        sx = sy = wsum = 0.0
        for q in self._linked(n):
            dx = nodes[q, 0] - nodes[n, 0]
            dy = nodes[q, 1] - nodes[n, 1]
            dist = float(np.sqrt(dx * dx + dy * dy))
            if dist > 1e-10:
                w = 1.0 / dist
                df = field[q] - field[n]
                sx += w * (df * dx / dist)
                sy += w * (df * dy / dist)
                wsum += w
        if wsum > 0.0:
            return float(field[n]), sx / wsum, sy / wsum, -1
        return float(field[n]), 0.0, 0.0, -1

    def evaluate_many(self, x, y, fields, gradient: bool = False, zero_outside: bool = False):
        """Values (F, P), gradients (F, P) x 2 and elements (P,) for fields (F, N)."""
        fields = np.atleast_2d(np.asarray(fields, dtype=np.float64))
        P = len(x)
        val = np.zeros((fields.shape[0], P))
        gx = np.zeros_like(val)
        gy = np.zeros_like(val)
        el = np.zeros(P, dtype=np.int64)
        for i in range(P):
            for f in range(fields.shape[0]):
                v, a, b, e = self.evaluate(float(x[i]), float(y[i]), fields[f], gradient,
                                           zero_outside)
                val[f, i], gx[f, i], gy[f, i] = v, a, b
                el[i] = e
        return val, gx, gy, el

"""FP64 restatement of QDSim's refinement flags.
TEST INFRASTRUCTURE ONLY (the checker, never the product path).

``refinement_flags`` follows ``AdaptiveMesh::computeRefinementFlags``
(backend/src/adaptive_mesh.cpp:431-494) element by element. For each element
it takes the coordinates and values of its K nodes, A = [1 x y] (K x 3), the
Moore-Penrose pseudo-inverse of A (the reference calls
``completeOrthogonalDecomposition().pseudoInverse()``) and
grad = pinv(A)[1:3] psi_e. The element is flagged when |grad| > threshold.
Pinned by known answers in ``tests/test_cpu_adapt.py``: a linear field's
gradient is exact on every element, so every element is flagged just below
its norm and none just above.
"""
from __future__ import annotations

import numpy as np


def element_gradients(nodes, elems, psi) -> np.ndarray:
    """Least-squares gradient (E, 2) of the nodal field over each element."""
    out = np.zeros((elems.shape[0], 2))
    for e, el in enumerate(elems):
        A = np.ones((len(el), 3))
        A[:, 1:] = nodes[el]
        out[e] = np.linalg.pinv(A)[1:3] @ psi[el]
    return out


def refinement_flags(nodes, elems, psi, threshold) -> np.ndarray:
    g = element_gradients(nodes, elems, np.asarray(psi, dtype=np.float64))
    return np.sqrt(g[:, 0] ** 2 + g[:, 1] ** 2) > threshold

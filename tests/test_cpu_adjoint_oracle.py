"""The oracle's adjoint gradients against central finite differences of the
oracle's own eigenvalues (pins the checker the GPU adjoint is compared with).

* Differentiation configuration (P3 150x75 cells, L = E1+E2+E3+E4 + (E2-E1)):
  the oracle gradient's projections on the 32 + 32 seeded directions equal
  the committed finite differences (tests/golden/c3_fd.npz, made by
  tests/golden/make_c3_golden.py: 128 oracle solves).
* Open system (complex-symmetric CAP pencil, small mesh): the gradient of a
  real loss of the complex eigenvalues, with bilinearly normalised
  eigenvectors and complex weights, equals central differences of the
  oracle's shift-invert eigenvalues.
"""
import os
import sys

import numpy as np

from oracle import adjoint as OA, fem as O

HERE = os.path.dirname(os.path.abspath(__file__))


def test_oracle_gradient_matches_committed_fd_at_config_size():
    sys.path.insert(0, os.path.join(HERE, "golden"))
    import make_c3_golden as G
    z = np.load(os.path.join(HERE, "golden", "c3_fd.npz"))
    _, om, V, inv_m = G._problem()
    a = O.assemble(om, O.C0_EV_NM2 * inv_m, V)
    E, X = O.eig_lowest(a.H, a.M, 5, O.sigma_below(V))
    assert np.allclose(E, z["E"], rtol=1e-12, atol=0)
    psi = np.zeros((om.num_nodes, 4))
    keep = a.dm >= 0
    psi[keep] = X[a.dm[keep], :4]
    gV, gc = OA.gradients(om, psi, z["weights"])
    dv, di = G.directions(om.num_nodes, om.num_elements, int(z["seed"]))
    pv, pm = dv @ gV, di @ (gc * O.C0_EV_NM2)
    # normwise over the 32 directions: |g.d - fd| <= 1e-6 max |fd|
    assert np.abs(pv - z["fd_v"]).max() <= 1e-6 * np.abs(z["fd_v"]).max()
    assert np.abs(pm - z["fd_m"]).max() <= 1e-6 * np.abs(z["fd_m"]).max()


def _cap_case():
    from qdsim_b200 import workloads as W
    d = W.c2_dot(0, nx=24, ny=12)
    om = O.structured_mesh(2, 24, 12, 200.0, 100.0)
    return d, om


def _cap_levels(om, c, V, Wn, k, sigma, ref=None):
    a = O.assemble(om, c, V, Wn)
    E, X = O.eig_nearest_complex(a.H - 1j * a.Wm, a.M, k, sigma)
    if ref is not None:            # follow each reference level to its nearest
        idx = [int(np.argmin(np.abs(E - e))) for e in ref]
        assert len(set(idx)) == len(idx)
        E, X = E[idx], X[:, idx]
    return E, X, a


def test_oracle_cap_gradient_matches_finite_differences():
    d, om = _cap_case()
    k, sigma = 6, -0.05
    E, X, a = _cap_levels(om, d.c, d.V, d.W, k, sigma)
    rng = np.random.default_rng(3)
    wa, wb = rng.uniform(0.5, 1.5, k), rng.uniform(-1.0, 1.0, k)   # L = a.Re E + b.Im E

    def loss(Es):
        return float(wa @ Es.real + wb @ Es.imag)

    psi = np.zeros((om.num_nodes, k), complex)
    keep = a.dm >= 0
    psi[keep] = X[a.dm[keep]]
    gV, gc = OA.gradients(om, psi, wa - 1j * wb)
    h = 1e-6
    for _ in range(3):
        dv = rng.standard_normal(om.num_nodes)
        fd = (loss(_cap_levels(om, d.c, d.V + h * dv, d.W, k, sigma, E)[0])
              - loss(_cap_levels(om, d.c, d.V - h * dv, d.W, k, sigma, E)[0])) / (2 * h)
        assert abs(gV @ dv - fd) <= 1e-6 * abs(fd), (gV @ dv, fd)
        dc = rng.standard_normal(om.num_elements) * d.c.mean()
        fd = (loss(_cap_levels(om, d.c + h * dc, d.V, d.W, k, sigma, E)[0])
              - loss(_cap_levels(om, d.c - h * dc, d.V, d.W, k, sigma, E)[0])) / (2 * h)
        assert abs(gc @ dc - fd) <= 1e-6 * abs(fd), (gc @ dc, fd)


def test_cluster_weights_symmetric():
    from qdsim_b200.adjoint import cluster_weights
    w = cluster_weights([-0.3, -0.2, -0.2 + 1e-12, -0.1], [0.0, 2.0, 1.0, 1.0])
    assert np.allclose(w, [0.0, 1.5, 1.5, 1.0])


def test_cluster_weights_complex_levels_in_any_order():
    """Open-system levels come nearest-sigma first, not sorted: clusters are
    found over all pairs, and complex weights are averaged."""
    from qdsim_b200.adjoint import cluster_weights
    E = np.array([-0.05 - 1e-3j, -0.02 - 2e-3j, -0.05 - 1e-3j + 1e-13, -0.08 - 1e-4j])
    w = cluster_weights(E, np.array([1.0 + 1j, 2.0, 3.0 - 1j, 4.0]))
    assert np.allclose(w, [2.0, 2.0, 2.0, 4.0])


def test_cluster_cut_at_the_last_level_warns():
    import pytest
    from qdsim_b200.adjoint import cluster_weights
    with pytest.warns(RuntimeWarning):
        cluster_weights([-0.3, -0.2], [1.0, 1.0], E_next=[-0.2 + 1e-13])
    import warnings
    with warnings.catch_warnings():
        warnings.simplefilter("error")
        cluster_weights([-0.3, -0.2], [1.0, 0.0], E_next=[-0.2 + 1e-13])   # zero weight: fine
        cluster_weights([-0.3, -0.2], [1.0, 1.0], E_next=[-0.1])

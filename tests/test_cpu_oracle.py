"""Known-answer tests of the FP64 oracle and cross-checks of the product's
host-side input generation against it."""
import os

import numpy as np
import pytest

from oracle import fem as O


@pytest.mark.parametrize("order,rate", [(1, 2.0), (2, 4.0), (3, 6.0)])
def test_box_eigenvalue_convergence_rates(order, rate):
    """E_11 of a 10x10 box (c = 1): O(h^2), O(h^4), O(h^6) for P1/P2/P3."""
    exact = np.pi ** 2 * (2 / 100)
    errs = []
    for n in (4, 8, 16):
        m = O.structured_mesh(order, n, n, 10.0, 10.0)
        a = O.assemble(m, np.ones(m.num_elements), np.zeros(m.num_nodes))
        E, _ = O.eig_lowest(a.H, a.M, 1, -1.0)
        errs.append(abs(E[0] - exact) / exact)
    rates = [np.log2(errs[i] / errs[i + 1]) for i in range(2)]
    assert abs(rates[-1] - rate) < 0.15, rates


@pytest.mark.parametrize("order", [1, 2, 3])
def test_patch_identities(order):
    m = O.structured_mesh(order, 5, 4, 5.0, 4.0)
    a = O.assemble(m, np.ones(m.num_elements), np.zeros(m.num_nodes), dirichlet=False)
    one = np.ones(a.n)
    assert np.abs(a.K @ one).max() < 1e-12          # K 1 = 0
    assert abs(one @ (a.M @ one) - 20.0) < 1e-12     # 1^T M 1 = area
    assert abs(a.H - a.H.T).max() < 1e-14
    # constant V: H = K + V0 M
    a2 = O.assemble(m, np.ones(m.num_elements), np.full(m.num_nodes, 0.3), dirichlet=False)
    assert abs((a2.H - a.K) - 0.3 * a.M).max() < 1e-13


def test_oscillator_levels():
    """2-D harmonic oscillator: E = hw (nx + ny + 1), P2 on a fine box."""
    L = 40.0
    m = O.structured_mesh(2, 80, 80, L, L)
    w = 0.5           # hbar w in eV; V = (1/2) m w^2 r^2 with c = hbar^2/(2m) = 1
    x, y = m.nodes[:, 0] - L / 2, m.nodes[:, 1] - L / 2
    V = (w ** 2 / 4.0) * (x ** 2 + y ** 2)
    a = O.assemble(m, np.ones(m.num_elements), V)
    E, _ = O.eig_lowest(a.H, a.M, 6, -0.5)
    assert np.allclose(E, w * np.array([1, 2, 2, 3, 3, 3]), rtol=2e-4), E / w


def test_c1_dot_oracle_values():
    mesh, c, V = O.dot_config_c1(0)
    a = O.assemble(mesh, c, V)
    assert a.H.nnz == 33367
    E, X = O.eig_lowest(a.H, a.M, 10, O.sigma_below(V))
    assert -0.3 < E[0] < -0.2                # bound state inside the 0.3 eV dot
    assert np.all(np.diff(E) >= 0)
    assert O.residuals(a.H, a.M, E, X).max() < 1e-10


def test_sweep_golden_reproduced_for_two_dots():
    g = np.load(os.path.join(os.path.dirname(__file__), "golden", "sweep256.npz"))
    for i in (0, 17):
        om, c, V = O.dot_config_sweep(i)
        if om.nx > 120:
            continue
        a = O.assemble(om, c, V)
        E, _ = O.eig_lowest(a.H, a.M, 10, O.sigma_below(V))
        assert np.allclose(E[:8], g["E"][i], rtol=1e-11, atol=0)


def test_product_generators_match_oracle():
    from qdsim_b200 import workloads as W
    from qdsim_b200.mesh import StructuredMesh
    for i in (0, 3, 200):
        d = W.sweep_dot(i)
        om, c, V = O.dot_config_sweep(i)
        assert np.array_equal(d.mesh.elems, om.elems) and np.allclose(d.mesh.nodes, om.nodes)
        assert np.array_equal(d.c, c) and np.array_equal(d.V, V)
    d = W.c1_dot(0)
    om, c, V = O.dot_config_c1(0)
    assert np.array_equal(d.c, c) and np.array_equal(d.V, V)
    for p in (1, 2, 3):
        m = StructuredMesh(p, 7, 3, 7.0, 3.0)
        om = O.structured_mesh(p, 7, 3, 7.0, 3.0)
        assert np.array_equal(m.elems, om.elems) and np.array_equal(m.boundary, om.boundary)


def test_poisson_oracle_linear_ramp():
    from oracle import poisson as OP
    om = O.structured_mesh(1, 10, 4, 50.0, 20.0)
    phi = OP.solve(om, np.full(om.num_elements, 12.0), np.zeros(om.num_nodes), 0.0, 1.0)
    assert np.allclose(phi, om.nodes[:, 0] / 50.0, atol=1e-12)


def test_anderson_coefficients_restatement():
    """Full-rank least squares equals lstsq; clipping and the sum cap apply."""
    from oracle import sc as OS
    rng = np.random.default_rng(3)
    r = [rng.standard_normal(50) for _ in range(3)]
    al = OS.anderson_coefficients(r)
    F = np.stack([r[0] - r[2], r[1] - r[2]], axis=1)
    ref, *_ = np.linalg.lstsq(F, -r[2], rcond=None)
    ref = np.clip(ref, -2, 2)
    if abs(ref.sum()) > 2:
        ref *= 2 / abs(ref.sum())
    assert np.allclose(al, ref, rtol=1e-10)
    # a dependent pair takes the regularised branch and stays finite
    r2 = [r[0], 2 * r[0] - r[2] + 0 * r[1], r[2]]
    r2[1] = r[2] + 2 * (r[0] - r[2])
    al2 = OS.anderson_coefficients(r2)
    assert al2 is not None and np.all(np.isfinite(al2)) and abs(al2.sum()) <= 2 + 1e-12


def test_sc_restatement_runs_and_contracts():
    """The oracle loop on a tiny junction: the error drops over the iterations."""
    import dataclasses
    from oracle import fem as O, sc as OS
    from qdsim_b200 import workloads as W
    j = W.c5_junction(n_bias=2, nx=16, ny=8, Lx=16.0, Ly=8.0)
    j = dataclasses.replace(j, mesh=O.structured_mesh(1, 16, 8, 16.0, 8.0))
    phi, err, E = OS.run(j, k=3, iterations=15)
    assert np.all(np.isfinite(phi)) and err[-1].max() < err[0].max()

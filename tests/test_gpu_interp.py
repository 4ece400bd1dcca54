"""qd_fe_interpolate on the GPU against the oracle's element scan
(backend/src/fe_interpolator.cpp restated in oracle/interp.py).

Containing elements must match exactly (including points on shared edges and
vertices, inside and outside the -1e-10 acceptance band, and non-finite
points); values to 1e-12 and gradients to 1e-10 of fields of order one.  At
full size (4M points) the checks are size-independent: polynomials of the
element degree reproduced with their gradients, every returned element
containing its point.
"""
import numpy as np
import pytest
import torch

from oracle.fem import structured_mesh
from oracle.interp import Interpolator

pytestmark = pytest.mark.gpu


def _mesh_pair(order, nx, ny, Lx, Ly):
    from qdsim_b200.mesh import StructuredMesh
    return StructuredMesh(order, nx, ny, Lx, Ly), structured_mesh(order, nx, ny, Lx, Ly)


def _probe_points(om, rng):
    """Random points (some outside), points on grid lines, diagonals and
    nodes, points just inside / outside the acceptance band, non-finite."""
    p, nx, ny, Lx, Ly = om.order, om.nx, om.ny, om.Lx, om.Ly
    NX = p * nx + 1
    vx = om.nodes[: NX: p, 0]                        # vertex columns
    vy = om.nodes[:: p * NX, 1][: ny + 1]            # vertex rows
    hx, hy = Lx / nx, Ly / ny
    xs, ys = [], []
    xs += list(rng.uniform(-0.1 * Lx, 1.1 * Lx, 300))
    ys += list(rng.uniform(-0.1 * Ly, 1.1 * Ly, 300))
    xs += list(rng.choice(vx, 60))
    ys += list(rng.uniform(0, Ly, 60))
    xs += list(rng.uniform(0, Lx, 60))
    ys += list(rng.choice(vy, 60))
    k = rng.choice(om.num_nodes, 60)
    xs += list(om.nodes[k, 0])
    ys += list(om.nodes[k, 1])
    ci, cj, s = rng.integers(0, nx, 40), rng.integers(0, ny, 40), rng.uniform(0, 1, 40)
    xs += list(vx[ci] + s * hx)
    ys += list(vy[cj] + (1 - s) * hy)
    # the boundary band: 1e-11 of a cell inside the band (found), 1e-9 past it
    for d in (1e-11, 1e-9):
        yy = rng.uniform(0.1 * Ly, 0.9 * Ly, 5)
        xs += list(-d * hx + 0 * yy) + list(Lx + d * hx + 0 * yy)
        ys += list(yy) + list(yy)
    xs += [np.nan, 0.5 * Lx, np.inf, 1e200, -1e200, 0.0, Lx, 0.0]
    ys += [0.5 * Ly, np.nan, 0.5 * Ly, 0.5 * Ly, 0.5 * Ly, 0.0, Ly, Ly]
    return np.array(xs), np.array(ys)


CASES = [(1, 12, 8, 30.0, 20.0), (2, 12, 8, 30.0, 20.0), (3, 12, 8, 30.0, 20.0),
         (2, 5, 7, 40.0, 3.0)]   # the last with 8 x 0.43 cells (anisotropic)


@pytest.mark.parametrize("case", CASES)
@pytest.mark.parametrize("outside", ["nearest", "zero"])
def test_points_match_oracle_scan(cuda, case, outside):
    from qdsim_b200.interp import FieldInterpolator
    sm, om = _mesh_pair(*case)
    rng = np.random.default_rng(case[0] * 10 + case[1])
    x, y = _probe_points(om, rng)
    fields = rng.standard_normal((2, om.num_nodes))
    fi = FieldInterpolator(sm, device=cuda, outside=outside)
    r = fi.evaluate(x, y, fields, gradient=True, element=True)
    ov, ogx, ogy, oe = Interpolator(om).evaluate_many(x, y, fields, gradient=True,
                                                     zero_outside=outside == "zero")
    el = r["element"].cpu().numpy()
    np.testing.assert_array_equal(el, oe)
    assert (el >= 0).sum() > 300 and (el < 0).sum() > 20
    np.testing.assert_allclose(r["value"].cpu().numpy(), ov, rtol=0, atol=1e-12)
    np.testing.assert_allclose(r["grad_x"].cpu().numpy(), ogx, rtol=0, atol=1e-10)
    np.testing.assert_allclose(r["grad_y"].cpu().numpy(), ogy, rtol=0, atol=1e-10)
    # value-only launch (other kernel instantiation) gives the same values
    v = fi.evaluate(x, y, fields)["value"].cpu().numpy()
    np.testing.assert_allclose(v, ov, rtol=0, atol=1e-12)


def _poly(order, x, y):
    if order == 1:
        return 0.3 + 1.7 * x - 0.9 * y, 1.7 + 0 * x, -0.9 + 0 * y
    f = 0.3 + 1.7 * x - 0.9 * y + 0.5 * x * x - 1.1 * x * y + 0.7 * y * y
    return f, 1.7 + 1.0 * x - 1.1 * y, -0.9 - 1.1 * x + 1.4 * y


@pytest.mark.parametrize("order", [1, 2])
def test_full_size_polynomial_reproduction_and_containment(cuda, order):
    """4M points on the 400 x 200-cell mesh of 200 x 100 nm: fields of the
    element degree (in units of the domain) are reproduced exactly, and every
    element returned contains its point."""
    from qdsim_b200.interp import FieldInterpolator
    nx, ny, Lx, Ly = 400, 200, 200.0, 100.0
    sm, _ = _mesh_pair(order, nx, ny, Lx, Ly)
    g = torch.Generator(device=cuda).manual_seed(order)
    P = 1 << 22
    x = torch.rand(P, generator=g, device=cuda, dtype=torch.float64) * Lx
    y = torch.rand(P, generator=g, device=cuda, dtype=torch.float64) * Ly
    nodes = torch.as_tensor(sm.nodes, device=cuda)
    f, _, _ = _poly(order, nodes[:, 0] / Lx, nodes[:, 1] / Ly)
    r = FieldInterpolator(sm, device=cuda).evaluate(x, y, f, gradient=True, element=True)
    ev, egx, egy = _poly(order, x / Lx, y / Ly)
    assert (r["value"] - ev).abs().max().item() < 1e-11
    assert (r["grad_x"] - egx / Lx).abs().max().item() < 1e-11
    assert (r["grad_y"] - egy / Ly).abs().max().item() < 1e-11
    e = r["element"].long()
    assert (e >= 0).all().item()
    cell, t = e // 2, e % 2
    ci, cj = (cell % nx).double(), (cell // nx).double()
    hx, hy = Lx / nx, Ly / ny
    u, w = x / hx - ci, y / hy - cj               # local cell coordinates
    tol = 1e-9
    inside0 = (u >= -tol) & (w >= -tol) & (u + w <= 1 + tol)
    inside1 = (u <= 1 + tol) & (w <= 1 + tol) & (u + w >= 1 - tol)
    assert torch.where(t == 0, inside0, inside1).all().item()


def test_resample_linear_field_between_meshes(cuda):
    from qdsim_b200.interp import FieldInterpolator
    from qdsim_b200.mesh import StructuredMesh
    src = StructuredMesh(1, 30, 10, 300.0, 100.0)       # Poisson-like P1 mesh
    dst = StructuredMesh(2, 64, 24, 300.0, 100.0)       # finer P2 mesh
    f = 0.2 - 0.003 * src.nodes[:, 0] + 0.001 * src.nodes[:, 1]
    out = FieldInterpolator(src, device=cuda).resample(f, dst).cpu().numpy()
    want = 0.2 - 0.003 * dst.nodes[:, 0] + 0.001 * dst.nodes[:, 1]
    np.testing.assert_allclose(out, want, rtol=0, atol=1e-12)


def test_frontend_interpolator_and_interpolated_potential(cuda):
    from qdsim_b200 import frontend as F
    mesh = F.Mesh(30e-9, 20e-9, 12, 8, 2)
    om = structured_mesh(2, 12, 8, 30e-9, 20e-9)
    it = Interpolator(om)
    fi = F.FEMSolver(mesh, lambda x, y: 0.067 * 9.1093837015e-31, lambda x, y: 0.0 * x,
                     lambda x, y: 0.0 * x).get_interpolator()
    rng = np.random.default_rng(5)
    f = rng.standard_normal(mesh.get_num_nodes())
    for x, y in [(3.3e-9, 7.1e-9), (2.5e-9, 5e-9), (31e-9, 4e-9), (-1e-9, -2e-9)]:
        v, gx, gy, e = it.evaluate(x, y, f, gradient=True)
        assert fi.interpolate(x, y, f) == pytest.approx(v, abs=1e-12)
        got = fi.interpolate_with_gradient(x, y, f)
        assert got[0] == pytest.approx(v, abs=1e-12)
        assert got[1] == pytest.approx(gx, rel=1e-10, abs=1e-3)
        assert got[2] == pytest.approx(gy, rel=1e-10, abs=1e-3)
        assert fi.find_element(x, y) == e
        assert fi.is_inside_domain(x, y) == (e >= 0)
    xs, ys = rng.uniform(0, 30e-9, 50), rng.uniform(0, 20e-9, 50)
    want = Interpolator(om).evaluate_many(xs, ys, f)[0][0]
    np.testing.assert_allclose(fi.interpolate_vector(xs, ys, f), want, rtol=0, atol=1e-12)

    # the interpolated-potential assembly equals the callback assembly with
    # the same nodal values
    Q = 1.602176634e-19

    def V(x, y):
        return -0.1 * Q * np.exp(-((x - 15e-9) ** 2 + (y - 10e-9) ** 2) / (5e-9) ** 2)

    mstar = lambda x, y: 0.067 * 9.1093837015e-31 + 0 * x
    zero = lambda x, y: 0.0 * x
    a = F.FEMSolver(mesh, mstar, V, zero)
    a.assemble_matrices()
    b = F.FEMSolver(mesh, mstar, zero, zero)
    nodes = mesh.get_nodes()
    b.set_potential_values(V(nodes[:, 0], nodes[:, 1]))
    b.use_interpolated_potential(True)
    b.assemble_matrices()
    d = (a.get_H() - b.get_H()).tocoo()
    assert np.abs(d.data).max(initial=0.0) <= 1e-12 * np.abs(a.get_H().data).max()


def _refined_pair(order, nx, ny, Lx, Ly, steps=2):
    """A structured mesh refined twice where a seeded Gaussian varies fastest
    (the quarter of elements with the largest gradient, red-green closure),
    and the oracle mesh with the same nodes and elements."""
    from oracle.adapt import element_gradients
    from oracle.fem import Mesh
    from qdsim_b200.adapt import refine, refinement_flags
    from qdsim_b200.mesh import StructuredMesh
    m = StructuredMesh(order, nx, ny, Lx, Ly)
    for _ in range(steps):
        x, y = m.nodes[:, 0], m.nodes[:, 1]
        psi = np.exp(-((x - 0.4 * Lx) ** 2 + (y - 0.55 * Ly) ** 2) / (0.02 * Lx * Lx))
        g = element_gradients(m.nodes, m.elems, psi)
        m = refine(m, refinement_flags(m, psi, float(np.quantile(np.hypot(g[:, 0], g[:, 1]),
                                                                 0.75))))
    om = Mesh(m.order, m.nx, m.ny, m.Lx, m.Ly, m.nodes, m.elems, m.boundary)
    return m, om


@pytest.mark.parametrize("order", [1, 2, 3])
@pytest.mark.parametrize("outside", ["nearest", "zero"])
def test_refined_mesh_points_match_oracle_scan(cuda, order, outside):
    """qd_fe_interpolate_tri on a mesh refined twice: containing elements
    identical to the oracle's scan over all elements (points on refined edges
    and vertices, hanging-free green bisections, the boundary band, outside
    and non-finite points), values 1e-12, gradients 1e-10."""
    from qdsim_b200.interp import FieldInterpolator
    m, om = _refined_pair(order, 10, 6, 30.0, 18.0)
    assert m.num_elements > 2 * 10 * 6
    rng = np.random.default_rng(order)
    sm, om0 = _mesh_pair(order, 10, 6, 30.0, 18.0)
    x, y = _probe_points(om0, rng)
    # plus the refined mesh's own nodes and edge midpoints of its elements
    k = rng.choice(m.num_nodes, 80)
    e = rng.choice(m.num_elements, 60)
    v = m.nodes[m.elems[e, :3]]
    x = np.concatenate([x, m.nodes[k, 0], 0.5 * (v[:, 0, 0] + v[:, 1, 0])])
    y = np.concatenate([y, m.nodes[k, 1], 0.5 * (v[:, 0, 1] + v[:, 1, 1])])
    fields = rng.standard_normal((2, m.num_nodes))
    fi = FieldInterpolator(m, device=cuda, outside=outside)
    r = fi.evaluate(x, y, fields, gradient=True, element=True)
    ov, ogx, ogy, oe = Interpolator(om).evaluate_many(x, y, fields, gradient=True,
                                                     zero_outside=outside == "zero")
    el = r["element"].cpu().numpy()
    np.testing.assert_array_equal(el, oe)
    assert (el >= 0).sum() > 300 and (el < 0).sum() > 20
    np.testing.assert_allclose(r["value"].cpu().numpy(), ov, rtol=0, atol=1e-12)
    np.testing.assert_allclose(r["grad_x"].cpu().numpy(), ogx, rtol=0, atol=1e-10)
    np.testing.assert_allclose(r["grad_y"].cpu().numpy(), ogy, rtol=0, atol=1e-10)
    v = fi.evaluate(x, y, fields)["value"].cpu().numpy()
    np.testing.assert_allclose(v, ov, rtol=0, atol=1e-12)

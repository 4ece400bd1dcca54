"""Finite-element field interpolation without a GPU: the oracle pinned by known
answers, the C entry point's argument checks and the frontend's host logic.

The reference's C++ FEInterpolator (backend/src/fe_interpolator.cpp) needs
Eigen, which this image lacks.  The oracle is pinned by golden vectors of the
reference's own Python P1 interpolator (tests/golden/interp_p1.npz) and by
properties any correct implementation of the C++ file has: nodal values are
reproduced, polynomials of the element degree are reproduced with their
gradients, the first element in index order wins on shared edges, and outside
points follow the nearest-node rule and its gradient estimate, computed here
by hand.
"""
import ctypes as C

import numpy as np
import pytest

from oracle.fem import structured_mesh
from oracle.interp import Interpolator, barycentric


def _poly(order, x, y):
    """A polynomial of total degree ``order`` and its gradient."""
    if order == 1:
        return 0.3 + 1.7 * x - 0.9 * y, 1.7 + 0 * x, -0.9 + 0 * y
    if order == 2:
        f = 0.3 + 1.7 * x - 0.9 * y + 0.05 * x * x - 0.11 * x * y + 0.07 * y * y
        return f, 1.7 + 0.1 * x - 0.11 * y, -0.9 - 0.11 * x + 0.14 * y
    f = (0.3 + 1.7 * x - 0.9 * y + 0.05 * x * x - 0.11 * x * y + 0.07 * y * y
         + 0.004 * x ** 3 - 0.003 * x * x * y + 0.002 * x * y * y - 0.001 * y ** 3)
    gx = 1.7 + 0.1 * x - 0.11 * y + 0.012 * x * x - 0.006 * x * y + 0.002 * y * y
    gy = -0.9 - 0.11 * x + 0.14 * y - 0.003 * x * x + 0.004 * x * y - 0.003 * y * y
    return f, gx, gy


@pytest.mark.parametrize("order", [1, 2, 3])
def test_oracle_reproduces_polynomials_of_element_degree(order):
    m = structured_mesh(order, 5, 4, 10.0, 6.0)
    it = Interpolator(m)
    f, _, _ = _poly(order, m.nodes[:, 0], m.nodes[:, 1])
    rng = np.random.default_rng(order)
    for x, y in zip(rng.uniform(0, 10, 40), rng.uniform(0, 6, 40)):
        v, gx, gy, e = it.evaluate(x, y, f, gradient=True)
        ev, egx, egy = _poly(order, x, y)
        assert e >= 0
        assert abs(v - ev) < 1e-11
        assert abs(gx - egx) < 1e-10 and abs(gy - egy) < 1e-10


@pytest.mark.parametrize("order", [1, 2, 3])
def test_oracle_reproduces_nodal_values(order):
    m = structured_mesh(order, 3, 2, 3.0, 2.0)
    it = Interpolator(m)
    f = np.random.default_rng(0).standard_normal(m.num_nodes)
    for n in range(m.num_nodes):
        v, _, _, e = it.evaluate(m.nodes[n, 0], m.nodes[n, 1], f)
        assert e >= 0 and abs(v - f[n]) < 1e-12


def test_oracle_first_element_wins_on_shared_edges():
    m = structured_mesh(1, 3, 2, 3.0, 2.0)   # unit cells
    it = Interpolator(m)
    # on the diagonal of cell (1, 0): both triangles of the cell, t = 0 first
    assert it.find_element(1.5, 0.5) == 2 * (0 * 3 + 1) + 0
    # on the vertical line x = 1 inside row 0: cell 0's t = 1 precedes cell 1
    assert it.find_element(1.0, 0.25) == 2 * (0 * 3 + 0) + 1
    # on the horizontal line y = 1: row 0's t = 1 precedes row 1
    assert it.find_element(2.25, 1.0) == 2 * (0 * 3 + 2) + 1
    # interior vertex (1, 1): the first of its six triangles
    assert it.find_element(1.0, 1.0) == 1
    assert it.find_element(-0.5, 0.5) == -1


def test_oracle_outside_points_take_nearest_node_and_its_estimate():
    m = structured_mesh(1, 1, 1, 1.0, 1.0)   # nodes (0,0) (1,0) (0,1) (1,1)
    it = Interpolator(m)
    f = np.array([1.0, 3.0, 2.0, 7.0])
    v, gx, gy, e = it.evaluate(-0.3, -0.2, f, gradient=True)
    assert e == -1 and v == 1.0
    # node 0 lies in element 0 only: neighbours 1 at (1, 0) and 2 at (0, 1),
    # each at distance 1: grad = ((3-1) (1,0) + (2-1) (0,1)) / 2
    assert (gx, gy) == (1.0, 0.5)
    # node 3 at (1, 1) lies in element 1 (nodes 1, 3, 2): neighbours 1 and 2
    v, gx, gy, _ = it.evaluate(1.4, 1.1, f, gradient=True)
    assert v == 7.0
    assert gx == pytest.approx(((3 - 7) * 0 + (2 - 7) * -1) / 2)
    assert gy == pytest.approx(((3 - 7) * -1 + (2 - 7) * 0) / 2)
    # ties go to the first node; zero mode and non-finite points give 0
    assert it.evaluate(0.5, -1.0, f)[0] == 1.0
    assert it.evaluate(-0.3, -0.2, f, zero_outside=True)[:3] == (0.0, 0.0, 0.0)
    assert it.evaluate(float("nan"), 0.5, f)[0] == 0.0
    assert it.evaluate(1e200, 0.5, f)[0] == 0.0


def test_oracle_matches_reference_python_interpolator_golden():
    """The reference's own P1 interpolator (frontend/qdsim/fe_interpolator.py
    with its quadtree), run by tests/golden/make_interp_golden.py: values,
    gradients and elements at points strictly inside one element, and the
    nearest-node values of points outside the mesh, except at the interior
    points its quadtree misses (recorded in the fixture)."""
    import os
    d = np.load(os.path.join(os.path.dirname(__file__), "golden", "interp_p1.npz"))
    m = structured_mesh(1, int(d["nx"]), int(d["ny"]), float(d["Lx"]), float(d["Ly"]))
    it = Interpolator(m)
    n_in = int(d["n_inside"])
    val, gx, gy, el = it.evaluate_many(d["x"], d["y"], d["field"], gradient=True)
    ok = ~d["quadtree_miss"]
    ok_in = ok[:n_in]
    np.testing.assert_array_equal(el[ok], d["element"][ok])
    np.testing.assert_allclose(val[0][ok], d["value"][ok], rtol=0, atol=1e-13)
    np.testing.assert_allclose(gx[0, :n_in][ok_in], d["grad_x"][ok_in], rtol=0, atol=1e-12)
    np.testing.assert_allclose(gy[0, :n_in][ok_in], d["grad_y"][ok_in], rtol=0, atol=1e-12)
    assert (el[:n_in] >= 0).all() and (el[n_in:] < 0).all()
    assert ok_in.sum() >= 390 and ok[n_in:].all()
    # a recorded fact about the reference: where its quadtree missed, the
    # element it returned does not contain the point, and the oracle's does
    for i in np.flatnonzero(~ok):
        v = m.nodes[m.elems[d["element"][i], :3]]
        assert barycentric(d["x"][i], d["y"][i], v).min() < -1e-3
        v = m.nodes[m.elems[el[i], :3]]
        assert barycentric(d["x"][i], d["y"][i], v).min() >= -1e-10


def test_oracle_barycentric_formula():
    lam = barycentric(0.25, 0.5, [(0.0, 0.0), (1.0, 0.0), (0.0, 1.0)])
    assert np.allclose(lam, [0.25, 0.25, 0.5])


def test_interpolate_entry_point_rejects_bad_arguments_without_gpu():
    """Argument checks of qd_fe_interpolate return before any device work."""
    from qdsim_b200 import _native as N
    L = N.lib()
    p = C.c_void_p(256)   # never dereferenced: every call below is rejected or empty

    def call(order=1, nx=4, ny=3, Lx=1.0, Ly=1.0, nfield=1, stride=20, npts=5, field=p,
             gx=None, gy=None, outside=0):
        return L.qd_fe_interpolate(order, nx, ny, Lx, Ly, nfield, stride, field, npts, p, p, p,
                                   gx, gy, None, outside, None)

    assert call(order=0) == N.QD_ERR_INVALID
    assert call(order=4) == N.QD_ERR_INVALID
    assert call(nx=0) == N.QD_ERR_INVALID
    assert call(Lx=0.0) == N.QD_ERR_INVALID
    assert call(Ly=float("nan")) == N.QD_ERR_INVALID
    assert call(Lx=float("inf")) == N.QD_ERR_INVALID
    assert call(nfield=0) == N.QD_ERR_INVALID
    assert call(stride=19) == N.QD_ERR_INVALID           # (4+1)(3+1) = 20 nodes
    assert call(order=2, stride=20) == N.QD_ERR_INVALID  # 9 x 7 = 63 nodes
    assert call(gx=p) == N.QD_ERR_INVALID                 # one gradient pointer
    assert call(outside=2) == N.QD_ERR_INVALID
    assert call(field=None) == N.QD_ERR_INVALID
    assert call(npts=-1) == N.QD_ERR_INVALID
    assert call(nx=60000, ny=60000, stride=1 << 40) == N.QD_ERR_LIMIT
    assert call(npts=0) == N.QD_OK                        # nothing to do


def test_frontend_interpolator_host_logic():
    from qdsim_b200 import frontend as F
    inside, lam = F.FEInterpolator.compute_barycentric_coordinates(
        0.25, 0.5, [(0.0, 0.0), (1.0, 0.0), (0.0, 1.0)])
    assert inside and np.allclose(lam, [0.25, 0.25, 0.5])
    inside, _ = F.FEInterpolator.compute_barycentric_coordinates(
        1.0, 1.0, [(0.0, 0.0), (1.0, 0.0), (0.0, 1.0)])
    assert not inside
    mesh = F.Mesh(10e-9, 6e-9, 5, 3, 1)
    fem = F.FEMSolver(mesh, lambda x, y: 0.067 * 9.109e-31, lambda x, y: 0.0,
                      lambda x, y: 0.0, device="cpu")
    with pytest.raises(ValueError):
        fem.set_potential_values(np.zeros(5))
    fem.set_potential_values(np.ones(mesh.get_num_nodes()))
    fem.use_interpolated_potential(True)
    assert fem._use_interp


def test_frontend_physics_callbacks():
    """The reference's physics callbacks (backend/src/physics.cpp) on scalars
    and arrays; the electrostatic part of ``potential`` through a stand-in
    interpolator (its GPU evaluation is covered by the GPU tests of
    FEInterpolator)."""
    from qdsim_b200 import frontend as F
    q = 1.602e-19
    dot, host = {"m_e": 0.041, "Delta_E_c": 0.3}, {"m_e": 0.067, "Delta_E_c": 0.0}
    assert F.effective_mass(0.5, 0.5, dot, host, 1.0) == 0.041
    assert F.effective_mass(1.0, 0.5, dot, host, 1.0) == 0.067
    np.testing.assert_array_equal(F.effective_mass(np.array([0.0, 2.0]), np.zeros(2), dot, host,
                                                   1.0), [0.041, 0.067])
    assert F.epsilon_r(-1.0, 0.0, {"epsilon_r": 12.9}, {"epsilon_r": 13.1}) == 12.9
    assert F.epsilon_r(0.0, 0.0, {"epsilon_r": 12.9}, {"epsilon_r": 13.1}) == 13.1
    # quadratic in (|x| - Lx/2) / d past |x| = Lx/2 - d, the larger of x and y
    assert F.cap(3.0, 0.0, 2.0, 10.0, 10.0, 1.0) == 0.0
    assert F.cap(4.5, 0.0, 2.0, 10.0, 10.0, 1.0) == pytest.approx(2.0 * 0.25)
    assert F.cap(4.5, 4.8, 2.0, 10.0, 10.0, 1.0) == pytest.approx(2.0 * 0.25)
    # dot term alone
    assert F.potential(0.0, 0.0, dot, host, 1.0, "square", []) == pytest.approx(-0.3 * q)
    assert F.potential(2.0, 0.0, dot, host, 1.0, "square", []) == 0.0
    assert F.potential(1.0, 0.0, dot, host, 1.0, "gaussian", []) == pytest.approx(
        -0.3 * np.exp(-0.5) * q)
    deep = {"Delta_E_c": 500.0}
    assert F.potential(0.0, 0.0, deep, host, 1.0, "square", []) == pytest.approx(-100.0 * q)
    # no interpolator: phi[0] clipped to +-100
    assert F.potential(5.0, 0.0, dot, host, 1.0, "square", [250.0, 1.0]) == pytest.approx(100 * q)
    assert F.potential(5.0, 0.0, dot, host, 1.0, "square", [-0.2]) == pytest.approx(-0.2 * q)

    class Stand:
        def interpolate(self, x, y, field):
            return field[0] * x + 300.0 * (y > 10)

    x = np.array([0.0, 0.5, 3.0, 3.0])
    y = np.array([0.0, 0.0, 0.0, 20.0])
    v = F.potential(x, y, dot, host, 1.0, "square", [0.1, 9.0], Stand())
    want = (np.array([-0.3, -0.3, 0.0, 0.0]) + np.array([0.0, 0.05, 0.3, 100.0])) * q
    np.testing.assert_allclose(v, want, rtol=1e-12)

    class Broken:
        def interpolate(self, x, y, field):
            raise RuntimeError("no element")

    assert F.potential(3.0, 0.0, dot, host, 1.0, "square", [-0.25], Broken()) == \
        pytest.approx(-0.25 * q)


def test_frontend_complex_interpolation_host_logic():
    """interpolate_complex splits the field into real and imaginary rows of one
    evaluation and combines them; the evaluation is replaced by the oracle."""
    import torch
    from qdsim_b200 import frontend as F
    mesh = F.Mesh(12e-9, 8e-9, 6, 4, 2)
    fi = F.FEInterpolator(mesh, device="cpu")
    om = structured_mesh(2, 6, 4, 12e-9, 8e-9)
    it = Interpolator(om)
    calls = []

    def fake(x, y, field, gradient=False, element=False, stream=None):
        calls.append(np.asarray(field).shape)
        v = it.evaluate_many(np.asarray(x), np.asarray(y), field)[0]
        return {"value": torch.as_tensor(v)}

    fi._fi.evaluate = fake
    rng = np.random.default_rng(3)
    z = rng.standard_normal(mesh.get_num_nodes()) + 1j * rng.standard_normal(mesh.get_num_nodes())
    x, y = 5.3e-9, 2.9e-9
    re = it.evaluate(x, y, z.real)[0]
    im = it.evaluate(x, y, z.imag)[0]
    assert fi.interpolate_complex(x, y, z, "real") == pytest.approx(re, abs=1e-14)
    assert fi.interpolate_complex(x, y, z, "imag") == pytest.approx(im, abs=1e-14)
    assert fi.interpolate_complex(x, y, z, "abs") == pytest.approx(abs(re + 1j * im), abs=1e-14)
    assert calls == [(2, mesh.get_num_nodes())] * 3
    with pytest.raises(ValueError):
        fi.interpolate_complex(x, y, z, "phase")


def test_frontend_charge_density_callback():
    """q (p - n) from resampled carrier densities (physics.cpp:184-216), with
    a stand-in interpolator; first entries without one, 0 when empty."""
    from qdsim_b200 import frontend as F
    q = 1.602e-19

    class Stand:
        def interpolate(self, x, y, field):
            return field[0] + x

    assert F.charge_density(1.0, 0.0, [2.0, 9.0], [5.0]) == pytest.approx(q * (5.0 - 2.0))
    assert F.charge_density(1.0, 0.0, [], [5.0]) == pytest.approx(q * 5.0)
    assert F.charge_density(1.0, 0.0, [], []) == 0.0
    v = F.charge_density(np.array([0.0, 2.0]), np.zeros(2), [1.0], [3.0], Stand(), Stand())
    np.testing.assert_allclose(v, q * np.array([(3.0 + 0.0) - (1.0 + 0.0),
                                                (3.0 + 2.0) - (1.0 + 2.0)]))

    class Broken:
        def interpolate(self, x, y, field):
            raise RuntimeError("outside")

    assert F.charge_density(0.5, 0.5, [4.0], [1.0], Broken(), None) == pytest.approx(q * -3.0)


def test_field_interpolator_rejects_bad_arguments_without_gpu():
    """FieldInterpolator checks its arguments before any launch."""
    from qdsim_b200.adapt import refine
    from qdsim_b200.interp import FieldInterpolator
    from qdsim_b200.mesh import StructuredMesh
    m = StructuredMesh(2, 4, 3, 4.0, 3.0)
    with pytest.raises(ValueError):
        FieldInterpolator(m, device="cpu", outside="clamp")
    fi = FieldInterpolator(m, device="cpu")
    with pytest.raises(ValueError):
        fi.evaluate([0.5, 1.0], [0.5], np.zeros(m.num_nodes))          # x and y differ
    with pytest.raises(ValueError):
        fi.evaluate([0.5], [0.5], np.zeros(m.num_nodes - 1))           # wrong field length
    with pytest.raises(ValueError):
        fi.evaluate([0.5], [0.5], np.zeros((2, 3, m.num_nodes)))       # not (N,) or (F, N)
    with pytest.raises(TypeError):
        FieldInterpolator(object(), device="cpu")                      # not a mesh


def test_element_buckets_hold_every_candidate():
    """The bucket grid of a refined mesh: every element is listed in each
    cell its (padded) bounding box meets, lists ascend, and for seeded
    points the oracle's containing element is in the bucket of the point's
    cell (so the kernel's first passing element is the scan's)."""
    from oracle.adapt import element_gradients
    from oracle.fem import Mesh
    from oracle.interp import Interpolator
    from qdsim_b200.adapt import refine, refinement_flags
    from qdsim_b200.interp import element_buckets
    from qdsim_b200.mesh import StructuredMesh
    m = StructuredMesh(2, 10, 6, 30.0, 18.0)
    for _ in range(2):
        psi = np.exp(-((m.nodes[:, 0] - 12.0) ** 2 + (m.nodes[:, 1] - 10.0) ** 2) / 18.0)
        g = element_gradients(m.nodes, m.elems, psi)
        m = refine(m, refinement_flags(m, psi, float(np.quantile(np.hypot(*g.T), 0.75))))
    ptr, cel = element_buckets(m.nodes, m.elems, m.nx, m.ny, m.Lx, m.Ly)
    assert ptr[0] == 0 and ptr[-1] == cel.size
    for c in range(m.nx * m.ny):
        lst = cel[ptr[c]:ptr[c + 1]]
        assert np.all(np.diff(lst) > 0)
    hx, hy = m.Lx / m.nx, m.Ly / m.ny
    for e in range(m.num_elements):
        v = m.nodes[m.elems[e, :3]]
        for i in range(int(v[:, 0].min() // hx), min(int(v[:, 0].max() // hx), m.nx - 1) + 1):
            for j in range(int(v[:, 1].min() // hy), min(int(v[:, 1].max() // hy), m.ny - 1) + 1):
                c = j * m.nx + i
                assert e in cel[ptr[c]:ptr[c + 1]]
    om = Mesh(m.order, m.nx, m.ny, m.Lx, m.Ly, m.nodes, m.elems, m.boundary)
    it = Interpolator(om)
    rng = np.random.default_rng(2)
    for x, y in zip(rng.uniform(0, m.Lx, 200), rng.uniform(0, m.Ly, 200)):
        e = it.find_element(x, y)
        c = min(int(y // hy), m.ny - 1) * m.nx + min(int(x // hx), m.nx - 1)
        assert e in cel[ptr[c]:ptr[c + 1]]

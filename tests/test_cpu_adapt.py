"""Adaptive refinement on the host: the reference's gradient flags against the
oracle's element-by-element restatement, and the refined meshes checked for
conformity, orientation, area, node placement and boundary flags. Uniform
refinement must reproduce the structured mesh of twice the cells, which the
oracle's assembly confirms through identical eigenvalues."""
import numpy as np
import pytest

from oracle import adapt as OA
from oracle import fem as O
from qdsim_b200 import adapt as A
from qdsim_b200.fem import build_pattern, dof_map_for
from qdsim_b200.mesh import LOCAL_NODES, StructuredMesh


def _field(nodes):
    x, y = nodes[:, 0], nodes[:, 1]
    return np.exp(-((x - 6.0) ** 2 + (y - 4.0) ** 2) / 8.0)


@pytest.mark.parametrize("order", [1, 2, 3])
def test_flags_match_oracle_restatement(order):
    m = StructuredMesh(order, 10, 6, 12.0, 8.0)
    psi = _field(m.nodes)
    g = OA.element_gradients(m.nodes, m.elems, psi)
    gn = np.sqrt((g ** 2).sum(1))
    for thr in (0.05, 0.2, float(np.median(gn))):
        np.testing.assert_array_equal(A.refinement_flags(m, psi, thr),
                                      OA.refinement_flags(m.nodes, m.elems, psi, thr))


def test_flags_known_answer_linear_field():
    m = StructuredMesh(2, 4, 3, 4.0, 3.0)
    psi = 0.3 * m.nodes[:, 0] - 0.4 * m.nodes[:, 1]      # |grad| = 0.5 everywhere
    assert A.refinement_flags(m, psi, 0.5 - 1e-9).all()
    assert not A.refinement_flags(m, psi, 0.5 + 1e-9).any()
    assert OA.refinement_flags(m.nodes, m.elems, psi, 0.5 - 1e-9).all()


def _areas(nodes, tri):
    p = nodes[tri]
    return 0.5 * ((p[:, 1, 0] - p[:, 0, 0]) * (p[:, 2, 1] - p[:, 0, 1])
                  - (p[:, 2, 0] - p[:, 0, 0]) * (p[:, 1, 1] - p[:, 0, 1]))


def _check_conforming(tm):
    """Every edge is shared by at most two triangles, and no vertex lies on
    the interior of another triangle's edge (no hanging node)."""
    tri = tm.elems[:, :3]
    edges = {}
    for t in tri:
        for a, b in ((0, 1), (1, 2), (2, 0)):
            k = (min(t[a], t[b]), max(t[a], t[b]))
            edges[k] = edges.get(k, 0) + 1
    assert max(edges.values()) <= 2
    verts = np.unique(tri)
    P = tm.nodes[verts]
    for (u, v), cnt in edges.items():
        if cnt != 1:
            continue
        # a boundary edge must lie on the rectangle's boundary; an interior
        # edge seen once would be a hanging-node edge
        pu, pv = tm.nodes[u], tm.nodes[v]
        on_x = np.isclose(pu[0], pv[0]) and (np.isclose(pu[0], 0) or np.isclose(pu[0], tm.Lx))
        on_y = np.isclose(pu[1], pv[1]) and (np.isclose(pu[1], 0) or np.isclose(pu[1], tm.Ly))
        assert on_x or on_y, (pu, pv)
    assert P.shape[0] == verts.size


@pytest.mark.parametrize("order", [1, 2, 3])
def test_refined_mesh_is_conforming_and_consistent(order):
    m = StructuredMesh(order, 10, 6, 12.0, 8.0)
    psi = _field(m.nodes)
    flags = A.refinement_flags(m, psi, 0.2)
    assert 0 < flags.sum() < m.num_elements
    tm = A.refine(m, flags)
    tri = tm.elems[:, :3]
    ar = _areas(tm.nodes, tri)
    assert (ar > 0).all()                                   # orientation kept
    assert np.isclose(ar.sum(), 12.0 * 8.0, rtol=1e-12)     # area conserved
    assert tm.num_elements >= m.num_elements + 3 * int(flags.sum())
    _check_conforming(tm)
    # higher-order nodes sit at their barycentric positions
    V = tm.nodes[tri]
    for a, bc in enumerate(LOCAL_NODES[order]):
        want = (bc[0] * V[:, 0] + bc[1] * V[:, 1] + bc[2] * V[:, 2]) / order
        np.testing.assert_allclose(tm.nodes[tm.elems[:, a]], want, atol=1e-12)
    # each node is used, and boundary flags mark exactly the rectangle's edge
    assert np.unique(tm.elems).size == tm.num_nodes
    x, y = tm.nodes[:, 0], tm.nodes[:, 1]
    geo = np.isclose(x, 0) | np.isclose(x, 12.0) | np.isclose(y, 0) | np.isclose(y, 8.0)
    np.testing.assert_array_equal(tm.boundary, geo)
    # the host pattern builder accepts the refined mesh (row valences in range)
    dm, n = dof_map_for(tm, True)
    P = build_pattern(tm.elems, dm, n, tm.num_nodes)
    assert P.nnz > 0 and n == int((~tm.boundary).sum())


def test_green_closure_bisects_single_split_edges():
    m = StructuredMesh(1, 3, 3, 3.0, 3.0)
    flags = np.zeros(m.num_elements, bool)
    flags[2 * (1 * 3 + 1)] = True                          # one triangle in the middle
    tm = A.refine(m, flags)
    # the flagged triangle becomes 4; each of its 3 neighbours is bisected
    assert tm.num_elements == m.num_elements - 1 + 4 + 3
    _check_conforming(tm)


@pytest.mark.parametrize("order", [1, 2, 3])
def test_uniform_refinement_equals_the_doubled_structured_mesh(order):
    """All elements flagged: the same triangles as the structured mesh of
    twice the cells, so the oracle's assembly gives the same eigenvalues."""
    nx, ny, Lx, Ly = 6, 4, 24.0, 16.0
    m = StructuredMesh(order, nx, ny, Lx, Ly)
    tm = A.refine(m, np.ones(m.num_elements, bool))
    fine = StructuredMesh(order, 2 * nx, 2 * ny, Lx, Ly)
    assert tm.num_elements == fine.num_elements and tm.num_nodes == fine.num_nodes

    def levels(mesh):
        om = O.Mesh(mesh.order, mesh.nx, mesh.ny, mesh.Lx, mesh.Ly, mesh.nodes,
                    mesh.elems, mesh.boundary)
        x, y = mesh.nodes[:, 0], mesh.nodes[:, 1]
        V = -0.3 * np.exp(-((x - 11.0) ** 2 + (y - 7.5) ** 2) / 18.0)
        c = np.full(mesh.num_elements, O.C0_EV_NM2 / 0.067)
        a = O.assemble(om, c, V)
        return O.eig_lowest(a.H, a.M, 4, O.sigma_below(V))[0]

    np.testing.assert_allclose(levels(tm), levels(fine), rtol=1e-10)


def test_trimesh_rejects_mismatched_order_and_flags():
    m = StructuredMesh(2, 2, 2, 2.0, 2.0)
    with pytest.raises(ValueError):
        A.TriMesh(3, m.nodes, m.elems, m.boundary, 2.0, 2.0, 2, 2)
    with pytest.raises(ValueError):
        A.refine(m, np.zeros(3, bool))
    with pytest.raises(ValueError):
        A.refinement_flags(m, np.zeros(5), 0.1)


def test_frontend_adapt_mesh_host_logic(tmp_path, monkeypatch):
    """FEMSolver.adapt_mesh refines the SI and nm meshes alike, keeps the
    reference's accessors, caches the refined mesh by the eigenvector norm
    and reassembles (the GPU assembly is replaced here by a recorder)."""
    from qdsim_b200 import frontend as F
    calls = []
    monkeypatch.setattr(F.FEMSolver, "assemble_matrices", lambda self: calls.append(
        self.mesh.get_num_nodes()))
    mesh = F.Mesh(12e-9, 8e-9, 10, 6, 2)
    fem = F.FEMSolver(mesh, lambda x, y: 0.067 * 9.109e-31 + 0 * x, lambda x, y: 0 * x,
                      lambda x, y: 0 * x, device="cpu")
    nodes = mesh.get_nodes()
    psi = _field(nodes * 1e9)
    thr = 0.2e9                                  # per metre (SI mesh)
    n0, e0 = mesh.get_num_nodes(), mesh.get_num_elements()
    fem.adapt_mesh(psi, thr, str(tmp_path))
    assert mesh.is_refined() and mesh.get_num_elements() > e0 and mesh.get_num_nodes() > n0
    assert calls == [mesh.get_num_nodes()]
    assert (mesh.get_nx(), mesh.get_ny(), mesh.get_element_order()) == (10, 6, 2)
    np.testing.assert_allclose(mesh._nm.nodes * 1e-9, mesh._si.nodes, rtol=1e-12, atol=1e-24)
    np.testing.assert_array_equal(mesh._nm.elems, mesh._si.elems)
    files = list(tmp_path.iterdir())
    assert len(files) == 1 and files[0].name == f"mesh_{np.linalg.norm(psi):.6f}.npz"
    # same eigenvector on a fresh solver: the cached mesh is loaded
    mesh2 = F.Mesh(12e-9, 8e-9, 10, 6, 2)
    fem2 = F.FEMSolver(mesh2, fem.m_star, fem.V, fem.cap, device="cpu")
    fem2.adapt_mesh(psi, thr, str(tmp_path))
    np.testing.assert_array_equal(mesh2.get_elements(), mesh.get_elements())
    np.testing.assert_allclose(mesh2.get_nodes(), mesh.get_nodes(), rtol=0, atol=0)
    # the interpolator works on the refined mesh through its bucket grid
    fi = fem.get_interpolator()
    assert fi._fi._tri is not None and fi._fi._tri["cell_ptr"].numel() == 10 * 6 + 1


def test_adaptive_step_improves_levels_with_fewer_elements():
    """One adapt step on a dot (the oracle's assembly and eigensolve on the
    refined mesh): the lowest levels move toward those of a mesh four times
    finer, with fewer elements than refining everything."""
    Lx, Ly, nx, ny = 40.0, 30.0, 16, 12

    def levels(mesh, k=3):
        om = O.Mesh(mesh.order, mesh.nx, mesh.ny, mesh.Lx, mesh.Ly, mesh.nodes,
                    mesh.elems, mesh.boundary)
        x, y = mesh.nodes[:, 0], mesh.nodes[:, 1]
        V = -0.4 * np.exp(-((x - 17.0) ** 2 + (y - 14.0) ** 2) / (2 * 3.0 ** 2))
        c = np.full(mesh.num_elements, O.C0_EV_NM2 / 0.067)
        a = O.assemble(om, c, V)
        E, X = O.eig_lowest(a.H, a.M, k, O.sigma_below(V))
        psi = np.zeros(mesh.num_nodes)
        psi[a.dm >= 0] = X[a.dm[a.dm >= 0], 0]
        return E, psi

    coarse = StructuredMesh(1, nx, ny, Lx, Ly)
    E_c, psi = levels(coarse)
    E_f, _ = levels(StructuredMesh(1, 4 * nx, 4 * ny, Lx, Ly))
    g = OA.element_gradients(coarse.nodes, coarse.elems, np.abs(psi))
    gn = np.sqrt((g ** 2).sum(1))
    flags = A.refinement_flags(coarse, np.abs(psi), float(np.quantile(gn, 0.6)))
    tm = A.refine(coarse, flags)
    E_a, _ = levels(tm)
    assert tm.num_elements < 4 * coarse.num_elements
    assert (np.abs(E_a - E_f) < 0.6 * np.abs(E_c - E_f)).all(), (E_c, E_a, E_f)


def test_host_batch_accepts_a_refined_mesh():
    """The host half of the eigensolve path on a refined mesh: HostBatch
    builds its pattern and arrays for a TriMesh (natural boundaries, as the
    frontend's EigenSolver uses, so no lattice preconditioner is asked for)."""
    from qdsim_b200 import batch as B
    from qdsim_b200.workloads import Dot
    m = StructuredMesh(2, 10, 6, 12.0, 8.0)
    tm = A.refine(m, A.refinement_flags(m, _field(m.nodes), 0.2))
    c = np.full(tm.num_elements, 0.5)
    V = -0.1 * _field(tm.nodes)
    hb = B.HostBatch([Dot(tm, c, V)], dirichlet=False)
    assert hb.n == tm.num_nodes and hb.prec_specs is None
    assert hb.arrays["elems"].shape == tm.elems.shape
    assert int(hb.arrays["rowptr"][-1]) == hb.nnz
    # the same topology twice hits the pattern cache (shape_key of the TriMesh)
    hb2 = B.HostBatch([Dot(tm, c, V), Dot(tm, c, V)], dirichlet=False)
    assert hb2.nnz == 2 * hb.nnz


@pytest.mark.parametrize("order", [1, 2])
def test_repeated_refinement_stays_conforming_and_shape_regular(order):
    """Green triangles are never bisected again (green removal): over
    repeated refinements the mesh stays conforming, the smallest angle does
    not shrink after the first step, and vertex valences stay within the 16
    elements per node the pattern builder accepts."""
    cur = StructuredMesh(order, 10, 6, 12.0, 8.0)
    first_min = None
    for step in range(4):
        cur = A.refine(cur, A.refinement_flags(cur, _field(cur.nodes), 0.15))
        _check_conforming(cur)
        tri = cur.elems[:, :3]
        ar = _areas(cur.nodes, tri)
        assert (ar > 0).all() and np.isclose(ar.sum(), 96.0, rtol=1e-12)
        assert np.unique(cur.elems).size == cur.num_nodes
        P = cur.nodes[tri]
        ang = []
        for k in range(3):
            u, v = P[:, (k + 1) % 3] - P[:, k], P[:, (k + 2) % 3] - P[:, k]
            c = np.sum(u * v, 1) / np.linalg.norm(u, axis=1) / np.linalg.norm(v, axis=1)
            ang.append(np.degrees(np.arccos(np.clip(c, -1, 1))))
        amin = float(np.min(ang))
        first_min = amin if first_min is None else first_min
        assert amin >= first_min - 1e-9
        assert np.bincount(tri.ravel()).max() <= 16
        dm, n = dof_map_for(cur, True)
        build_pattern(cur.elems, dm, n, cur.num_nodes)


def test_frontend_adaptive_mesh_helpers():
    """qdsim_cpp.AdaptiveMesh's static helpers on the frontend Mesh."""
    from qdsim_b200 import frontend as F
    mesh = F.Mesh(12e-9, 8e-9, 10, 6, 1)
    psi = _field(mesh.get_nodes() * 1e9)
    flags = F.AdaptiveMesh.compute_refinement_flags(mesh, psi, 0.2e9)
    assert isinstance(flags, list) and 0 < sum(flags) < mesh.get_num_elements()
    np.testing.assert_array_equal(flags, OA.refinement_flags(mesh.get_nodes(),
                                                             mesh.get_elements(), psi, 0.2e9))
    # right isosceles cells: quality 4 sqrt(3) (h^2/2) / (4 h^2) = sqrt(3)/2
    sq = F.Mesh(10e-9, 10e-9, 5, 5, 1)
    assert F.AdaptiveMesh.compute_triangle_quality(sq, 0) == pytest.approx(np.sqrt(3) / 2)
    e0 = mesh.get_num_elements()
    F.AdaptiveMesh.refine_mesh(mesh, flags)
    assert mesh.is_refined() and mesh.get_num_elements() > e0
    assert F.AdaptiveMesh.is_mesh_conforming(mesh)


def test_red_children_follow_the_reference_order():
    """A flagged element's four children replace it in place, in the order and
    vertex order of adaptive_mesh.cpp:105-108: (n0, m01, m20), (n1, m12, m01),
    (n2, m20, m12), (m01, m12, m20)."""
    m = StructuredMesh(1, 3, 3, 3.0, 3.0)
    e = 2 * (1 * 3 + 1)                                     # the middle cell's t = 0
    flags = np.zeros(m.num_elements, bool)
    flags[e] = True
    tm = A.refine(m, flags)
    n0, n1, n2 = (m.nodes[i] for i in m.elems[e])
    m01, m12, m20 = (n0 + n1) / 2, (n1 + n2) / 2, (n2 + n0) / 2
    want = [(n0, m01, m20), (n1, m12, m01), (n2, m20, m12), (m01, m12, m20)]
    # children are consecutive, where the parent was: after the outputs of
    # the elements before it (a bisected neighbour among them yields two)
    P = tm.nodes[tm.elems[:, :3]]
    first = [i for i in range(tm.num_elements) if np.allclose(P[i], np.array(want[0]))]
    assert len(first) == 1
    for k, tri in enumerate(want):
        np.testing.assert_allclose(P[first[0] + k], np.array(tri), atol=1e-12)
    # two neighbours precede it (across its bottom and left edges), each
    # bisected into two
    assert first[0] == e + 2

"""Assembly kernel vs the FP64 oracle: CSR values within 1e-12 (norm-wise)."""
import numpy as np
import pytest

from oracle import fem as O

pytestmark = pytest.mark.gpu


def _rel_err(a, b):
    a = a.toarray() if hasattr(a, "toarray") else a
    b = b.toarray() if hasattr(b, "toarray") else b
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


def _case(order, nx, ny, seed, cap):
    rng = np.random.default_rng(seed)
    Lx, Ly = nx * 1.3, ny * 0.9
    om = O.structured_mesh(order, nx, ny, Lx, Ly)
    # jitter interior nodes so elements are not all congruent
    return om, rng


@pytest.mark.parametrize("order", [1, 2, 3])
@pytest.mark.parametrize("dirichlet", [True, False])
def test_assembly_matches_oracle(cuda, order, dirichlet):
    from qdsim_b200 import fem as F, mesh as Mh
    nx, ny = 9, 6
    Lx, Ly = 13.0, 7.0
    rng = np.random.default_rng(order * 10 + dirichlet)
    om = O.structured_mesh(order, nx, ny, Lx, Ly)
    m = Mh.StructuredMesh(order, nx, ny, Lx, Ly)
    c = rng.uniform(0.3, 1.2, m.num_elements)
    V = rng.uniform(-0.4, 0.1, m.num_nodes)
    W = rng.uniform(0.0, 0.05, m.num_nodes)
    ref = O.assemble(om, c, V, W, dirichlet=dirichlet)
    prob = F.FEMProblem(m, dirichlet=dirichlet, device=cuda)
    out = prob.assemble(c, V, W)
    H = prob.to_scipy(out["H"])
    M = prob.to_scipy(out["M"])
    Wi = prob.to_scipy(out["Himag"])
    assert _rel_err(H, ref.H) < 1e-12
    assert _rel_err(M, ref.M) < 1e-12
    assert _rel_err(-Wi, ref.Wm) < 1e-12
    # same pattern, same ordering
    assert np.array_equal(H.indptr, ref.H.indptr) and np.array_equal(H.indices, ref.H.indices)


def test_assembly_c1_and_determinism(cuda):
    from qdsim_b200 import fem as F, mesh as Mh
    om, c, V = O.dot_config_c1(seed=0)
    m = Mh.StructuredMesh(1, 100, 50, 100.0, 50.0)
    prob = F.FEMProblem(m, device=cuda)
    a = prob.assemble(c, V)
    b = prob.assemble(c, V)
    assert prob.nnz == 33367               # interior pattern of the 100x50 P1 mesh
    ref = O.assemble(om, c, V)
    assert _rel_err(prob.to_scipy(a["H"]), ref.H) < 1e-12
    assert _rel_err(prob.to_scipy(a["M"]), ref.M) < 1e-12
    # bitwise reproducible (no atomics)
    assert bool((a["H"] == b["H"]).all()) and bool((a["M"] == b["M"]).all())


def test_assembly_full_pattern_nnz_matches_reference(cuda):
    """The full (no elimination) P1 pattern of the 101x51-point mesh has the
    35,451 nonzeros the compiled reference FixedOpenSystemSolver reports."""
    from qdsim_b200 import fem as F, mesh as Mh
    m = Mh.StructuredMesh(1, 100, 50, 100.0, 50.0)
    prob = F.FEMProblem(m, dirichlet=False, device=cuda)
    assert prob.nnz == 35451


def test_degenerate_element_flagged(cuda):
    from qdsim_b200 import fem as F, mesh as Mh, _native as N
    m = Mh.StructuredMesh(1, 4, 3, 4.0, 3.0)
    m.nodes[m.elems[0, 1]] = m.nodes[m.elems[0, 0]]   # collapse one element
    prob = F.FEMProblem(m, dirichlet=False, device=cuda)
    with pytest.raises(N.QDError):
        prob.assemble(np.ones(m.num_elements), np.zeros(m.num_nodes))
    m2 = Mh.StructuredMesh(1, 4, 3, 4.0, 3.0)
    prob2 = F.FEMProblem(m2, dirichlet=False, device=cuda)
    V = np.zeros(m2.num_nodes)
    V[3] = np.nan
    with pytest.raises(N.QDError):
        prob2.assemble(np.ones(m2.num_elements), V)

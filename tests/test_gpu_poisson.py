"""Jacobi-PCG Poisson step vs the FP64 oracle (sparse LU with Dirichlet elimination)."""
import numpy as np
import pytest

from oracle import fem as O, poisson as OP

pytestmark = pytest.mark.gpu


def _setup(nx=60, ny=20, Lx=300.0, Ly=100.0, seed=0):
    rng = np.random.default_rng(seed)
    om = O.structured_mesh(1, nx, ny, Lx, Ly)
    eps = rng.uniform(10.0, 14.0, om.num_elements)
    x = om.nodes[:, 0]
    rho = 1.602176634e-19 * 1e24 * np.where(x < Lx / 2, -1.0, 1.0) * (
        1 + 0.1 * rng.standard_normal(om.num_nodes))
    return om, eps, rho


@pytest.mark.parametrize("nrhs", [1, 3, 64])
def test_pcg_matches_oracle(cuda, nrhs):
    from qdsim_b200 import mesh as Mh, poisson as P
    om, eps, rho = _setup()
    rng = np.random.default_rng(1)
    R = rho[:, None] * rng.uniform(0.5, 1.5, (1, nrhs))
    vp = np.zeros(nrhs)
    vn = rng.uniform(0.0, 1.0, nrhs)
    ref = OP.solve(om, eps, R, vp, vn)
    m = Mh.StructuredMesh(1, om.nx, om.ny, om.Lx, om.Ly)
    prob = P.PoissonProblem(m, eps, device=cuda)
    if nrhs == 1:
        phi = prob.solve(R[:, 0], vp[0], vn[0], tol=1e-13)
    else:
        phi = prob.solve(R, vp, vn, tol=1e-13)
    got = phi.cpu().numpy().reshape(om.num_nodes, -1)
    err = np.abs(got - ref.reshape(om.num_nodes, -1)).max() / np.abs(ref).max()
    assert err < 1e-9, (err, prob.last_iters, prob.last_relres)
    assert prob.last_relres <= 1e-13


def test_pcg_zero_rhs_is_linear_ramp(cuda):
    from qdsim_b200 import mesh as Mh, poisson as P
    m = Mh.StructuredMesh(1, 10, 4, 50.0, 20.0)
    prob = P.PoissonProblem(m, np.full(m.num_elements, 12.0), device=cuda)
    phi = prob.solve(np.zeros(m.num_nodes), 0.0, 1.0).cpu().numpy()
    # no charge: the potential is the linear ramp between the contacts
    assert np.allclose(phi, m.nodes[:, 0] / 50.0, atol=1e-10)


def test_pcg_reproducible(cuda):
    from qdsim_b200 import mesh as Mh, poisson as P
    om, eps, rho = _setup(seed=3)
    m = Mh.StructuredMesh(1, om.nx, om.ny, om.Lx, om.Ly)
    prob = P.PoissonProblem(m, eps, device=cuda)
    a = prob.solve(rho, 0.0, 0.7).clone()
    b = prob.solve(rho, 0.0, 0.7)
    assert bool((a == b).all())

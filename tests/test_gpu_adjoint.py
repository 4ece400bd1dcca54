"""Adjoint gradients (qd_adjoint, autograd) vs the FP64 oracle gradient and
central finite differences of FP64 oracle eigenvalues."""
import numpy as np
import pytest

from oracle import adjoint as OA, fem as O

pytestmark = pytest.mark.gpu
W = np.array([0.0, 2.0, 1.0, 1.0])     # L = E1+E2+E3+E4 + (E2 - E1)


def _case(order=3, nx=16, ny=8):
    rng = np.random.default_rng(7)
    Lx, Ly = 2.0 * nx, 2.0 * ny
    om = O.structured_mesh(order, nx, ny, Lx, Ly)
    x, y = om.nodes[:, 0], om.nodes[:, 1]
    depth, w = 0.3, 5.0
    V = -depth * np.exp(-((x - 0.47 * Lx) ** 2 + 1.3 * (y - 0.52 * Ly) ** 2) / (2 * w * w))
    inv_m = 1.0 / np.where(rng.random(om.num_elements) < 0.5, 0.041, 0.067)
    return om, V, inv_m


def _oracle_E(om, V, inv_m, k=4):
    a = O.assemble(om, O.C0_EV_NM2 * inv_m, V)
    E, X = O.eig_lowest(a.H, a.M, k, O.sigma_below(V))
    return E, X, a


def test_adjoint_kernel_matches_oracle_gradient(cuda):
    import torch
    from qdsim_b200 import adjoint as A, fem as F, mesh as Mh
    om, V, inv_m = _case()
    E, X, a = _oracle_E(om, V, inv_m)
    psi_nodal = np.zeros((om.num_nodes, 4))
    psi_nodal[a.dm >= 0] = X[a.dm[a.dm >= 0]]
    gV, gc = OA.gradients(om, psi_nodal, W)
    m = Mh.StructuredMesh(3, om.nx, om.ny, om.Lx, om.Ly)
    prob = F.FEMProblem(m, device=cuda)
    dV, dc = A.energy_gradients(prob, torch.from_numpy(X), W)
    assert np.abs(dV.cpu().numpy() - gV).max() <= 1e-11 * np.abs(gV).max()
    assert np.abs(dc.cpu().numpy() - gc).max() <= 1e-11 * np.abs(gc).max()


def test_autograd_matches_finite_differences(cuda):
    import torch
    from qdsim_b200 import adjoint as A, mesh as Mh
    om, V, inv_m = _case()
    m = Mh.StructuredMesh(3, om.nx, om.ny, om.Lx, om.Ly)
    Vt = torch.tensor(V, device=cuda, requires_grad=True)
    it = torch.tensor(inv_m, device=cuda, requires_grad=True)
    E = A.lowest_eigenvalues(Vt, it, m, 4, b=8, precision="fp64", tol=1e-12, max_iter=2000)
    loss = (torch.as_tensor(W, device=cuda) * E).sum()
    loss.backward()
    gV, gm = Vt.grad.cpu().numpy(), it.grad.cpu().numpy()
    rng = np.random.default_rng(11)
    h = 1e-6

    def L(Vx, ix):
        return float(W @ _oracle_E(om, Vx, ix)[0])

    for _ in range(4):
        dv = rng.standard_normal(om.num_nodes)
        di = rng.standard_normal(om.num_elements)
        fd_v = (L(V + h * dv, inv_m) - L(V - h * dv, inv_m)) / (2 * h)
        hi = h * float(np.mean(inv_m))      # step 1e-6 relative to 1/m*
        fd_i = (L(V, inv_m + hi * di) - L(V, inv_m - hi * di)) / (2 * hi)
        assert abs(gV @ dv - fd_v) <= 1e-6 * max(abs(fd_v), 1e-8), (gV @ dv, fd_v)
        assert abs(gm @ di - fd_i) <= 1e-6 * max(abs(fd_i), 1e-8), (gm @ di, fd_i)


@pytest.mark.parametrize("unused", [0])
def test_cluster_weights_symmetric(unused):
    from qdsim_b200.adjoint import cluster_weights
    w = cluster_weights([-0.3, -0.2, -0.2 + 1e-12, -0.1], [0.0, 2.0, 1.0, 1.0])
    assert np.allclose(w, [0.0, 1.5, 1.5, 1.0])

"""Adjoint gradients (qd_adjoint, autograd) vs the FP64 oracle gradient and
central finite differences of FP64 oracle eigenvalues: a small P3 dot, the
differentiation configuration at its stated size (P3 150x75 cells, 32 + 32
seeded directions against tests/golden/c3_fd.npz), and the open system's
complex-symmetric CAP pencil."""
import os
import sys

import numpy as np
import pytest

from oracle import adjoint as OA, fem as O

HERE = os.path.dirname(os.path.abspath(__file__))

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


def _c3():
    sys.path.insert(0, os.path.join(HERE, "golden"))
    import make_c3_golden as G
    z = np.load(os.path.join(HERE, "golden", "c3_fd.npz"))
    _, om, V, inv_m = G._problem()
    return G, z, om, V, inv_m


def test_c3_kernel_matches_oracle_gradient_at_size(cuda):
    """qd_adjoint on the oracle's own eigenvectors (P3 150x75 cells, 100,576
    DOFs, 4 states) equals the oracle gradient at 1e-11."""
    import torch
    from qdsim_b200 import adjoint as A, fem as F, mesh as Mh
    G, z, om, V, inv_m = _c3()
    a = O.assemble(om, O.C0_EV_NM2 * inv_m, V)
    E, X = O.eig_lowest(a.H, a.M, 4, O.sigma_below(V))
    psi = np.zeros((om.num_nodes, 4))
    keep = a.dm >= 0
    psi[keep] = X[a.dm[keep]]
    gV, gc = OA.gradients(om, psi, z["weights"])
    prob = F.FEMProblem(Mh.StructuredMesh(3, 150, 75, 150.0, 75.0), device=cuda)
    dV, dc = A.energy_gradients(prob, torch.from_numpy(X), z["weights"])
    assert np.abs(dV.cpu().numpy() - gV).max() <= 1e-11 * np.abs(gV).max()
    assert np.abs(dc.cpu().numpy() - gc).max() <= 1e-11 * np.abs(gc).max()


def test_c3_autograd_matches_committed_finite_differences(cuda):
    """End to end at the configuration's size: GPU assembly, FP64 LOBPCG and
    the adjoint through torch.autograd; the gradient's projections on the 32
    seeded V directions and the 32 seeded 1/m* directions equal the oracle's
    central differences (step 1e-6) to 1e-6 of the largest, and the gradient
    equals the FP64 oracle gradient to 1e-6.  E2 and E3 are 4.5e-5 eV apart
    and weighted differently, so their eigenvectors must be resolved well
    inside that gap: the solve runs to a residual far below the eigenvalue
    target (tol 1e-22 on the quadratic estimate, capped at 400 iterations)."""
    import torch
    from qdsim_b200 import adjoint as A, mesh as Mh
    G, z, om, V, inv_m = _c3()
    m = Mh.StructuredMesh(3, 150, 75, 150.0, 75.0)
    Vt = torch.tensor(V, device=cuda, requires_grad=True)
    it = torch.tensor(inv_m, device=cuda, requires_grad=True)
    E = A.lowest_eigenvalues(Vt, it, m, 4, b=8, precision="fp64", tol=1e-22, max_iter=400)
    assert np.abs(E.detach().cpu().numpy() - z["E"][:4]).max() <= 1e-12 * abs(z["E"][0])
    loss = (torch.as_tensor(z["weights"], device=cuda) * E).sum()
    loss.backward()
    gV, gm = Vt.grad.cpu().numpy(), it.grad.cpu().numpy()
    dv, di = G.directions(om.num_nodes, om.num_elements, int(z["seed"]))
    pv, pm = dv @ gV, di @ gm
    assert np.abs(pv - z["fd_v"]).max() <= 1e-6 * np.abs(z["fd_v"]).max()
    assert np.abs(pm - z["fd_m"]).max() <= 1e-6 * np.abs(z["fd_m"]).max()


def _cap_case():
    from qdsim_b200 import workloads as W
    d = W.c2_dot(0, nx=24, ny=12)
    om = O.structured_mesh(2, 24, 12, 200.0, 100.0)
    return d, om


def test_cap_kernel_matches_oracle_gradient(cuda):
    """Complex-symmetric pencil: qd_adjoint on the oracle's bilinearly
    normalised complex eigenvectors with complex weights equals the oracle
    gradient at 1e-11."""
    import torch
    from qdsim_b200 import adjoint as A, fem as F
    d, om = _cap_case()
    a = O.assemble(om, d.c, d.V, d.W)
    E, X = O.eig_nearest_complex(a.H - 1j * a.Wm, a.M, 6, -0.05)
    rng = np.random.default_rng(5)
    w = rng.uniform(0.5, 1.5, 6) - 1j * rng.uniform(-1.0, 1.0, 6)
    psi = np.zeros((om.num_nodes, 6), complex)
    keep = a.dm >= 0
    psi[keep] = X[a.dm[keep]]
    gV, gc = OA.gradients(om, psi, w)
    prob = F.FEMProblem(d.mesh, device=cuda)
    dV, dc = A.energy_gradients(prob, torch.from_numpy(X), w)
    assert np.abs(dV.cpu().numpy() - gV).max() <= 1e-11 * np.abs(gV).max()
    assert np.abs(dc.cpu().numpy() - gc).max() <= 1e-11 * np.abs(gc).max()


def test_cap_autograd_matches_finite_differences(cuda):
    """The open system's eigenvalues nearest -0.05 eV through
    torch.autograd (GPU assembly, complex LOBPCG, complex adjoint) against
    central differences of the oracle's shift-invert eigenvalues: a real loss
    of both parts of six complex levels, three V and three 1/m* directions,
    1e-6 relative."""
    import torch
    from qdsim_b200 import adjoint as A
    d, om = _cap_case()
    k, sigma = 6, -0.05
    inv_m = d.c / O.C0_EV_NM2
    Vt = torch.tensor(d.V, device=cuda, requires_grad=True)
    it = torch.tensor(inv_m, device=cuda, requires_grad=True)
    E = A.nearest_eigenvalues(Vt, it, d.mesh, d.W, k, sigma, nev=32, b=40, precision="fp64",
                              tol=1e-11)
    rng = np.random.default_rng(3)
    wa, wb = rng.uniform(0.5, 1.5, k), rng.uniform(-1.0, 1.0, k)
    Eo, _ = O.eig_nearest_complex(O.assemble(om, d.c, d.V, d.W).H
                                  - 1j * O.assemble(om, d.c, d.V, d.W).Wm,
                                  O.assemble(om, d.c, d.V, d.W).M, k, sigma)
    En = E.detach().cpu().numpy()
    assert np.abs(np.sort_complex(En) - np.sort_complex(Eo)).max() <= 1e-9 * np.abs(Eo).max()
    loss = (torch.as_tensor(wa, device=cuda) * E.real + torch.as_tensor(wb, device=cuda)
            * E.imag).sum()
    loss.backward()
    gV, gm = Vt.grad.cpu().numpy(), it.grad.cpu().numpy()

    def L(Vx, ix):
        a = O.assemble(om, O.C0_EV_NM2 * ix, Vx, d.W)
        Ex, _ = O.eig_nearest_complex(a.H - 1j * a.Wm, a.M, k, sigma)
        idx = [int(np.argmin(np.abs(Ex - e))) for e in En]
        Ex = Ex[idx]
        return float(wa @ Ex.real + wb @ Ex.imag)

    h = 1e-6
    for _ in range(3):
        dv = rng.standard_normal(om.num_nodes)
        fd = (L(d.V + h * dv, inv_m) - L(d.V - h * dv, inv_m)) / (2 * h)
        assert abs(gV @ dv - fd) <= 1e-6 * abs(fd), (gV @ dv, fd)
        di = rng.standard_normal(om.num_elements)
        hi = h * float(np.mean(inv_m))
        fd = (L(d.V, inv_m + hi * di) - L(d.V, inv_m - hi * di)) / (2 * hi)
        assert abs(gm @ di - fd) <= 1e-6 * abs(fd), (gm @ di, fd)

"""Batched self-consistent loop (qd_sc_* + batched LOBPCG + batched PCG) vs
its FP64 restatement, and the implicit bias derivative vs finite differences."""
import dataclasses

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _small(n_bias=3):
    from qdsim_b200 import workloads as W
    return W.c5_junction(n_bias=n_bias, nx=40, ny=16, Lx=40.0, Ly=16.0)


def test_sc_loop_matches_restatement(cuda):
    from oracle import fem as O, sc as OS
    from qdsim_b200.sc import BatchedSC
    j = _small()
    sc = BatchedSC(j, k=4, device=cuda, precision="fp64", tol=1e-13, pcg_tol=1e-14)
    phi, err = sc.solve(iterations=12)
    jo = dataclasses.replace(j, mesh=O.structured_mesh(1, 40, 16, 40.0, 16.0))
    phi_o, err_o, E_o = OS.run(jo, k=4, iterations=12)
    phi = phi.cpu().numpy()
    # iterations 0-4 damping, 5-11 Anderson with the line search
    rel = np.abs(phi - phi_o).max() / np.abs(phi_o).max()
    assert rel < 1e-6, rel
    assert np.allclose(err.cpu().numpy(), err_o, rtol=1e-4, atol=1e-12)
    E = sc.E.cpu().numpy()
    assert np.allclose(E, E_o, rtol=1e-8)


def test_sc_implicit_bias_derivative(cuda):
    from qdsim_b200.sc import BatchedSC
    j = _small(n_bias=2)
    sc = BatchedSC(j, k=4, device=cuda, precision="fp64", tol=1e-13, pcg_tol=1e-14)
    phi, err = sc.solve(iterations=60)
    assert err[-1].max().item() < 1e-9, err[-1]
    dE = sc.dE1_dbias(phi).cpu().numpy()
    # central differences of the converged E1 over the bias
    d = 2e-3
    fd = []
    for b in range(2):
        Es = []
        for s in (+1, -1):
            jb = dataclasses.replace(j, biases=np.array([j.biases[b] + s * d]))
            sb = BatchedSC(jb, k=4, device=cuda, precision="fp64", tol=1e-13, pcg_tol=1e-14)
            sb.solve(iterations=60, phi0=phi[:, b:b + 1] + s * d * sc.lifting()[:, :1])
            Es.append(float(sb.E[0, 0].item()))
        fd.append((Es[0] - Es[1]) / (2 * d))
    fd = np.array(fd)
    assert np.allclose(dE, fd, rtol=2e-3, atol=1e-6), (dE, fd)

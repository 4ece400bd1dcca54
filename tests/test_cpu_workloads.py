"""The package's seeded workload generators and the oracle's own generators
produce identical meshes and coefficients, so that the GPU path, the oracle
and the committed golden fixtures (tests/golden/sweep256.npz and the others)
all describe the same problems."""
import numpy as np
import pytest

from oracle import fem as O


@pytest.mark.parametrize("i", [0, 1, 17, 255])
def test_sweep_dot_matches_oracle_generator(i):
    from qdsim_b200 import workloads as W
    d = W.sweep_dot(i)
    om, c, V = O.dot_config_sweep(i)
    assert (d.mesh.order, d.mesh.nx, d.mesh.ny) == (om.order, om.nx, om.ny)
    assert np.array_equal(d.mesh.nodes, om.nodes)
    assert np.array_equal(d.mesh.elems, om.elems)
    assert np.array_equal(d.c, c) and np.array_equal(d.V, V)


def test_c1_dot_matches_oracle_generator():
    from qdsim_b200 import workloads as W
    d = W.c1_dot(0)
    om, c, V = O.dot_config_c1(0)
    assert np.array_equal(d.mesh.nodes, om.nodes) and np.array_equal(d.mesh.elems, om.elems)
    assert np.array_equal(d.c, c) and np.array_equal(d.V, V)


def test_sweep_sizes_follow_the_configuration():
    """nx ~ U{40..240}, ny = nx // 2, 1 nm cells, P2."""
    from qdsim_b200 import workloads as W
    for i in range(0, 256, 37):
        d = W.sweep_dot(i)
        m = d.mesh
        assert m.order == 2 and 40 <= m.nx <= 240 and m.ny == m.nx // 2
        assert (m.Lx, m.Ly) == (float(m.nx), float(m.ny))

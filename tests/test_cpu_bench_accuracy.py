"""bench.py's accuracy report on the CPU: given the oracle's own eigenpairs in
the packed layout the batched solver returns, the recomputed residuals are at
rounding level and the subspace angles vanish, for the smallest dots of the
batch (the GPU run reports the same quantities for the solver's vectors)."""
import numpy as np
import torch

import bench
from oracle import fem as O
from qdsim_b200 import batch as B
from qdsim_b200 import workloads as W


def test_accuracy_report_on_oracle_pairs():
    k = 8
    dots = W.sweep_batch(4)                     # nx 235, 56, 126, 69
    hb = B.HostBatch(dots)
    ro = hb.row_off
    E = np.ones((4, k))
    X = torch.zeros(ro[-1], k, dtype=torch.float64)
    for i in (1, 3):                            # the two smallest dots
        om, c, V = O.dot_config_sweep(i)
        a = O.assemble(om, c, V)
        E0, X0 = O.eig_lowest(a.H, a.M, k, O.sigma_below(V))
        assert X0.shape[0] == ro[i + 1] - ro[i]
        E[i] = E0
        X[ro[i]:ro[i + 1]] = torch.from_numpy(X0)
    rel = np.zeros((4, k))
    rel[0, 0] = 1.0                             # one pair not counted
    Rn = np.full(4 * k, 1e-7)
    Rn[0] = 5.0
    rep = bench.accuracy_report(hb, E, X, Rn, rel, k)
    assert rep["solver_max_over_counted"] == 1e-7
    assert rep["solver_max_all"] == 5.0
    checks = rep["vs_oracle_vectors"]
    assert [c["dot"] for c in checks] == [1, 3]
    for c in checks:
        assert c["max_residual"] < 1e-8
        assert c["max_subspace_angle_rad"] < 1e-6
        assert 1 <= c["levels_compared"] <= k

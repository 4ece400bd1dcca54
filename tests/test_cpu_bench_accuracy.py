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


def test_algorithmic_bytes_model():
    """bench.algorithmic_bytes per kernel kind for two small dots and known
    launch counts, against the per-row formulas written out here: FP32 phase
    (4-byte vectors, 8-byte (H, M) pairs, 2-byte staged column positions) and
    the mixed form's finishing phase (FP64 X and its products, FP32 W, P)."""
    dots = [W.sweep_dot(0, nx=20), W.sweep_dot(1, nx=24)]
    hb = B.HostBatch(dots)
    Bk = 12
    z = np.asarray(hb.nnz_per_dot, np.float64)
    n = np.asarray(hb.rows_per_dot, np.float64)
    counts = np.zeros((2, 6), np.int64)
    counts[:, 0] = [10, 6]     # FP32 phase: SpMM launches (two per iteration)
    counts[:, 1] = [5, 3]      #   Gram launches
    counts[:, 2] = [5, 3]      #   update launches
    counts[:, 3] = [4, 2]      # finishing phase
    counts[:, 4] = [2, 1]
    counts[:, 5] = [2, 1]
    got = bench.algorithmic_bytes(hb, counts, Bk, mixed=True)
    it32, gr32, up32 = counts[:, 0] / 2, counts[:, 1], counts[:, 2]
    it64, gr64, up64 = counts[:, 3] / 2, counts[:, 4], counts[:, 5]
    spmm = (it32 * (2 * (z * (2 + 8) + 4 * n) + 10 * n * Bk * 4)
            + it64 * (z * (4 + 16) + z * (2 + 8) + 8 * n + n * Bk * (8 + 4 + 16 + 12 + 4 + 8)))
    want = {
        "spmm": spmm.sum(),
        "gram": (gr32 * 9 * n * Bk * 4 + gr64 * n * Bk * (3 * 8 + 6 * 4)).sum(),
        "dst_precond": (gr32 * n * Bk * (2 * 4 + 12) + gr64 * n * Bk * 20).sum(),
        # W only: (MX)^T W reads MX, W; W - X C reads X, W and writes W
        "ortho": (gr32 * 5 * n * Bk * 4 + gr64 * n * Bk * (8 + 4 + 8 + 4 + 4)).sum(),
        "update": (up32 * 5 * n * Bk * 4 + up64 * n * Bk * (8 + 2 * 4 + 8 + 4)).sum(),
    }
    for kind, v in want.items():
        assert abs(got[kind] - v) <= 1e-9 * v, (kind, got[kind], v)

"""Generate tests/golden/sweep256.npz: FP64 oracle eigenvalues of the 256-dot
batched sweep (8 lowest per dot).  The inputs come from the seeded generator of
``oracle.fem.dot_config_sweep`` (identical to ``qdsim_b200.workloads.sweep_dot``,
checked by tests/test_cpu_workloads.py); the eigenvalues from the oracle's
scipy shift-invert eigsh followed by an FP64 Rayleigh-Ritz refinement.

Run: python tests/golden/make_sweep_golden.py [n_dots] [workers]
"""
import os
import sys
import time
from multiprocessing import get_context

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
os.environ.setdefault("OMP_NUM_THREADS", "1")

K = 8


def solve(i):
    from oracle import fem as O
    om, c, V = O.dot_config_sweep(i)
    a = O.assemble(om, c, V)
    E, X = O.eig_lowest(a.H, a.M, K + 2, O.sigma_below(V))
    return i, E[:K], E[K:K + 2], om.nx


def main():
    n = int(sys.argv[1]) if len(sys.argv) > 1 else 256
    workers = int(sys.argv[2]) if len(sys.argv) > 2 else os.cpu_count()
    t = time.time()
    with get_context("spawn").Pool(workers) as pool:
        out = sorted(pool.map(solve, range(n), chunksize=1))
    E = np.array([o[1] for o in out])
    Enext = np.array([o[2] for o in out])
    nx = np.array([o[3] for o in out], dtype=np.int32)
    np.savez_compressed(os.path.join(os.path.dirname(os.path.abspath(__file__)), "sweep256.npz"),
                        E=E, E_next=Enext, nx=nx, k=K, base_seed=20261203)
    print(f"{n} dots in {time.time() - t:.1f} s")


if __name__ == "__main__":
    main()

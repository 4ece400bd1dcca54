"""Generate tests/golden/c3_fd.npz: central finite differences of the FP64
oracle's eigenvalues for the differentiation workload (P3 150x75 cells on
150x75 nm, seeded Gaussian dot of ``qdsim_b200.workloads.c3_dot(0)``).

Loss L = E1+E2+E3+E4 + (E2-E1), i.e. weights (0, 2, 1, 1) on the four
lowest levels.  32 seeded directions each for the nodal potential V (eV,
step h = 1e-6) and for the per-element inverse effective mass 1/m* (units of
1/m0, step 1e-6 times its mean); every difference takes two oracle solves
(scipy shift-invert eigsh to 1e-14, then an FP64 Rayleigh-Ritz refinement),
128 solves in all.  The directions are regenerated from SEED by the test.

Stored: the five lowest levels at the base point, the 32 + 32 central
differences, the seed and the steps.  Run (a few minutes on 8 cores):
    python tests/golden/make_c3_golden.py [workers]
"""
import os
import sys
import time
from multiprocessing import get_context

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
os.environ.setdefault("OMP_NUM_THREADS", "1")

SEED = 20261204
NDIR = 32
H_V = 1e-6
H_M_REL = 1e-6
WEIGHTS = np.array([0.0, 2.0, 1.0, 1.0])


def directions(n_nodes, n_elems, seed=SEED, ndir=NDIR):
    """The seeded directions (dv [ndir, n_nodes], di [ndir, n_elems])."""
    rng = np.random.default_rng(seed)
    return rng.standard_normal((ndir, n_nodes)), rng.standard_normal((ndir, n_elems))


def _problem():
    from oracle import fem as O
    from qdsim_b200 import workloads as W
    d = W.c3_dot(0)
    om = O.structured_mesh(3, 150, 75, 150.0, 75.0)
    inv_m = d.c / O.C0_EV_NM2
    return O, om, d.V, inv_m


def _loss(args):
    V, inv_m = args
    O, om, _, _ = _problem()
    a = O.assemble(om, O.C0_EV_NM2 * inv_m, V)
    E, _ = O.eig_lowest(a.H, a.M, 5, O.sigma_below(V))
    return float(WEIGHTS @ E[:4]), E


def main(workers=8):
    O, om, V, inv_m = _problem()
    dv, di = directions(om.num_nodes, om.num_elements)
    hm = H_M_REL * float(np.mean(inv_m))
    jobs = [(V, inv_m)]
    for j in range(NDIR):
        jobs += [(V + H_V * dv[j], inv_m), (V - H_V * dv[j], inv_m)]
    for j in range(NDIR):
        jobs += [(V, inv_m + hm * di[j]), (V, inv_m - hm * di[j])]
    t0 = time.time()
    with get_context("spawn").Pool(int(workers)) as pool:
        out = pool.map(_loss, jobs, chunksize=1)
    L = np.array([o[0] for o in out])
    E0 = out[0][1]
    fd_v = (L[1:1 + 2 * NDIR:2] - L[2:2 + 2 * NDIR:2]) / (2 * H_V)
    b = 1 + 2 * NDIR
    fd_m = (L[b::2] - L[b + 1::2]) / (2 * hm)
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "c3_fd.npz")
    np.savez_compressed(path, E=E0, fd_v=fd_v, fd_m=fd_m, seed=SEED, h_v=H_V, h_m=hm,
                        weights=WEIGHTS)
    print(f"wrote {path} in {time.time() - t0:.0f} s; E = {E0}")


if __name__ == "__main__":
    main(*sys.argv[1:])

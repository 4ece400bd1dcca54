"""Generate tests/golden/c2_nearest20.npz: the oracle's 20 eigenvalues of the
open-system pencil nearest -0.05 eV at full size (P2 400 x 200 cells on
200 x 100 nm, 318,801 DOFs, CAP W = 50 meV in a 10 nm layer, seed 0).  The
inputs come from ``qdsim_b200.workloads.c2_dot``; the pencil from the FP64
oracle assembly; the eigenvalues from scipy's shift-invert eigs (complex LU),
which takes several minutes on one host, too long to repeat in every bench run.

Run: python tests/golden/make_c2_golden.py
"""
import os
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

K, SIGMA, SEED = 20, -0.05, 0


def main():
    from oracle import fem as O
    from qdsim_b200 import workloads as W
    d = W.c2_dot(SEED)
    m = d.mesh
    om = O.structured_mesh(2, m.nx, m.ny, m.Lx, m.Ly)
    a = O.assemble(om, d.c, d.V, d.W)
    t = time.time()
    w, _ = O.eig_nearest_complex(a.H - 1j * a.Wm, a.M, K, SIGMA)
    secs = time.time() - t
    out = os.path.join(os.path.dirname(os.path.abspath(__file__)), "c2_nearest20.npz")
    np.savez(out, E=w, sigma=SIGMA, seed=SEED, n=a.n, nnz=a.H.nnz, seconds=secs)
    print(f"wrote {out}: n={a.n} nnz={a.H.nnz} eigs {secs:.1f} s")


if __name__ == "__main__":
    main()

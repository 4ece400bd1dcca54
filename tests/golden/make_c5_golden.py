"""Generate tests/golden/c5_sc.npz: the FP64 restatement of the batched
self-consistent p-n junction (``oracle.sc.run``) at the configuration's size
(P1 300x100 cells on 300x100 nm, 10 states, 40 iterations: damping, then
Anderson with the line search) for two of the 64 seeded bias points of
``qdsim_b200.workloads.c5_junction(64)``: the lowest and the highest.

Stored per bias point: the error of every iteration, the ten levels of the
last map, the final potential at every 7th node, and the 2-norm of the potential
after iterations 5, 20 and 40.  Each bias point runs in its own process (the
oracle's map is independent per bias point).  Run (~10-20 min):
    python tests/golden/make_c5_golden.py
"""
import dataclasses
import os
import sys
import time
from multiprocessing import get_context

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
os.environ.setdefault("OMP_NUM_THREADS", "1")

BIAS_IDX = (0, 63)
ITERATIONS = 40
K = 10
NORM_AT = (5, 20, 40)
STRIDE = 7          # the final potential is stored at every 7th node


def _run(b):
    from oracle import fem as O, sc as OS
    from qdsim_b200 import workloads as W
    j = W.c5_junction(64)
    jo = dataclasses.replace(j, biases=j.biases[[b]],
                             mesh=O.structured_mesh(1, 300, 100, 300.0, 100.0))
    norms = []

    def record(it, phi, E):
        if it + 1 in NORM_AT:
            norms.append(float(np.linalg.norm(phi[:, 0])))

    phi, err, E = OS.run(jo, k=K, iterations=ITERATIONS, on_iter=record)
    return b, err[:, 0], E[0], phi[:, 0], np.array(norms)


def main():
    t0 = time.time()
    with get_context("spawn").Pool(len(BIAS_IDX)) as pool:
        out = pool.map(_run, BIAS_IDX)
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "c5_sc.npz")
    np.savez_compressed(path, bias_idx=np.array(BIAS_IDX), errors=np.stack([o[1] for o in out], 1),
                        E=np.stack([o[2] for o in out]),
                        phi=np.stack([o[3][::STRIDE] for o in out], 1), stride=STRIDE,
                        norms=np.stack([o[4] for o in out], 1), norm_at=np.array(NORM_AT))
    print(f"wrote {path} in {time.time() - t0:.0f} s")


if __name__ == "__main__":
    main()

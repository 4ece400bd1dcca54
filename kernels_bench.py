"""Run one kernel family on a named workload and report its CUDA-event time.

    python kernels_bench.py cap_spmm [--prec fp64|fp32] [--b 48] [--launches 10]
    python kernels_bench.py pcg [--iters 32]
    python kernels_bench.py interp [--points 16777216] [--gradient] [--sorted]
    python kernels_bench.py adjoint [--launches 10]
    python kernels_bench.py sc [--iters 6]
    python kernels_bench.py cap_solve [--prec fp64|mixed] [--cells 400]

``cap_spmm``: ``qd_cap_spmm`` on the open-system pencil of P2 400x200 cells on
200x100 nm (318,801 DOFs, 3.65M nonzeros) for a block of b complex columns;
prints ms per launch and GB/s of algorithmic bytes.  ``pcg``: the Jacobi-PCG
of the p-n junction's Poisson step (P1 300x100 cells, 30,401 nodes, 64
right-hand sides) for a fixed number of iterations; prints ms per iteration.
``interp``: ``qd_fe_interpolate`` of one nodal field of the P2 400x200-cell
mesh on 200x100 nm at uniformly random points (values, optionally gradients
and elements), in random order or sorted by cell (``--sorted``, the order of
a resampling onto another mesh's nodes); prints ms per launch and GB/s of
algorithmic bytes (16 B of coordinates in, 8 B per value out, 20 B more with
gradients and elements, the field read once).
``adjoint``: ``qd_adjoint`` (element pass and node gather) on the P3 150x75-cell
dot with the four lowest eigenvectors from the GPU solve; prints ms per call.
``sc``: the batched self-consistent loop of the p-n junction (P1 300x100
cells, 64 bias points, 10 states) for a few iterations; prints ms per
iteration (densities, mixing, the batched eigensolve and PCG inside).
``cap_solve``: one open-system solve (``qd_cap_lobpcg_solve``: the 20
eigenvalues nearest -0.05 eV from the lowest 40, block 48) on P2 cells x
cells/2 on 200x100 nm, after a 3-iteration warm-up solve; prints seconds,
iterations and the largest Schur sweep count.
The launch sequence is fixed, so a profiler can select launches by index.
"""
from __future__ import annotations

import argparse
import json
import os
import sys

import numpy as np
import torch

sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))


def cap_spmm(prec: str, b: int, launches: int, dev):
    from qdsim_b200.cap import CAPProblem
    from qdsim_b200.workloads import c2_dot
    d = c2_dot(0)
    prob = CAPProblem(d.mesh, d.c, d.V, d.W, device=dev)
    ct, s = (torch.complex64, 4) if prec == "fp32" else (torch.complex128, 8)
    g = torch.Generator(device="cpu").manual_seed(0)
    X = torch.view_as_complex(torch.randn(prob.n, b, 2, generator=g)).to(dev, ct)
    AX, MX = torch.empty_like(X), torch.empty_like(X)
    prob.spmm(X, AX, MX)                        # launch 0 (warm-up)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(launches):
        prob.spmm(X, AX, MX)
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / launches
    nnz = prob.fem.nnz
    alg = nnz * (4 + 3 * s) + 4 * (prob.n + 1) + 3 * prob.n * b * 2 * s
    return {"kernel": "cap_spmm_kernel", "prec": prec, "b": b, "rows": prob.n, "nnz": int(nnz),
            "ms_per_launch": ms, "algorithmic_bytes": int(alg), "GBps": alg / (ms * 1e-3) / 1e9}


def pcg(iters: int, dev):
    from qdsim_b200 import _native as N
    from qdsim_b200.poisson import PoissonProblem
    from qdsim_b200.workloads import c5_junction
    j = c5_junction(64)
    prob = PoissonProblem(j.mesh, j.eps_r, device=dev)
    rng = np.random.default_rng(0)
    rho = 1.6e5 * rng.standard_normal((j.mesh.num_nodes, 64))
    out = {}
    for tag, it in (("warm-up", 2), ("timed", iters)):
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        try:
            prob.solve(rho, 0.0, np.asarray(j.biases), tol=1e-300, max_iter=it)
        except N.QDError as e:
            if e.status != N.QD_ERR_NOT_CONVERGED:
                raise
        e1.record()
        torch.cuda.synchronize()
        out[tag] = e0.elapsed_time(e1)
    n, nnz = j.mesh.num_nodes, prob.fem.nnz
    alg = nnz * 12 + 4 * (n + 1) + 11 * n * 8 * 64
    ms = out["timed"] / iters
    return {"kernels": ["pcg_spmv_kernel", "pcg_axpy_kernel"], "nodes": n, "nnz": int(nnz),
            "nrhs": 64, "iterations": iters, "ms_per_iteration": ms,
            "algorithmic_bytes_per_iteration": int(alg), "GBps": alg / (ms * 1e-3) / 1e9}


def interp(points: int, gradient: bool, ordered: bool, launches: int, dev):
    from qdsim_b200.interp import FieldInterpolator
    from qdsim_b200.mesh import StructuredMesh
    m = StructuredMesh(2, 400, 200, 200.0, 100.0)
    g = torch.Generator(device=dev).manual_seed(0)
    x = torch.rand(points, generator=g, device=dev, dtype=torch.float64) * m.Lx
    y = torch.rand(points, generator=g, device=dev, dtype=torch.float64) * m.Ly
    f = torch.randn(m.num_nodes, generator=g, device=dev, dtype=torch.float64)
    if ordered:
        key = (y * (m.ny / m.Ly)).long().clamp(max=m.ny - 1) * m.nx + \
            (x * (m.nx / m.Lx)).long().clamp(max=m.nx - 1)
        order = torch.argsort(key)
        x, y = x[order].contiguous(), y[order].contiguous()
        del key, order
    fi = FieldInterpolator(m, device=dev)
    fi.evaluate(x, y, f, gradient=gradient, element=gradient)   # launch 0 (warm-up)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(launches):
        fi.evaluate(x, y, f, gradient=gradient, element=gradient)
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / launches
    alg = points * (16 + 8 + (20 if gradient else 0)) + m.num_nodes * 8
    return {"kernel": "interp_kernel", "order": 2, "nodes": int(m.num_nodes), "points": points,
            "gradient": gradient, "sorted": ordered, "ms_per_launch": ms, "algorithmic_bytes": int(alg),
            "GBps": alg / (ms * 1e-3) / 1e9, "Gpoints_per_s": points / (ms * 1e-3) / 1e9}


def adjoint(launches: int, dev):
    from qdsim_b200 import adjoint as AD, batch as Bt, fem as F, workloads as W
    d = W.c3_dot(0)
    hb = Bt.HostBatch([d])
    db = Bt.DeviceBatch(hb, dev)
    db.upload(non_blocking=False)
    db.assemble()
    X = db.solve(4, b=8, precision="fp64", tol=1e-12, max_iter=400)[1]
    prob = F.FEMProblem(d.mesh, device=dev)
    w = np.array([0.0, 2.0, 1.0, 1.0])
    AD.energy_gradients(prob, X, w)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(launches):
        AD.energy_gradients(prob, X, w)
    e1.record()
    torch.cuda.synchronize()
    return {"kernel": "adjoint_elem_kernel + adjoint_node_kernel", "nodes": int(d.mesh.num_nodes),
            "elements": int(d.mesh.num_elements), "ms_per_call": e0.elapsed_time(e1) / launches}


def sc(iters: int, dev):
    from qdsim_b200 import workloads as W
    from qdsim_b200.sc import BatchedSC
    s = BatchedSC(W.c5_junction(64), k=10, device=dev)
    s.solve(iterations=2)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    s.solve(iterations=iters)
    e1.record()
    torch.cuda.synchronize()
    return {"case": "p-n junction, 64 bias points", "ms_per_iteration": e0.elapsed_time(e1) / iters}


def cap_solve(prec: str, cells: int, dev):
    import time
    from qdsim_b200.cap import CAPSolver
    from qdsim_b200.workloads import c2_dot
    d = c2_dot(0, nx=cells, ny=cells // 2)
    solver = CAPSolver(d.mesh, d.c, d.V, d.W, device=dev)
    solver.solve(k=20, sigma=-0.05, nev=40, b=48, precision=prec, max_iter=3)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    res = solver.solve(k=20, sigma=-0.05, nev=40, b=48, precision=prec, tol=1e-9)
    torch.cuda.synchronize()
    return {"case": f"open system, P2 {cells}x{cells // 2} cells", "prec": prec,
            "seconds": time.perf_counter() - t0, "iterations": res.info["iterations"],
            "schur_sweeps_max": res.info["schur_sweeps_max"], "complete": res.info["complete"]}


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("case", choices=["cap_spmm", "pcg", "interp", "adjoint", "sc", "cap_solve"])
    ap.add_argument("--prec", default="fp64", choices=["fp64", "fp32", "mixed"])
    ap.add_argument("--cells", type=int, default=400)
    ap.add_argument("--b", type=int, default=48)
    ap.add_argument("--launches", type=int, default=10)
    ap.add_argument("--iters", type=int, default=32)
    ap.add_argument("--points", type=int, default=1 << 24)
    ap.add_argument("--gradient", action="store_true")
    ap.add_argument("--sorted", action="store_true")
    a = ap.parse_args(argv)
    if not torch.cuda.is_available():
        raise SystemExit("a CUDA device is required")
    dev = torch.device("cuda:0")
    if a.case == "cap_spmm":
        r = cap_spmm(a.prec, a.b, a.launches, dev)
    elif a.case == "pcg":
        r = pcg(a.iters, dev)
    elif a.case == "adjoint":
        r = adjoint(a.launches, dev)
    elif a.case == "sc":
        r = sc(a.iters, dev)
    elif a.case == "cap_solve":
        r = cap_solve("mixed" if a.prec == "mixed" else "fp64", a.cells, dev)
    else:
        r = interp(a.points, a.gradient, a.sorted, a.launches, dev)
    print(json.dumps(r))


if __name__ == "__main__":
    main()

"""Batched LOBPCG vs the FP64 oracle (scipy shift-invert + FP64 Rayleigh-Ritz)."""
import numpy as np
import pytest

from oracle import fem as O

pytestmark = pytest.mark.gpu


def _solve_single(cuda, om, c, V, k, precision, b=None, tol=1e-9):
    from qdsim_b200 import fem as F, eigen as G, mesh as Mh
    m = Mh.StructuredMesh(om.order, om.nx, om.ny, om.Lx, om.Ly)
    prob = F.FEMProblem(m, device=cuda)
    a = prob.assemble(c, V)
    res = G.solve_batch([(prob.d_rowptr, prob.d_col, a["H"], a["M"])], k, b=b,
                        precision=precision, tol=tol, max_iter=3000)
    return prob, res


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_c1_lowest10(cuda, precision):
    om, c, V = O.dot_config_c1(seed=0)
    ref = O.assemble(om, c, V)
    E0, X0 = O.eig_lowest(ref.H, ref.M, 10, O.sigma_below(V))
    prob, res = _solve_single(cuda, om, c, V, 10, precision, b=16)
    assert res.status == 0, res.info
    E = res.E[0]
    rel = np.abs(E - E0) / np.abs(E0)
    assert rel.max() <= 1e-9, (rel, res.info)
    X = res.X[0].cpu().numpy()
    # M-orthonormal and small FP64 residuals recomputed from scratch
    G = X.T @ (ref.M @ X)
    assert np.abs(G - np.eye(10)).max() < 1e-8
    r = O.residuals(ref.H, ref.M, E, X)
    assert r.max() < 1e-4
    ang = O.subspace_angles(X[:, :3], X0[:, :3], ref.M)
    assert ang.max() < 1e-5


def test_batch_matches_single(cuda):
    from qdsim_b200 import fem as F, eigen as G, mesh as Mh
    dots = [O.dot_config_sweep(seed, nx=nx) for seed, nx in ((1, 20), (2, 28), (3, 24))]
    mats, probs, refs = [], [], []
    for om, c, V in dots:
        m = Mh.StructuredMesh(2, om.nx, om.ny, om.Lx, om.Ly)
        p = F.FEMProblem(m, device=cuda)
        a = p.assemble(c, V)
        mats.append((p.d_rowptr, p.d_col, a["H"], a["M"]))
        probs.append(p)
        ra = O.assemble(om, c, V)
        refs.append(O.eig_lowest(ra.H, ra.M, 8, O.sigma_below(V))[0])
    res = G.solve_batch(mats, 8, b=12, precision="mixed", tol=1e-9, max_iter=3000)
    assert res.status == 0, res.info
    for i in range(3):
        rel = np.abs(res.E[i] - refs[i]) / np.abs(refs[i])
        assert rel.max() <= 1e-9, (i, rel)
    # solving one dot alone gives the same eigenvalues as inside the batch
    single = G.solve_batch(mats[1:2], 8, b=12, precision="mixed", tol=1e-9, max_iter=3000)
    assert np.allclose(single.E[0], res.E[1], rtol=1e-10, atol=0)


def test_spmm_dual_matches_scipy(cuda):
    import torch
    from qdsim_b200 import fem as F, mesh as Mh, _native as N
    om, c, V = O.dot_config_sweep(5, nx=30)
    m = Mh.StructuredMesh(2, om.nx, om.ny, om.Lx, om.Ly)
    p = F.FEMProblem(m, device=cuda)
    a = p.assemble(c, V)
    H, M = p.to_scipy(a["H"]), p.to_scipy(a["M"])
    rng = np.random.default_rng(0)
    for b in (4, 8, 12, 16):
        for fp32 in (0, 1):
            X = rng.standard_normal((p.n, b))
            dt = torch.float32 if fp32 else torch.float64
            Xd = torch.from_numpy(X).to(cuda, dt).contiguous()
            HX = torch.empty_like(Xd)
            MX = torch.empty_like(Xd)
            N.check(N.lib().qd_spmm_dual(p.n, b, fp32, N.ptr(p.d_rowptr), N.ptr(p.d_col),
                                         N.ptr(a["H"]), N.ptr(a["M"]), N.ptr(Xd), N.ptr(HX),
                                         N.ptr(MX), F.stream_ptr()), "spmm")
            Xr = Xd.double().cpu().numpy()
            tol = 1e-6 if fp32 else 1e-13
            for got, A in ((HX, H), (MX, M)):
                ref = A @ Xr
                err = np.abs(got.double().cpu().numpy() - ref).max() / np.abs(ref).max()
                assert err < tol, (b, fp32, err)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_preconditioned_sweep_dots(cuda, precision):
    """Batched solve of sweep dots through the product path (DST-preconditioned)."""
    from qdsim_b200 import batch as Bt, workloads as W
    ids = [0, 1, 2, 3, 17]
    dots = [W.sweep_dot(i, nx=nx) for i, nx in zip(ids, (40, 64, 52, 90, 41))]
    res = Bt.solve_dots(dots, 8, device=cuda, b=12, precision=precision, tol=1e-9,
                        max_iter=1000)
    assert res.status == 0, res.info
    assert res.info["iterations"] < 200, res.info      # preconditioning works
    for j, (i, nx) in enumerate(zip(ids, (40, 64, 52, 90, 41))):
        om, c, V = O.dot_config_sweep(i, nx=nx)
        a = O.assemble(om, c, V)
        E0 = O.eig_lowest(a.H, a.M, 8, O.sigma_below(V))[0]
        rel = np.abs(res.E[j] - E0) / np.abs(E0)
        assert rel.max() <= 1e-9, (j, rel, res.info)


def test_sweep_pipeline_steps_match_batch(cuda):
    """SweepPipeline (two alternating device batches, copies on a side stream):
    every step's host E and X equal a plain batched solve of the same dots."""
    import torch
    from qdsim_b200 import batch as Bt, workloads as W
    dots = [W.sweep_dot(i, nx=nx) for i, nx in ((0, 24), (1, 32), (2, 28))]
    hb = Bt.HostBatch(dots)
    kw = dict(b=12, precision="mixed", tol=1e-9, max_iter=3000)
    ref = Bt.DeviceBatch(hb, cuda)
    ref.upload(non_blocking=False)
    ref.assemble()
    E_ref, X_ref = (t.cpu().numpy() for t in ref.solve(8, **kw)[:2])
    pinned = hb.pin()
    steps = 3
    outE = [torch.zeros((3, 8), dtype=torch.float64).pin_memory() for _ in range(steps)]
    outX = [torch.zeros((hb.n, 8), dtype=torch.float64).pin_memory() for _ in range(steps)]
    pipe = Bt.SweepPipeline(hb, cuda)
    pipe.run(steps, 8, lambda s: pinned, lambda s: outE[s], lambda s: outX[s], **kw)
    torch.cuda.synchronize()
    for s in range(steps):
        assert np.array_equal(outE[s].numpy(), E_ref), s
        assert np.array_equal(outX[s].numpy(), X_ref), s


def test_p3_mixed_staged_and_gathered_subtiles(cuda):
    """P3 dot (30 x 15 cells, 3,916 DOFs) in mixed precision.  Its stencil spans
    seven lattice lines, so about half of the FP32 SpMM's sub-tiles (64 rows for
    X and P, 128 rows for W) exceed the staged runs and read their operands
    from global memory while the others are staged in shared memory; the
    eigenvalues of both paths together against the oracle."""
    om, c, V = O.dot_config_sweep(3, order=3, nx=30)
    ref = O.assemble(om, c, V)
    E0 = O.eig_lowest(ref.H, ref.M, 8, O.sigma_below(V))[0]
    prob, res = _solve_single(cuda, om, c, V, 8, "mixed", b=12)
    assert res.status == 0, res.info
    rel = np.abs(res.E[0] - E0) / np.abs(E0)
    assert rel.max() <= 1e-9, (rel, res.info)

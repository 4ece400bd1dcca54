"""Failure detection on the GPU: every failure comes back as a status code
from the C-ABI, with the results the call could still produce, never as
dummy eigenpairs (the reference's RecoveryManager returns zeros,
backend/src/solver.cpp:183-192) and never as a trap, a fault or a hang.

The failures are made on the host: an iteration cap that is too small,
matrix values that the caller poisons with NaN or flips to an indefinite
pencil, a degenerate element, and a device-side wait on a barrier that
nothing completes (the library's own bounded wait, run by a diagnostic
entry point, so that it expires after a short limit)."""
import ctypes as C

import numpy as np
import pytest


pytestmark = pytest.mark.gpu


def _dot_batch(cuda, nx=24):
    from qdsim_b200 import batch as Bt, workloads as W
    hb = Bt.HostBatch([W.sweep_dot(3, nx=nx)])
    db = Bt.DeviceBatch(hb, cuda)
    db.upload(non_blocking=False)
    db.assemble()
    db.check_status()
    return hb, db


@pytest.mark.parametrize("precision", ["mixed", "fp64"])
def test_iteration_cap_reports_not_converged_with_residuals(cuda, precision):
    from qdsim_b200 import _native as N
    hb, db = _dot_batch(cuda)
    E, X, R, it, info, st = db.solve(8, b=12, precision=precision, tol=1e-9, max_iter=3)
    assert st == N.QD_ERR_NOT_CONVERGED
    R = R.cpu().numpy()
    E = E.cpu().numpy()
    assert np.isfinite(E).all() and np.isfinite(R).all()
    assert (R > 0).all() and R.max() > 1e-6        # the residuals of where it stopped
    # the cap counts every iteration; the mixed form's FP64 phase always runs
    # one iteration after the hand-over before it tests the residuals again
    assert int(it.cpu().numpy()[0]) == (4 if precision == "mixed" else 3)
    assert info["converged_dots"] == 0
    # the same call with not-converged treated as an error raises
    with pytest.raises(N.QDError) as exc:
        db.solve(8, b=12, precision=precision, tol=1e-9, max_iter=3, allow_not_converged=False)
    assert exc.value.status == N.QD_ERR_NOT_CONVERGED


def test_nan_mass_matrix_is_a_breakdown(cuda):
    import torch
    from qdsim_b200 import _native as N
    hb, db = _dot_batch(cuda)
    db.M[::7] = float("nan")
    with pytest.raises(N.QDError) as exc:
        db.solve(8, b=12, precision="fp64", tol=1e-9, max_iter=50)
    assert exc.value.status == N.QD_ERR_BREAKDOWN
    torch.cuda.synchronize()          # the context is still usable


@pytest.mark.parametrize("precision", ["mixed", "fp64"])
def test_indefinite_pencil_is_a_breakdown(cuda, precision):
    from qdsim_b200 import _native as N
    hb, db = _dot_batch(cuda)
    db.M.neg_()                        # negative definite "mass matrix"
    with pytest.raises(N.QDError) as exc:
        db.solve(8, b=12, precision=precision, tol=1e-9, max_iter=50)
    assert exc.value.status == N.QD_ERR_BREAKDOWN
    # a healthy solve on the same device afterwards
    db.assemble()
    E, X, R, it, info, st = db.solve(8, b=12, precision=precision, tol=1e-9, max_iter=500)
    assert st == N.QD_OK


def test_drop_in_solver_raises_on_non_finite_potential(cuda):
    """A NaN potential is flagged by the assembly kernel (QD_ERR_DEGENERATE);
    the drop-in solver raises instead of printing and returning empty arrays,
    unless swallow_errors restores the reference's behaviour."""
    from qdsim_b200 import _native as N
    from qdsim_b200.mesh import SimpleMesh
    from qdsim_b200.solvers import CythonSchrodingerSolver
    m = SimpleMesh(21, 11, 40e-9, 20e-9)

    def mstar(x, y):
        return 0.067 * 9.1093837015e-31

    def bad_v(x, y):
        return np.where(x > 20e-9, np.nan, 0.0)

    with pytest.raises(N.QDError) as exc:
        CythonSchrodingerSolver(m, mstar, bad_v).solve(4)
    assert exc.value.status == N.QD_ERR_DEGENERATE
    E, psi = CythonSchrodingerSolver(m, mstar, bad_v, swallow_errors=True).solve(4)
    assert E.size == 0 and psi == []


def test_pcg_iteration_cap_reports_not_converged(cuda):
    import torch
    from qdsim_b200 import _native as N, mesh as Mh, poisson as P
    m = Mh.StructuredMesh(1, 30, 10, 150.0, 50.0)
    prob = P.PoissonProblem(m, np.full(m.num_elements, 12.9), device=cuda)
    rho = 1.6e5 * np.sign(m.nodes[:, 0] - 75.0)
    with pytest.raises(N.QDError) as exc:
        prob.solve(rho, 0.0, 0.4, max_iter=2)
    assert exc.value.status == N.QD_ERR_NOT_CONVERGED
    phi = prob.solve(rho, 0.0, 0.4)            # the default cap converges
    assert torch.isfinite(phi).all()


@pytest.mark.parametrize("with_copy", [0, 1])
def test_bounded_wait_expires_with_a_status(cuda, with_copy):
    """The bounded mbarrier wait, on a barrier nothing completes, gives up
    after its limit (20 ms here), the kernel drains its own bulk copy and
    returns, and the host reads QD_ERR_TIMEOUT; the context stays usable."""
    import time
    import torch
    from qdsim_b200 import _native as N
    src = torch.arange(64, dtype=torch.int32, device=cuda)
    d_status = torch.zeros(1, dtype=torch.int32, device=cuda)
    h_status = C.c_int32(0)
    t0 = time.perf_counter()
    st = N.lib().qd_bounded_wait_selftest(20_000_000, N.ptr(src), with_copy, N.ptr(d_status),
                                          C.byref(h_status), None)
    dt = time.perf_counter() - t0
    assert st == N.QD_ERR_TIMEOUT
    assert h_status.value == 1                 # expired; the copy drained intact
    assert 0.015 <= dt <= 5.0
    assert int(src.sum().item()) == 64 * 63 // 2

"""Open-system (CAP) eigensolve on the GPU: qd_cap_spmm against scipy on the
device-assembled pencil, and the k eigenvalues nearest sigma against the
oracle's shift-invert eigs (both precision forms)."""
import numpy as np
import pytest

from oracle import fem as O

pytestmark = pytest.mark.gpu


def _c2(nx, ny):
    from qdsim_b200 import workloads as W
    d = W.c2_dot(0, nx=nx, ny=ny)
    return d


@pytest.mark.parametrize("fp32", [0, 1])
def test_cap_spmm_matches_scipy(cuda, fp32):
    import torch
    from qdsim_b200 import cap as CP
    d = _c2(30, 15)
    prob = CP.CAPProblem(d.mesh, d.c, d.V, d.W, device=cuda)
    A = prob.fem.to_scipy(prob.H) + 1j * prob.fem.to_scipy(prob.G)
    M = prob.fem.to_scipy(prob.M)
    n = prob.n
    ct = torch.complex64 if fp32 else torch.complex128
    rng = np.random.default_rng(3)
    for b, lo_x, ld_x, lo_y, ld_y in [(40, 3, 64, 5, 72), (33, 0, 33, 0, 33), (7, 1, 9, 2, 11)]:
        xb = rng.standard_normal((n, ld_x)) + 1j * rng.standard_normal((n, ld_x))
        Xbuf = torch.from_numpy(xb).to(cuda, ct)
        AXbuf = torch.zeros(n, ld_y, dtype=ct, device=cuda)
        MXbuf = torch.zeros(n, ld_y, dtype=ct, device=cuda)
        prob.spmm(Xbuf[:, lo_x:lo_x + b], AXbuf[:, lo_y:lo_y + b], MXbuf[:, lo_y:lo_y + b])
        x = Xbuf[:, lo_x:lo_x + b].cpu().numpy().astype(np.complex128)
        ax, mx = A @ x, M @ x
        got_a = AXbuf.cpu().numpy()
        got_m = MXbuf.cpu().numpy()
        tol = 2e-6 if fp32 else 1e-13
        assert np.linalg.norm(got_a[:, lo_y:lo_y + b] - ax) / np.linalg.norm(ax) < tol
        assert np.linalg.norm(got_m[:, lo_y:lo_y + b] - mx) / np.linalg.norm(mx) < tol
        # columns outside the slice are untouched
        assert not np.any(got_a[:, :lo_y]) and not np.any(got_a[:, lo_y + b:])


def test_cap_spmm_without_cap_is_hermitian_product(cuda):
    import ctypes as C
    import torch
    from qdsim_b200 import _native as N, cap as CP
    from qdsim_b200.fem import stream_ptr
    d = _c2(20, 10)
    prob = CP.CAPProblem(d.mesh, d.c, d.V, d.W, device=cuda)
    H = prob.fem.to_scipy(prob.H)
    X = torch.randn(prob.n, 5, dtype=torch.complex128, device=cuda)
    AX, MX = torch.empty_like(X), torch.empty_like(X)
    N.check(N.lib().qd_cap_spmm(prob.n, 5, 0, N.ptr(prob.fem.d_rowptr), N.ptr(prob.fem.d_col),
                                N.ptr(prob.H), None, N.ptr(prob.M), N.ptr(X), 5, N.ptr(AX),
                                N.ptr(MX), 5, stream_ptr()), "cap spmm")
    ref = H @ X.cpu().numpy()
    assert np.linalg.norm(AX.cpu().numpy() - ref) / np.linalg.norm(ref) < 1e-13
    assert N.lib().qd_cap_spmm(prob.n, 65, 0, N.ptr(prob.fem.d_rowptr), N.ptr(prob.fem.d_col),
                               N.ptr(prob.H), None, N.ptr(prob.M), N.ptr(X), 65, N.ptr(AX),
                               N.ptr(MX), 65, stream_ptr()) == N.QD_ERR_INVALID


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_cap_nearest20_matches_oracle(cuda, precision):
    """P2 100 x 50 cells on 200 x 100 nm (19,701 DOFs): the 20 eigenvalues
    nearest -0.05 eV are levels ~20-39 by real part."""
    from qdsim_b200 import cap as CP
    d = _c2(100, 50)
    om = O.structured_mesh(2, 100, 50, 200.0, 100.0)
    a = O.assemble(om, d.c, d.V, d.W)
    Ac = a.H - 1j * a.Wm
    w, _ = O.eig_nearest_complex(Ac, a.M, 20, -0.05)
    solver = CP.CAPSolver(d.mesh, d.c, d.V, d.W, device=cuda)
    res = solver.solve(k=20, sigma=-0.05, nev=40, b=48, precision=precision, tol=1e-9)
    assert res.info["complete"], res.info
    ws, Es = np.sort_complex(w), np.sort_complex(res.E)
    err = np.abs(Es - ws) / np.abs(ws)
    assert err.max() <= 1e-9, (err.max(), res.info)
    X = res.X.cpu().numpy()
    assert np.abs(np.einsum("ij,ij->j", X, a.M @ X) - 1.0).max() < 1e-9
    r = np.linalg.norm(Ac @ X - (a.M @ X) * res.E, axis=0) / (
        np.abs(res.E) * np.linalg.norm(a.M @ X, axis=0))
    assert r.max() < 1e-8, r.max()


@pytest.mark.parametrize("w_scale", [0.0, 1e-5])
def test_cap_solver_tends_to_hermitian_levels(cuda, w_scale):
    """As W -> 0 the open-system eigenvalues tend to the Hermitian ones: at
    W = 0 they coincide (imaginary parts zero); for a CAP scaled by 1e-5 the
    real parts move by second order only and -Im E stays below the largest W."""
    from qdsim_b200 import cap as CP
    d = _c2(100, 50)
    om = O.structured_mesh(2, 100, 50, 200.0, 100.0)
    a = O.assemble(om, d.c, d.V)
    Eh, _ = O.eig_lowest(a.H, a.M, 40, O.sigma_below(d.V))
    W = d.W * w_scale
    res = CP.CAPSolver(d.mesh, d.c, d.V, W, device=cuda).solve(
        k=20, sigma=-0.05, nev=40, b=48, precision="fp64", tol=1e-9)
    assert res.info["complete"], res.info
    near = np.sort(Eh[np.argsort(np.abs(Eh + 0.05), kind="stable")[:20]])
    got = np.sort(res.E.real)
    if w_scale == 0.0:
        assert np.abs(res.E.imag).max() <= 1e-12 * np.abs(res.E).max()
        assert (np.abs(got - near) / np.abs(near)).max() <= 1e-9
    else:
        assert (-res.E.imag).max() <= W.max() and (-res.E.imag).min() >= -1e-3 * W.max()
        assert (np.abs(got - near) / np.abs(near)).max() <= 1e-6


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_cap_nearest20_at_config_size(cuda, precision):
    """The open-system configuration at its stated size (P2 400x200 cells on
    200x100 nm, 318,801 DOFs, CAP -i 50 meV (d/10 nm)^2 in a 10 nm layer):
    the 20 eigenvalues nearest -0.05 eV against the oracle's shift-invert
    eigs on the same pencil (tests/golden/c2_nearest20.npz, made by
    tests/golden/make_c2_golden.py), 1e-9 relative, certified complete, with
    x^T M x = 1 and small residuals."""
    import os
    from qdsim_b200 import cap as CP
    gold = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden",
                                "c2_nearest20.npz"))["E"]
    d = _c2(400, 200)
    res = CP.CAPSolver(d.mesh, d.c, d.V, d.W, device=cuda).solve(
        k=20, sigma=-0.05, nev=40, b=48, precision=precision, tol=1e-9)
    assert res.info["complete"], res.info
    err = np.array([np.min(np.abs(res.E - g)) / abs(g) for g in gold])
    assert err.max() <= 1e-9, (err.max(), res.info)
    assert len({int(np.argmin(np.abs(res.E - g))) for g in gold}) == 20
    assert res.residual.max() < 1e-8, res.residual.max()


@pytest.mark.parametrize("n", [7, 48, 143, 144])
def test_complex_schur_kernel_matches_restatement(cuda, n):
    """qd_complex_schur (8-CTA cluster, matrix rows in distributed shared
    memory) against its restatement and LAPACK on a Hermitian matrix with a
    non-Hermitian perturbation: unitary Z, upper triangular T, C = Z T Z^H,
    the eigenvalues, and the sweep count of the same rotation sequence."""
    import ctypes as C
    import torch
    from qdsim_b200 import _native as N
    from qdsim_b200.fem import stream_ptr
    from oracle.cap_lobpcg import schur_jacobi
    rng = np.random.default_rng(n)
    A = rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))
    B = rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))
    Cm = 0.5 * (A + A.conj().T) + np.diag(np.linspace(0, 5, n)) + 0.02 * B
    ld = n + 3
    Cd = torch.zeros(n, ld, dtype=torch.complex128, device=cuda)
    Cd[:, :n] = torch.from_numpy(Cm)
    Td = torch.zeros(n, ld, dtype=torch.complex128, device=cuda)
    Zd = torch.zeros_like(Td)
    sw = C.c_int()
    N.check(N.lib().qd_complex_schur(n, N.ptr(Cd), ld, N.ptr(Td), N.ptr(Zd), ld, 60, C.byref(sw),
                                     stream_ptr()), "qd_complex_schur")
    T, Z = Td[:, :n].cpu().numpy(), Zd[:, :n].cpu().numpy()
    nc = np.linalg.norm(Cm)
    assert np.abs(Z.conj().T @ Z - np.eye(n)).max() < 1e-12
    assert np.abs(np.tril(T, -1)).max() <= 1e-13 * nc
    assert np.linalg.norm(Z @ T @ Z.conj().T - Cm) <= 1e-12 * nc
    w = np.linalg.eigvals(Cm)
    assert max(np.min(np.abs(w - x)) for x in np.diag(T)) <= 1e-10 * np.abs(w).max()
    _, _, sw_ref, conv = schur_jacobi(Cm)
    assert conv and abs(sw.value - sw_ref) <= 1, (sw.value, sw_ref)


def test_cap_solver_rejects_bad_blocks(cuda):
    from qdsim_b200 import _native as N, cap as CP
    d = _c2(20, 10)
    solver = CP.CAPSolver(d.mesh, d.c, d.V, d.W, device=cuda)
    for b in (7, 50):
        with pytest.raises(N.QDError) as e:
            solver.solve(k=4, sigma=-0.05, nev=6, b=b)
        assert e.value.status == N.QD_ERR_INVALID

"""The CAP (complex absorbing potential) eigensolve's algorithm on the CPU:
the restatement of the GPU's block LOBPCG (oracle/cap_lobpcg.py) driven by
scipy products and the FP64 DST, against the oracle's shift-invert eigs on
the same pencil, and the restatement of the GPU's Schur kernel (parallel
round-robin Jacobi-like method) against LAPACK."""
import numpy as np
import torch

from oracle import fem as O
from dst_emul import apply_exact


class _HostPencil:
    """spmm / precondition on the host (scipy CSR, exact DST)."""

    def __init__(self, A, M, spec):
        self.A, self.M, self.spec = A.tocsr(), M.tocsr(), spec
        self.n = A.shape[0]
        self.device = torch.device("cpu")

    def spmm(self, X, AX, MX):
        x = X.numpy()
        AX.copy_(torch.from_numpy(self.A @ x))
        MX.copy_(torch.from_numpy(self.M @ x))

    def precondition(self, R):
        r = R.numpy()
        nx, ny, cx, cy, sh = self.spec
        out = apply_exact(r.real, nx, ny, cx, cy, sh) + 1j * apply_exact(r.imag, nx, ny, cx, cy, sh)
        return torch.from_numpy(out).to(R.dtype)


def _pencil(nx=24, ny=12):
    from qdsim_b200 import workloads as W
    from qdsim_b200.eigen import DSTPreconditioner
    from qdsim_b200.mesh import StructuredMesh
    d = W.c2_dot(0, nx=nx, ny=ny)
    om = O.structured_mesh(2, nx, ny, 200.0, 100.0)
    a = O.assemble(om, d.c, d.V, d.W)
    spec = DSTPreconditioner.spec_for(StructuredMesh(2, nx, ny, 200.0, 100.0), d.c, d.V, 0.02)
    return a.H - 1j * a.Wm, a.M, spec


def test_svqb_orthonormalises_and_drops_dependent_columns():
    from oracle.cap_lobpcg import _svqb
    rng = np.random.default_rng(0)
    S = rng.standard_normal((50, 6)) + 1j * rng.standard_normal((50, 6))
    S = np.concatenate([S, S[:, :1] * (2 - 1j)], axis=1)   # a dependent column
    M = np.diag(rng.uniform(0.5, 2.0, 50))
    G = S.conj().T @ M @ S
    B = _svqb(G, 1e-12)
    assert B.shape == (7, 6)
    assert np.abs(B.conj().T @ G @ B - np.eye(6)).max() < 1e-10


def test_host_lobpcg_nearest_matches_shift_invert():
    from oracle.cap_lobpcg import solve_nearest
    A, M, spec = _pencil()
    k, sigma = 8, -0.05
    w, _ = O.eig_nearest_complex(A, M, k, sigma)
    # 24 levels lie below sigma on this 8 nm lattice: the 8 nearest are levels
    # ~20-27 by real part, inside the lowest 32
    res = solve_nearest(_HostPencil(A, M, spec), k=k, sigma=sigma, nev=32, b=40,
                        precision="fp64", tol=1e-9, max_iter=300)
    assert res.info["complete"], res.info
    err = np.abs(np.sort_complex(res.E) - np.sort_complex(w)) / np.abs(np.sort_complex(w))
    assert err.max() <= 1e-9, err
    X = res.X.numpy()
    assert np.abs(np.einsum("ij,ij->j", X, M @ X) - 1.0).max() < 1e-10   # x^T M x = 1
    assert res.residual.max() < 1e-8


def test_incomplete_window_is_reported():
    """Too few levels for the window: the check must say so."""
    from oracle.cap_lobpcg import solve_nearest
    A, M, spec = _pencil()
    res = solve_nearest(_HostPencil(A, M, spec), k=8, sigma=-0.05, nev=16, b=24,
                        precision="fp64", tol=1e-9, max_iter=300)
    assert not res.info["complete"]
    assert res.info["kth_distance"] > res.info["unconverged_bound"]


def test_zero_cap_reduces_to_hermitian_levels():
    """W -> 0: the complex-symmetric solve returns the Hermitian eigenvalues
    (the oracle's eigsh) with zero imaginary parts."""
    from oracle.cap_lobpcg import solve_nearest
    from qdsim_b200 import workloads as W
    from qdsim_b200.eigen import DSTPreconditioner
    from qdsim_b200.mesh import StructuredMesh
    d = W.c2_dot(0, nx=24, ny=12)
    om = O.structured_mesh(2, 24, 12, 200.0, 100.0)
    a = O.assemble(om, d.c, d.V)
    spec = DSTPreconditioner.spec_for(StructuredMesh(2, 24, 12, 200.0, 100.0), d.c, d.V, 0.02)
    Eh, _ = O.eig_lowest(a.H, a.M, 32, O.sigma_below(d.V))
    res = solve_nearest(_HostPencil(a.H.astype(np.complex128), a.M, spec), k=8, sigma=-0.05,
                        nev=32, b=40, precision="fp64", tol=1e-9, max_iter=300)
    assert res.info["complete"], res.info
    assert np.abs(res.E.imag).max() <= 1e-12 * np.abs(res.E).max()
    near = Eh[np.argsort(np.abs(Eh + 0.05), kind="stable")[:8]]
    err = np.abs(np.sort(res.E.real) - np.sort(near)) / np.abs(np.sort(near))
    assert err.max() <= 1e-9, err


def test_round_robin_order_covers_every_pair_once():
    from oracle.cap_lobpcg import round_robin_pairs
    for N in (2, 4, 10, 144):
        seen = set()
        for pairs in round_robin_pairs(N):
            idx = [i for pq in pairs for i in pq]
            assert sorted(idx) == list(range(N))          # disjoint, complete
            for p, q in pairs:
                assert p < q and (p, q) not in seen
                seen.add((p, q))
        assert len(seen) == N * (N - 1) // 2


def _nonnormal(n, seed, skew=0.05):
    """A Hermitian matrix plus a non-Hermitian perturbation (the kind of
    projected matrix the open system's Rayleigh-Ritz produces)."""
    rng = np.random.default_rng(seed)
    A = rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))
    B = rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))
    return 0.5 * (A + A.conj().T) + np.diag(np.linspace(0, 5, n)) + skew * B


def test_schur_jacobi_matches_lapack():
    from oracle.cap_lobpcg import schur_jacobi, schur_eigvecs
    for n, seed in ((7, 0), (24, 1), (61, 2)):
        C = _nonnormal(n, seed)
        T, Z, sweeps, conv = schur_jacobi(C)
        assert conv and sweeps <= 20, sweeps
        assert np.abs(Z.conj().T @ Z - np.eye(n)).max() < 1e-12          # unitary
        assert np.abs(np.tril(T, -1)).max() <= 1e-13 * np.linalg.norm(C)    # triangular
        assert np.linalg.norm(Z @ T @ Z.conj().T - C) <= 1e-12 * np.linalg.norm(C)
        w = np.linalg.eigvals(C)
        d = np.diag(T)
        assert max(np.min(np.abs(w - x)) for x in d) <= 1e-10 * np.abs(w).max()
        idx = np.argsort(d.real, kind="stable")[:5]
        V = schur_eigvecs(T, Z, idx)
        r = np.linalg.norm(C @ V - V * d[idx], axis=0) / np.linalg.norm(V, axis=0)
        assert r.max() <= 1e-11 * np.abs(w).max(), r


def test_schur_jacobi_hermitian_is_eigendecomposition():
    from oracle.cap_lobpcg import schur_jacobi
    rng = np.random.default_rng(5)
    A = rng.standard_normal((30, 30)) + 1j * rng.standard_normal((30, 30))
    H = A + A.conj().T
    T, Z, _, conv = schur_jacobi(H)
    assert conv
    assert np.linalg.norm(T - np.diag(np.diag(T))) <= 1e-13 * np.linalg.norm(H)
    assert np.allclose(np.sort(np.diag(T).real), np.linalg.eigvalsh(H), atol=1e-12 * 60)

"""CPU restatement of the open-system (complex absorbing potential) block
LOBPCG that ``qd_cap_lobpcg_solve`` runs on the GPU
(``qdsim_b200/csrc/cap_lobpcg.cu``).  TEST INFRASTRUCTURE ONLY (the checker,
never the product path).

Same iteration, step for step: residuals and the active columns, the
preconditioned search directions, a Hermitian M-orthonormal basis of [X P W]
(Cholesky of the diagonally scaled Gram matrix while its pivots exceed 1e-6,
else SVQB), the projected non-Hermitian eigenproblem with the b Ritz pairs of
smallest real part, x^H M x = 1 Ritz vectors, and the final bilinear
Rayleigh quotients, x^T M x = 1 normalisation and nearest-sigma selection.
The projected eigenproblem is solved with LAPACK here; ``schur_jacobi``
restates the GPU's Schur kernel (Stewart's Jacobi-like method for
non-Hermitian matrices, parallel round-robin order) for its own tests.
The problem object supplies ``n``, ``device``, ``spmm(X, AX, MX)`` and
``precondition(R)`` (scipy products and the exact DST in the CPU tests).
The reference solves the same pencil densely:
backend/src/schrodinger.cpp:699-818.
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np
import torch
from scipy.linalg import solve_triangular
from threadpoolctl import threadpool_limits


@dataclass
class CAPResult:
    E: np.ndarray            # complex [k], nearest sigma first
    X: torch.Tensor          # complex128 [n, k], x^T M x = 1
    residual: np.ndarray     # [k] ||A x - E M x|| / (|E| ||M x||)
    info: dict


def round_robin_pairs(N):
    """Pairs (p < q) of each round of the parallel order on N (even) indices:
    index N-1 fixed, the others rotating; N-1 rounds cover every pair once."""
    M = N - 1
    rounds = []
    for r in range(M):
        pr = []
        for k in range(N // 2):
            if k == 0:
                p, q = M, r
            else:
                p, q = (r + k) % M, (r - k + M) % M
            pr.append((min(p, q), max(p, q)))
        rounds.append(pr)
    return rounds


def schur_rotation(a, b, c, d):
    """Unitary U = [[u1, -conj(u2)], [u2, conj(u1)]] whose first column is the
    eigenvector of [[a, b], [c, d]] for the eigenvalue nearer a, so that
    U^H [[a, b], [c, d]] U is upper triangular."""
    h = 0.5 * (a - d)
    disc = np.sqrt(h * h + b * c)
    g1, g2 = h + disc, h - disc
    g = g1 if abs(g1) >= abs(g2) else g2
    delta = b * c / g if g != 0 else 0.0
    v1, v2 = 2.0 * h + delta, c
    nv = math.sqrt(abs(v1) ** 2 + abs(v2) ** 2)
    return v1 / nv, v2 / nv


def schur_jacobi(C, rel_tol=1e-14, max_sweeps=60):
    """Schur form C = Z T Z^H by cyclic 2 x 2 rotations in the parallel
    round-robin order (G. W. Stewart, SIAM J. Sci. Stat. Comput. 6 (1985)
    853-864), as the GPU kernel runs it: per round, all pairs' rotations from
    the current 2 x 2 blocks, then the row rotations, then the column
    rotations; a rotation only where |c_qp| > rel_tol ||C||_F; stop after a
    sweep without one.  Returns (T, Z, sweeps, converged)."""
    n = C.shape[0]
    N = n + (n & 1)
    T = np.zeros((N, N), complex)
    T[:n, :n] = C
    Z = np.eye(N, dtype=complex)
    thresh = rel_tol * np.linalg.norm(C)
    sweeps, converged = 0, N < 2
    rounds = round_robin_pairs(N) if N >= 2 else []
    for _ in range(max_sweeps if N >= 2 else 0):
        count = 0
        for pairs in rounds:
            rots = []
            for p, q in pairs:
                if abs(T[q, p]) > thresh:
                    rots.append((p, q) + schur_rotation(T[p, p], T[p, q], T[q, p], T[q, q]))
                    count += 1
            for p, q, u1, u2 in rots:
                x, y = T[p].copy(), T[q].copy()
                T[p] = np.conj(u1) * x + np.conj(u2) * y
                T[q] = u1 * y - u2 * x
            for p, q, u1, u2 in rots:
                for A in (T, Z):
                    x, y = A[:, p].copy(), A[:, q].copy()
                    A[:, p] = x * u1 + y * u2
                    A[:, q] = y * np.conj(u1) - x * np.conj(u2)
                T[q, p] = 0.0
        sweeps += 1
        if count == 0:
            converged = True
            break
    return T[:n, :n], Z[:n, :n], sweeps, converged


def schur_eigvecs(T, Z, idx):
    """Eigenvectors Z y of C for the diagonal positions idx of its Schur form
    (back-substitution in T, tiny denominators raised to eps max|T_ii|)."""
    tmax = np.abs(np.diag(T)).max()
    smin = max(2.220446049250313e-16 * tmax, 1e-300)
    V = np.zeros((T.shape[0], len(idx)), complex)
    for j, pos in enumerate(idx):
        lam = T[pos, pos]
        y = np.zeros(T.shape[0], complex)
        y[pos] = 1.0
        rhs = -T[:pos, pos].copy()
        for i in range(pos - 1, -1, -1):
            den = T[i, i] - lam
            if abs(den) < smin:
                den = smin
            y[i] = rhs[i] / den
            rhs[:i] -= T[:i, i] * y[i]
        V[:, j] = Z @ y
    return V


def _orthonormaliser(GM, drop):
    """B with B^H GM B = I: Cholesky of the diagonally scaled Gram matrix when
    its smallest pivot shows the basis is well conditioned (condition number
    below ~1e6), else SVQB, which also drops dependent directions."""
    d = np.sqrt(np.maximum(GM.diagonal().real, 0.0))
    if np.all(d > 0.0):
        Gs = GM / d[:, None] / d[None, :]
        try:
            L = np.linalg.cholesky(0.5 * (Gs + Gs.conj().T))
        except np.linalg.LinAlgError:
            L = None
        if L is not None and np.min(np.abs(L.diagonal())) ** 2 > 1e-6:
            Linv = solve_triangular(L, np.eye(L.shape[0]), lower=True)
            return Linv.conj().T / d[:, None]
    return _svqb(GM, drop)


def _svqb(GM, drop):
    """Hermitian M-orthonormalising transform of a basis from its Gram
    matrix: B with B^H GM B = I on the numerically independent directions."""
    d = np.sqrt(np.maximum(GM.diagonal().real, 0.0))
    ok = d > 0.0
    dinv = np.where(ok, 1.0 / np.where(ok, d, 1.0), 0.0)
    Gs = GM * dinv[:, None] * dinv[None, :]
    Gs = 0.5 * (Gs + Gs.conj().T)
    lam, U = np.linalg.eigh(Gs)
    keep = lam > drop * max(lam[-1], 1e-300)
    return (dinv[:, None] * U[:, keep]) / np.sqrt(lam[keep])[None, :]


class _Block:
    """Basis buffers S = [X P W], AS, MS (complex, [n, 3b]) of one precision."""

    def __init__(self, n, b, dtype, device):
        z = lambda: torch.zeros(n, 3 * b, dtype=dtype, device=device)  # noqa: E731
        self.S, self.AS, self.MS = z(), z(), z()


def lobpcg_cap(prob, b: int, nev: int, tol: float, max_iter: int,
               dtype=torch.complex128, X0=None, seed: int = 1234, eig_scale: float = 0.01,
               stall: int = 0, on_iter=None):
    """Block LOBPCG on (A, M) for the nev eigenvalues of smallest real part.

    Returns (theta [b] complex numpy sorted by real part, X [n, b], AX, MX,
    residuals [b], iterations).  With ``stall`` > 0 the iteration also stops
    when the largest of the first nev residuals has not decreased for that
    many iterations (the FP32 phase's hand-over)."""
    n, dev = prob.n, prob.device
    drop = 1e-6 if dtype == torch.complex64 else 1e-14
    cur, nxt = _Block(n, b, dtype, dev), _Block(n, b, dtype, dev)
    if X0 is None:
        g = torch.Generator(device="cpu").manual_seed(seed)
        X0 = torch.view_as_complex(torch.randn(n, b, 2, generator=g, dtype=torch.float64))
    cur.S[:, :b] = X0.to(dev, dtype)
    X, AX, MX = cur.S[:, :b], cur.AS[:, :b], cur.MS[:, :b]
    prob.spmm(X, AX, MX)
    # initial Rayleigh-Ritz on span(X)
    Y, theta = _rr(cur, b, b, 0, drop)
    _combine(cur, nxt, Y, b, b, 0, with_p=False)
    cur, nxt = nxt, cur
    prob.spmm(cur.S[:, :b], cur.AS[:, :b], cur.MS[:, :b])
    npc = 0
    best, since = math.inf, 0
    res = np.full(b, np.inf)
    it = 0
    for it in range(1, max_iter + 1):
        X, AX, MX = cur.S[:, :b], cur.AS[:, :b], cur.MS[:, :b]
        th = torch.from_numpy(theta).to(dev, dtype)
        R = AX - MX * th[None, :]
        rn = torch.linalg.vector_norm(R, dim=0).double().cpu().numpy()
        mn = torch.linalg.vector_norm(MX, dim=0).double().cpu().numpy()
        res = rn / (np.maximum(mn, 1e-300) * np.maximum(np.abs(theta), eig_scale))
        if on_iter is not None:
            on_iter(it, theta, res)
        worst = float(res[:nev].max())
        if worst <= tol:
            break
        if stall:
            if worst < 0.9 * best:
                best, since = worst, 0
            else:
                since += 1
                if since >= stall:
                    break
        act = np.nonzero(res > tol)[0]
        act = act if act.size >= 2 else np.arange(b - 2, b)
        m = int(act.size)
        Wc = prob.precondition(R[:, torch.from_numpy(act).to(dev)])
        w0 = b + npc
        cur.S[:, w0:w0 + m] = Wc
        prob.spmm(cur.S[:, w0:w0 + m], cur.AS[:, w0:w0 + m], cur.MS[:, w0:w0 + m])
        Y, theta = _rr(cur, b, b + npc + m, npc, drop)
        _combine(cur, nxt, Y, b, b + npc + m, npc, with_p=True)
        cur, nxt = nxt, cur
        npc = b
        # explicit products of the new X (P's products are combined)
        prob.spmm(cur.S[:, :b], cur.AS[:, :b], cur.MS[:, :b])
    X, AX, MX = cur.S[:, :b], cur.AS[:, :b], cur.MS[:, :b]
    return theta, X.clone(), AX.clone(), MX.clone(), res, it


def _rr(blk: _Block, b, used, npc, drop):
    """Ritz pairs of (A, M) on span S[:, :used]: (Y [used, b] device, theta)."""
    S = blk.S[:, :used]
    GM = (S.mH @ blk.MS[:, :used]).to(torch.complex128).cpu().numpy()
    GA = (S.mH @ blk.AS[:, :used]).to(torch.complex128).cpu().numpy()
    # the projected problem is at most 3b x 3b: one BLAS thread (a threaded
    # BLAS on matrices this small only contends with the host's other work)
    with threadpool_limits(limits=1, user_api="blas"):
        return _rr_small(GM, GA, b, drop, blk.S)


def _rr_small(GM, GA, b, drop, like):
    Bm = _orthonormaliser(0.5 * (GM + GM.conj().T), drop)
    C = Bm.conj().T @ GA @ Bm
    w, V = np.linalg.eig(C)
    order = np.argsort(w.real, kind="stable")[:b]
    Y = Bm @ V[:, order]
    # Hermitian M-normalise the Ritz vectors (x^H M x = 1)
    nrm = np.sqrt(np.maximum(np.sum(Y.conj() * (GM @ Y), axis=0).real, 1e-300))
    Y = Y / nrm[None, :]
    return torch.from_numpy(Y).to(like.device, like.dtype), w[order]


def _combine(cur: _Block, nxt: _Block, Y, b, used, npc, with_p):
    """nxt.X = cur.S Y; nxt.P = cur.S[:, b:] Y[b:] (and the same for AS, MS)."""
    for src, dst in ((cur.S, nxt.S), (cur.AS, nxt.AS), (cur.MS, nxt.MS)):
        dst[:, :b].copy_(src[:, :used] @ Y)
        if with_p:
            dst[:, b:2 * b].copy_(src[:, b:used] @ Y[b:])


def solve_nearest(prob, k: int = 20, sigma: float = -0.05, nev: int = 40, b: int = 48,
                  precision: str = "mixed", tol: float = 1e-9, tol32: float = 1e-4,
                  max_iter: int = 2000, seed: int = 1234, eig_scale: float = 0.01) -> CAPResult:
    """The k eigenvalues nearest sigma from the nev lowest (by real part) of a
    problem exposing ``n``, ``device``, ``spmm`` and ``precondition``."""
    info = {"block": b, "nev": nev, "precision": precision}
    X0 = None
    it32 = 0
    if precision == "mixed":
        _, X, _, _, res32, it32 = lobpcg_cap(prob, b, nev, tol32, max_iter, dtype=torch.complex64,
                                             seed=seed, eig_scale=eig_scale, stall=8)
        X0 = X.to(torch.complex128)
        info["fp32_residual"] = float(res32[:nev].max())
    elif precision != "fp64":
        raise ValueError("precision must be 'mixed' or 'fp64'")
    th, X, AX, MX, res, it64 = lobpcg_cap(prob, b, nev, tol, max_iter, dtype=torch.complex128,
                                          X0=X0, seed=seed, eig_scale=eig_scale)
    info.update(iters_fp32=int(it32), iters_fp64=int(it64), iterations=int(it32 + it64))
    E, Xn, rres, sel = nearest_from_block(th, X, AX, MX, res, k, sigma, nev, tol)
    info.update(sel)
    return CAPResult(E, Xn, rres, info)


def nearest_from_block(theta, X, AX, MX, res, k, sigma, nev, tol):
    """Bilinear Rayleigh quotients of the converged block columns, x^T M x = 1
    normalisation, the k nearest sigma and the completeness check."""
    xtax = (X * AX).sum(dim=0)
    xtmx = (X * MX).sum(dim=0)
    E = (xtax / xtmx).cpu().numpy()
    s = torch.sqrt(xtmx)
    Xn, AXn, MXn = X / s[None, :], AX / s[None, :], MX / s[None, :]
    Et = torch.from_numpy(E).to(X.device)
    R = AXn - MXn * Et[None, :]
    rres = (torch.linalg.vector_norm(R, dim=0) /
            (torch.linalg.vector_norm(MXn, dim=0) * torch.abs(Et))).cpu().numpy()
    conv = np.asarray(res) <= tol
    conv[nev:] = False
    idx_c = np.nonzero(conv)[0]
    pick = idx_c[np.argsort(np.abs(E[idx_c] - sigma), kind="stable")[:k]]
    dk = float(np.abs(E[pick] - sigma).max()) if pick.size else math.inf
    unconv = np.nonzero(~conv)[0]
    bound = float(np.asarray(theta)[unconv].real.min() - sigma) if unconv.size else math.inf
    sel = dict(converged=int(conv.sum()), complete=bool(pick.size == k and dk < bound),
               kth_distance=dk, unconverged_bound=bound,
               max_residual=float(rres[pick].max()) if pick.size else math.inf)
    return E[pick], Xn[:, torch.from_numpy(pick).to(X.device)], rres[pick], sel

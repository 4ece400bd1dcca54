"""FP64 restatement of the batched self-consistent loop (TEST INFRASTRUCTURE
ONLY; imported by tests, never by the product).

Fixed-point map, per bias point, as ``CythonSelfConsistentSolver``
(qdsim_cython/solvers/self_consistent_solver.pyx):
  * Schrodinger with V_static - phi (:211-232), k lowest states (:172);
  * E_F = E_0 + kT/2 (:252-254); f = 1/(1 + exp((E - E_F)/kT)) where the
    exponent is below 50, else 0 (:262-266); n = sum f |psi|^2 (:269-270),
    rescaled so that mean(n) = N_D (:273-274); p = N_A exp(-q phi/kT) where
    phi > 0, else N_A (:277-283);
  * Poisson with rho = q (p - n) and phi = V_p / V_n at x = 0 / Lx (:186-187,
    the charge function of the constructor).
Mixing as ``SelfConsistentSolver`` (backend/src/self_consistent.cpp):
  * damping phi_old + beta (phi_upd - phi_old), beta = 0.3 (:36, :1270-1273),
    for the first 5 iterations (:1575-1580);
  * then Anderson (:1291-1419): history of the last 3 updates and residuals;
    F_j = r_j - r_m; least squares min ||F a + r_m|| by column-pivoted QR with
    rank threshold 1e-10, else Tikhonov on the normal equations with
    1e-4 / 1e-6 / 1e-8 x s_max for condition numbers > 1e8 / > 1e6 / else;
    a clipped to [-2, 2], rescaled so |sum a| <= 2; phi_acc = upd_m +
    sum a_j (upd_j - upd_m); backtracking line search (:1433-1468) on
    ||phi_old + s (phi_acc - phi_old) - phi_upd|| <= (1 - s/2) ||phi_upd - phi_old||,
    s = 1, 1/2, ... (10 tries, else 0.1); non-finite or |phi| > 100 -> damping
    of the update; otherwise damping of the line-search point (:1418);
  * error ||phi_new - phi_old|| / ||phi_new|| (:1604); beta *= 0.8 when the
    error grows while beta > 0.1 (:1644-1647).
Lengths nm, energies eV, phi V, densities m^-3.
"""
import numpy as np

from . import fem as F
from . import poisson as OP

K_B_EV = 8.617333262e-5


def density(mesh, X, E, phi, kT, N_A, N_D):
    """n, p, rho for one bias point; X reduced eigenvectors [rows, k], E [k] (eV)."""
    dm = F.dof_map(mesh, True)
    ef = E[0] + 0.5 * kT
    a = (E - ef) / kT
    f = np.where(a < 50.0, 1.0 / (1.0 + np.exp(np.minimum(a, 50.0))), 0.0)
    n = np.zeros(mesh.num_nodes)
    keep = dm >= 0
    n[keep] = (X[dm[keep]] ** 2) @ f
    if n.sum() > 0:
        n *= N_D / n.mean()
    p = np.where(phi > 0, N_A * np.exp(-np.maximum(phi, 0.0) / kT), N_A)
    return n, p, OP.Q_E * (p - n)


def g_map(mesh, eps_r, c, V_static, phi, V_p, V_n, k, T, N_A, N_D):
    """G(phi) for all bias points: phi [N, nb] -> ([N, nb], E [nb, k])."""
    kT = K_B_EV * T
    nb = phi.shape[1]
    rho = np.zeros_like(phi)
    Es = np.zeros((nb, k))
    for b in range(nb):
        V = V_static - phi[:, b]
        a = F.assemble(mesh, c, V)
        E, X = F.eig_lowest(a.H, a.M, k, F.sigma_below(V))
        Es[b] = E
        _, _, rho[:, b] = density(mesh, X, E, phi[:, b], kT, N_A, N_D)
    return OP.solve(mesh, eps_r, rho, V_p, V_n), Es


def anderson_coefficients(res_hist):
    """Least-squares coefficients of self_consistent.cpp:1313-1380 (None: failed)."""
    m = len(res_hist) - 1
    Fm = np.stack([res_hist[j] - res_hist[m] for j in range(m)], axis=1)
    t = -res_hist[m]
    if m == 1:
        d = Fm[:, 0] @ Fm[:, 0]
        if not d > 0:
            return None
        al = np.array([(Fm[:, 0] @ t) / d])
    else:
        G = Fm.T @ Fm
        c = Fm.T @ t
        aa, bb = (G[1, 1], G[0, 0]) if G[1, 1] > G[0, 0] else (G[0, 0], G[1, 1])
        r11 = np.sqrt(max(bb - (G[0, 1] ** 2 / aa if aa > 0 else 0.0), 0.0))
        if aa > 0 and r11 > 1e-10 * np.sqrt(aa):
            al = np.linalg.solve(G, c)
        elif aa > 0:
            s = np.sqrt(np.maximum(np.linalg.eigvalsh(G)[::-1], 0.0))
            cond = s[0] / s[-1] if s[-1] > 0 else np.inf
            reg = (1e-4 if cond > 1e8 else 1e-6 if cond > 1e6 else 1e-8) * s[0]
            al = np.linalg.solve(G + reg * np.eye(2), c)
        else:
            return None
    if not np.all(np.isfinite(al)):
        return None
    al = np.clip(al, -2.0, 2.0)
    if abs(al.sum()) > 2.0:
        al *= 2.0 / abs(al.sum())
    return al


def mix(old, upd, hist_u, hist_r, beta, anderson):
    """One mixing step for one bias point; hist_* already hold this update."""
    if anderson and len(hist_u) >= 2:
        al = anderson_coefficients(hist_r)
        if al is not None:
            m = len(hist_u) - 1
            acc = hist_u[m] + sum(al[j] * (hist_u[j] - hist_u[m]) for j in range(m))
            r0 = np.linalg.norm(upd - old)
            s, chosen = 1.0, 0.1
            for _ in range(10):
                if np.linalg.norm(old + s * (acc - old) - upd) <= (1.0 - 0.5 * s) * r0:
                    chosen = s
                    break
                s *= 0.5
            ls = old + chosen * (acc - old)
            if np.all(np.isfinite(ls)) and np.max(np.abs(ls)) <= 100.0:
                return old + beta * (ls - old)
    return old + beta * (upd - old)


def run(junction, k, iterations, V_p=None, damping=0.3, anderson_start=5, history=3, phi0=None,
        on_iter=None):
    """The mixed fixed-point iteration for every bias point of ``junction``;
    returns phi [N, nb], errors [iterations, nb], E [nb, k] of the last map.
    ``on_iter(it, phi, E)`` (optional) sees each iteration's mixed potential
    and the levels of its map."""
    j = junction
    mesh = j.mesh
    nb = len(j.biases)
    V_n = np.asarray(j.biases, float)
    V_p = np.zeros(nb) if V_p is None else np.asarray(V_p, float)
    x = mesh.nodes[:, 0]
    phi = (phi0.copy() if phi0 is not None
           else V_p[None, :] + (V_n - V_p)[None, :] * (x / mesh.Lx)[:, None])
    beta = np.full(nb, damping)
    prev = np.full(nb, 1e10)
    hu = [[] for _ in range(nb)]
    hr = [[] for _ in range(nb)]
    errors = []
    E = None
    for it in range(iterations):
        upd, E = g_map(mesh, j.eps_r, j.c, j.V_static, phi, V_p, V_n, k, j.T, j.N_A, j.N_D)
        new = np.empty_like(phi)
        err = np.zeros(nb)
        anderson = it >= anderson_start
        for b in range(nb):
            if anderson:
                hu[b].append(upd[:, b].copy())
                hr[b].append(upd[:, b] - phi[:, b])
                if len(hu[b]) > history:
                    hu[b].pop(0)
                    hr[b].pop(0)
            new[:, b] = mix(phi[:, b], upd[:, b], hu[b], hr[b], beta[b], anderson)
            nn = np.linalg.norm(new[:, b])
            err[b] = np.linalg.norm(new[:, b] - phi[:, b]) / (nn if nn > 0 else 1.0)
            if err[b] > prev[b] and beta[b] > 0.1:
                beta[b] *= 0.8
            prev[b] = err[b]
        phi = new
        errors.append(err)
        if on_iter is not None:
            on_iter(it, phi, E)
    return phi, np.array(errors), E

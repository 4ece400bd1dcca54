"""Self-consistent Poisson-Schrodinger loop batched over bias points.

The fixed-point map is the one of ``CythonSelfConsistentSolver``
(qdsim_cython/solvers/self_consistent_solver.pyx:130-286): Schrodinger with
V_static - phi, Fermi-Dirac occupation of the k lowest states with
E_F = E_0 + kT/2, electron density rescaled to mean N_D, classical holes,
Poisson with rho = q (p - n) and phi = V_p / V_n on x = 0 / x = Lx.  The
mixing is the one of ``SelfConsistentSolver`` (backend/src/self_consistent.cpp:
1262-1468, 1570-1647): damping 0.3 for the first 5 iterations, then Anderson
acceleration over the last 3 updates with a backtracking line search and
damping, the damping factor shrinking by 0.8 whenever the error grows.

All bias points advance together: one batched LOBPCG over the bias points'
potentials (one mesh, one dot per bias), one batched Jacobi-PCG (one stiffness,
one right-hand side per bias), densities and mixing in ``qd_sc_density`` /
``qd_sc_mix`` (one CTA per bias).  The eigenvectors of one iteration warm-start
the next.  Units: nm, eV for Schrodinger; V and C/m^3 for Poisson.

``dE1_dbias`` differentiates the converged lowest level with respect to the
bias through the fixed point phi* = G(phi*, V): the bias enters G only through
the Dirichlet data, so dG/dV = h (the Laplace solution with phi = 0 at x = 0 and
1 at x = Lx), u = dphi*/dV solves (I - J) u = h with J = dG/dphi (GMRES, batched
over the bias points, J v by central differences of G), and
dE1/dV = -(dE1/dV_nodal) . u with dE1/dV_nodal from ``qd_adjoint``.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from . import _native as N
from .adjoint import energy_gradients
from .batch import DeviceBatch, HostBatch
from .fem import FEMProblem, dof_map_for, stream_ptr
from .poisson import PoissonProblem
from .workloads import Dot, Junction

K_B_EV = 8.617333262e-5     # Boltzmann constant, eV/K


class BatchedSC:
    def __init__(self, junction: Junction, k: int = 10, device="cuda", precision="mixed",
                 tol=1e-9, pcg_tol=1e-12, block=None, warm_start=True, eig_scale=0.1,
                 shift_ev=0.5):
        self.j = junction
        self.device = torch.device(device)
        self.k = int(k)
        self.nb = len(junction.biases)
        self.kT = K_B_EV * junction.T
        # levels of the biased junction cross zero energy: errors are measured
        # relative to max(|E|, eig_scale) (eV) rather than |E|
        self.solve_kw = dict(precision=precision, tol=tol, max_iter=4000,
                             b=block or max(8, (self.k + 4 + 3) // 4 * 4),
                             eig_scale=eig_scale)
        self.pcg_tol = pcg_tol
        mesh = junction.mesh
        self.n = mesh.num_nodes
        self.poisson = PoissonProblem(mesh, junction.eps_r, device=self.device)
        dots = [Dot(mesh, junction.c, junction.V_static) for _ in range(self.nb)]
        self.hb = HostBatch(dots)
        self.db = DeviceBatch(self.hb, self.device)
        self.db.upload(non_blocking=False)
        # DST preconditioner shift (eV): the junction's potential spans ~1 eV,
        # and on the 64-bias config a 0.5 eV shift needs 56-72 LOBPCG
        # iterations per self-consistent step where the sweep's 0.02 eV needs
        # 144-168
        if shift_ev is not None:
            self.db.set_shift(shift_ev)
        dm, nrow = dof_map_for(mesh, True)
        self.rows = nrow
        self.d_dof = torch.from_numpy(dm).to(self.device)
        self.d_Vs = torch.from_numpy(np.ascontiguousarray(junction.V_static, np.float64)).to(self.device)
        self.V_n = np.asarray(junction.biases, np.float64)
        self.V_p = np.zeros(self.nb)
        f64 = dict(dtype=torch.float64, device=self.device)
        self.n_e = torch.zeros(self.n, self.nb, **f64)
        self.p_h = torch.zeros(self.n, self.nb, **f64)
        self.rho = torch.zeros(self.n, self.nb, **f64)
        self._X = None          # last eigenvectors (warm start)
        # warm-start each eigensolve from the previous iteration's vectors
        self.warm_start = bool(warm_start)
        self.E = None
        self.X = None

    # -- one evaluation of the fixed-point map ---------------------------------
    def _eigen(self, phi):
        L = N.lib()
        N.check(L.qd_sc_potential(self.nb, self.n, N.ptr(self.d_Vs), N.ptr(phi),
                                  N.ptr(self.db.d["V"]), stream_ptr()), "qd_sc_potential")
        self.db.assemble()
        # warm start from the last stored eigenvectors (random the first time)
        E, X, _, _, info, _ = self.db.solve(self.k, x0=self._X if self.warm_start else None,
                                            **self.solve_kw)
        return E, X, info

    def g_map(self, phi, store=True):
        """G(phi) for every bias point: phi [N, nb] (device) -> [N, nb].  With
        ``store`` the eigenvectors become the next call's warm start."""
        E, X, info = self._eigen(phi)
        if store:
            self._X = X.clone()
        self.E, self.X = E, X
        N.check(N.lib().qd_sc_density(self.nb, self.n, self.k, self.rows, N.ptr(self.d_dof),
                                      N.ptr(X), N.ptr(E), self.kT, self.j.N_A, self.j.N_D,
                                      N.ptr(phi), N.ptr(self.n_e), N.ptr(self.p_h),
                                      N.ptr(self.rho), stream_ptr()), "qd_sc_density")
        return self.poisson.solve(self.rho, self.V_p, self.V_n, tol=self.pcg_tol,
                                  x0=phi).reshape(self.n, self.nb)

    # -- the loop ----------------------------------------------------------------
    def initial(self):
        x = torch.from_numpy(self.j.mesh.nodes[:, 0].copy()).to(self.device)
        return (torch.from_numpy(self.V_p).to(self.device)[None, :]
                + (torch.from_numpy(self.V_n - self.V_p).to(self.device)[None, :]
                   * (x / self.j.mesh.Lx)[:, None])).contiguous()

    def solve(self, iterations=40, phi0=None, damping=0.3, anderson_start=5, history=3):
        """Run the mixed fixed-point iteration; returns phi [N, nb] and the
        per-iteration errors ||phi_new - phi_old|| / ||phi_new|| [iter, nb]."""
        f64 = dict(dtype=torch.float64, device=self.device)
        phi = (phi0.clone() if phi0 is not None else self.initial()).contiguous()
        beta = torch.full((self.nb,), float(damping), **f64)
        prev = torch.full((self.nb,), 1e10, **f64)
        err = torch.zeros(self.nb, **f64)
        hist_u = [torch.empty(self.n, self.nb, **f64) for _ in range(history)]
        hist_r = [torch.empty(self.n, self.nb, **f64) for _ in range(history)]
        order = list(range(history))        # oldest first
        nhist = 0
        errors = []
        L = N.lib()
        for it in range(iterations):
            upd = self.g_map(phi)
            new = torch.empty_like(phi)
            anderson = it >= anderson_start
            if anderson:
                if nhist == history:
                    order = order[1:] + order[:1]    # drop the oldest, reuse its buffers
                else:
                    nhist += 1
                hu = (C.c_void_p * history)(*[hist_u[i].data_ptr() for i in order])
                hr = (C.c_void_p * history)(*[hist_r[i].data_ptr() for i in order])
            else:
                hu = hr = None
            N.check(L.qd_sc_mix(self.nb, self.n, 1 if anderson else 0, nhist if anderson else 0,
                                N.ptr(phi), N.ptr(upd), hu, hr, N.ptr(new), N.ptr(beta),
                                N.ptr(prev), N.ptr(err), stream_ptr()), "qd_sc_mix")
            phi = new
            errors.append(err.clone())
        self.phi = phi
        self.damping = beta
        return phi, torch.stack(errors)

    # -- implicit derivative of E1 with respect to the bias ---------------------
    def lifting(self):
        z = torch.zeros(self.n, self.nb, dtype=torch.float64, device=self.device)
        return self.poisson.solve(z, np.zeros(self.nb), np.ones(self.nb),
                                  tol=self.pcg_tol).reshape(self.n, self.nb)

    def _jvp(self, phi, v, eps):
        # central difference of G along v; the Dirichlet part of G cancels
        gp = self.g_map(phi + eps[None, :] * v, store=False)
        gm = self.g_map(phi - eps[None, :] * v, store=False)
        return (gp - gm) / (2.0 * eps[None, :])

    def dE1_dbias(self, phi_star, restart=12, rel_eps=1e-3, gmres_tol=1e-8):
        """dE_1/dV_n per bias point at the converged potential phi_star."""
        h = self.lifting()
        # GMRES on (I - J) u = h, one system per bias point (columns)
        beta0 = torch.linalg.vector_norm(h, dim=0)
        Q = [h / beta0[None, :]]
        Hm = torch.zeros(restart + 1, restart, self.nb, dtype=torch.float64, device=self.device)
        for j in range(restart):
            v = Q[j]
            eps = rel_eps * torch.clamp(phi_star.abs().amax(dim=0), min=1.0) / \
                torch.clamp(v.abs().amax(dim=0), min=1e-300)
            w = v - self._jvp(phi_star, v, eps)
            for i in range(j + 1):            # modified Gram-Schmidt, per column
                hij = (Q[i] * w).sum(dim=0)
                Hm[i, j] = hij
                w = w - hij[None, :] * Q[i]
            hn = torch.linalg.vector_norm(w, dim=0)
            Hm[j + 1, j] = hn
            Q.append(w / torch.clamp(hn, min=1e-300)[None, :])
            # least squares min || beta0 e1 - Hm y || per column
            H_ = Hm[: j + 2, : j + 1].permute(2, 0, 1).cpu().numpy()
            rhs = np.zeros((self.nb, j + 2))
            rhs[:, 0] = beta0.cpu().numpy()
            ys, res = [], []
            for b in range(self.nb):
                y, *_ = np.linalg.lstsq(H_[b], rhs[b], rcond=None)
                ys.append(y)
                res.append(np.linalg.norm(H_[b] @ y - rhs[b]) / max(rhs[b, 0], 1e-300))
            if max(res) < gmres_tol:
                break
        Y = torch.from_numpy(np.stack(ys, axis=1)).to(self.device)    # [j+1, nb]
        u = sum(Q[i] * Y[i][None, :] for i in range(Y.shape[0]))
        self.gmres_residual = float(max(res))
        # dE1/dphi = -(dE1/dV_nodal): adjoint gradient of the lowest level per bias
        self.g_map(phi_star, store=False)
        mesh = self.j.mesh
        prob = FEMProblem(mesh, device=self.device)
        X = self.X.reshape(self.nb, self.rows, self.k)
        dE = torch.empty(self.nb, dtype=torch.float64, device=self.device)
        for b in range(self.nb):
            gV, _ = energy_gradients(prob, X[b, :, :1], [1.0])
            dE[b] = -(gV * u[:, b]).sum()
        return dE

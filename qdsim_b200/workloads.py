"""Seeded synthetic inputs with the shapes of the benchmark configurations.

There is no public dataset for this path; every input is drawn from
``numpy.random.default_rng`` with a fixed seed so that the GPU, the oracle and
the committed golden fixtures see identical meshes and coefficients.
Lengths in nm, energies in eV, kinetic coefficient c = C0 m0/m* (eV nm^2).
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from .fem import C0_EV_NM2
from .mesh import StructuredMesh

SWEEP_SEED = 20261203


@dataclass
class Dot:
    mesh: StructuredMesh
    c: np.ndarray      # per element
    V: np.ndarray      # nodal
    W: np.ndarray | None = None


def c1_dot(seed: int = 0, nx: int = 100, ny: int = 50, Lx: float = 100.0, Ly: float = 50.0) -> Dot:
    """P1, 100x50 cells on 100x50 nm; Gaussian dot -0.3 exp(-r^2/(2 8^2)) eV
    centred within +-10 nm of the middle; m* 0.041 where V(centroid) < -0.15 eV
    else 0.067 m0; homogeneous Dirichlet boundary."""
    rng = np.random.default_rng(seed)
    cx = Lx / 2 + rng.uniform(-10, 10)
    cy = Ly / 2 + rng.uniform(-10, 10)
    mesh = StructuredMesh(1, nx, ny, Lx, Ly)

    def V(x, y):
        return -0.3 * np.exp(-((x - cx) ** 2 + (y - cy) ** 2) / (2 * 8.0 ** 2))

    Vn = V(mesh.nodes[:, 0], mesh.nodes[:, 1])
    cen = mesh.centroids()
    mstar = np.where(V(cen[:, 0], cen[:, 1]) < -0.15, 0.041, 0.067)
    return Dot(mesh, C0_EV_NM2 / mstar, Vn)


def sweep_dot(i: int, base_seed: int = SWEEP_SEED, order: int = 2, nx: int | None = None) -> Dot:
    """Dot i of the batched sweep: P2, nx ~ U{40..240}, ny = nx // 2, 1 nm cells,
    circular well of radius U[5,20] nm and depth U[0.1,0.5] eV centred within
    +-5 nm of the middle, m* 0.041 m0 inside (element centroid) / 0.067 outside."""
    rng = np.random.default_rng([base_seed, i])
    n = int(rng.integers(40, 241))
    if nx is not None:
        n = int(nx)
    ny = n // 2
    Lx, Ly = float(n), float(ny)
    R = rng.uniform(5.0, 20.0)
    depth = rng.uniform(0.1, 0.5)
    cx = Lx / 2 + rng.uniform(-5.0, 5.0)
    cy = Ly / 2 + rng.uniform(-5.0, 5.0)
    mesh = StructuredMesh(order, n, ny, Lx, Ly)
    x, y = mesh.nodes[:, 0], mesh.nodes[:, 1]
    Vn = np.where((x - cx) ** 2 + (y - cy) ** 2 < R * R, -depth, 0.0)
    cen = mesh.centroids()
    inside = (cen[:, 0] - cx) ** 2 + (cen[:, 1] - cy) ** 2 < R * R
    mstar = np.where(inside, 0.041, 0.067)
    return Dot(mesh, C0_EV_NM2 / mstar, Vn)


def sweep_batch(n_dots: int = 256, base_seed: int = SWEEP_SEED, first: int = 0):
    return [sweep_dot(first + i, base_seed) for i in range(n_dots)]


def c3_dot(seed: int = 0, nx: int = 150, ny: int = 75, Lx: float = 150.0, Ly: float = 75.0) -> Dot:
    """P3 150x75 cells; Gaussian dot with seeded depth U[0.1,0.4] eV and width
    U[5,15] nm near the middle; m* 0.041 where V(centroid) < -depth/2 else 0.067."""
    rng = np.random.default_rng(seed)
    depth = rng.uniform(0.1, 0.4)
    w = rng.uniform(5.0, 15.0)
    cx = Lx / 2 + rng.uniform(-5, 5)
    cy = Ly / 2 + rng.uniform(-5, 5)
    mesh = StructuredMesh(3, nx, ny, Lx, Ly)

    def V(x, y):
        return -depth * np.exp(-((x - cx) ** 2 + (y - cy) ** 2) / (2 * w * w))

    Vn = V(mesh.nodes[:, 0], mesh.nodes[:, 1])
    cen = mesh.centroids()
    mstar = np.where(V(cen[:, 0], cen[:, 1]) < -depth / 2, 0.041, 0.067)
    return Dot(mesh, C0_EV_NM2 / mstar, Vn)


def cap_profile(x, y, Lx, Ly, W0, L):
    """CAP amplitude W0 (d/L)^2 with d the penetration depth into the boundary
    layer of width L (zero in the interior, W0 at the wall)."""
    dist = np.minimum(np.minimum(x, Lx - x), np.minimum(y, Ly - y))
    d = np.clip(L - dist, 0.0, None)
    return W0 * (d / L) ** 2


def c2_dot(seed: int = 0, nx: int = 400, ny: int = 200, Lx: float = 200.0, Ly: float = 100.0) -> Dot:
    """Open system: P2 400x200 cells on 200x100 nm, double Gaussian dot (depths
    U[0.1,0.4] eV, widths U[5,15] nm), CAP -i 0.05 (d/10)^2 eV in a 10 nm layer."""
    rng = np.random.default_rng(seed)
    mesh = StructuredMesh(2, nx, ny, Lx, Ly)
    x, y = mesh.nodes[:, 0], mesh.nodes[:, 1]
    Vn = np.zeros(mesh.num_nodes)
    cen = mesh.centroids()
    Vc = np.zeros(mesh.num_elements)
    for _ in range(2):
        d = rng.uniform(0.1, 0.4)
        w = rng.uniform(5.0, 15.0)
        cx = Lx / 2 + rng.uniform(-30, 30)
        cy = Ly / 2 + rng.uniform(-15, 15)
        Vn -= d * np.exp(-((x - cx) ** 2 + (y - cy) ** 2) / (2 * w * w))
        Vc -= d * np.exp(-((cen[:, 0] - cx) ** 2 + (cen[:, 1] - cy) ** 2) / (2 * w * w))
    mstar = np.where(Vc < -0.05, 0.041, 0.067)
    W = cap_profile(x, y, Lx, Ly, 0.05, 10.0)
    return Dot(mesh, C0_EV_NM2 / mstar, Vn, W)


@dataclass
class Junction:
    """Self-consistent p-n junction batched over bias points."""
    mesh: StructuredMesh
    eps_r: np.ndarray       # per element
    c: np.ndarray           # per element, hbar^2/(2 m*) in eV nm^2
    V_static: np.ndarray    # nodal, eV
    biases: np.ndarray      # V_n per bias point (V_p = 0), V
    N_A: float = 1e24
    N_D: float = 1e24
    T: float = 300.0


def c5_junction(n_bias: int = 64, seed: int = 0, nx: int = 300, ny: int = 100,
                Lx: float = 300.0, Ly: float = 100.0) -> Junction:
    """P1 300x100 cells on 300x100 nm; eps_r 13.9; conduction-band offset 0.2 eV
    on the p side (x < Lx/2); Gaussian dot -0.3 exp(-r^2/(2 8^2)) eV at the
    junction; m* 0.041 m0 where the dot is deeper than 0.15 eV, else 0.067 m0;
    N_A = N_D = 1e24 m^-3; bias points V_n ~ U[0, 1] V (seeded), V_p = 0."""
    rng = np.random.default_rng([seed, 5])
    mesh = StructuredMesh(1, nx, ny, Lx, Ly)
    x, y = mesh.nodes[:, 0], mesh.nodes[:, 1]

    def dot(xx, yy):
        return -0.3 * np.exp(-((xx - Lx / 2) ** 2 + (yy - Ly / 2) ** 2) / (2 * 8.0 ** 2))

    V = np.where(x < Lx / 2, 0.2, 0.0) + dot(x, y)
    cen = mesh.centroids()
    c = C0_EV_NM2 / np.where(dot(cen[:, 0], cen[:, 1]) < -0.15, 0.041, 0.067)
    return Junction(mesh, np.full(mesh.num_elements, 13.9), c, V,
                    np.sort(rng.uniform(0.0, 1.0, n_bias)))

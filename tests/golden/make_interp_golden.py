"""Golden vectors for P1 field interpolation from the reference's own Python
FEInterpolator (frontend/qdsim/fe_interpolator.py with its quadtree,
frontend/qdsim/quadtree.py), imported from the reference tree.

The reference's C++ FEInterpolator needs Eigen (absent here); its Python
fallback implements the same P1 interpolation: barycentric values and P1
gradients inside an element (fe_interpolator.py:169-255), the value of the
nearest node (first on ties) outside.  The two differ only where the fixture
does not look: the quadtree snaps points within 1e-6 outside onto an element
(quadtree.py:350-392) and returns a zero gradient outside, where the C++ class
estimates one.  So the points are drawn strictly inside one element (at least
1e-3 from every edge, in barycentric units) or more than a tenth of a cell
outside the domain.

The quadtree misses the containing element of some interior points: its
element/box overlap test leaves the element out of the point's leaf, and its
fallback then accepts another candidate because it takes the smallest of the
three clipped barycentric distances, which is 0 whenever one coordinate is
non-negative (quadtree.py:350-392).  Those points are recorded
(``quadtree_miss``: the returned element's barycentric coordinates are not all
>= -1e-10) so that the test compares the rest and records the miss.

Writes tests/golden/interp_p1.npz.  Run from the repository root:
    python tests/golden/make_interp_golden.py [reference_root]
"""
import importlib.util
import sys
import types
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent
sys.path.insert(0, str(ROOT))

from oracle.fem import structured_mesh  # noqa: E402

NX, NY, LX, LY = 12, 8, 30.0, 20.0
SEED = 2026


def _load_reference(ref: Path):
    pkg = types.ModuleType("qdsim_ref_frontend")
    pkg.__path__ = [str(ref / "frontend" / "qdsim")]
    sys.modules[pkg.__name__] = pkg
    mods = {}
    for name in ("quadtree", "fe_interpolator"):
        spec = importlib.util.spec_from_file_location(
            f"{pkg.__name__}.{name}", ref / "frontend" / "qdsim" / f"{name}.py")
        mod = importlib.util.module_from_spec(spec)
        sys.modules[spec.name] = mod
        spec.loader.exec_module(mod)
        mods[name] = mod
    return mods["fe_interpolator"].FEInterpolator


class _Mesh:
    """The two accessors the Python FEInterpolator reads."""

    def __init__(self, m):
        self._m = m

    def get_nodes(self):
        return self._m.nodes.tolist()

    def get_elements(self):
        return self._m.elems.tolist()


def main(ref_root=None):
    from oracle.build_ref import default_root
    FEI = _load_reference(Path(ref_root or default_root()))
    m = structured_mesh(1, NX, NY, LX, LY)
    it = FEI(_Mesh(m), use_cpp=False)
    rng = np.random.default_rng(SEED)
    field = rng.standard_normal(m.num_nodes)
    hx, hy = LX / NX, LY / NY
    # interior points: random cell, triangle and barycentric coordinates >= 1e-3
    n_in = 400
    ci, cj, t = rng.integers(0, NX, n_in), rng.integers(0, NY, n_in), rng.integers(0, 2, n_in)
    lam = rng.dirichlet((1.0, 1.0, 1.0), n_in) * (1 - 3e-3) + 1e-3
    v00 = np.stack([ci * hx, cj * hy], 1)
    v10, v01, v11 = v00 + [hx, 0], v00 + [0, hy], v00 + [hx, hy]
    a = np.where(t[:, None] == 0, v00, v10)
    b = np.where(t[:, None] == 0, v10, v11)
    c = v01
    p_in = lam[:, :1] * a + lam[:, 1:2] * b + lam[:, 2:] * c
    # outside points: more than a tenth of a cell past the boundary
    n_out = 80
    side = rng.integers(0, 4, n_out)
    u = rng.uniform(-0.5, 1.5, n_out)
    d = rng.uniform(0.1, 3.0, n_out)
    xo = np.where(side == 0, -d * hx, np.where(side == 1, LX + d * hx, u * LX))
    yo = np.where(side == 2, -d * hy, np.where(side == 3, LY + d * hy,
                                                np.clip(u, 0, 1) * LY))
    xo = np.where(side >= 2, u * LX, xo)
    yo = np.where(side < 2, rng.uniform(-0.2, 1.2, n_out) * LY, yo)
    x = np.concatenate([p_in[:, 0], xo])
    y = np.concatenate([p_in[:, 1], yo])
    value = np.array([it.interpolate(px, py, field) for px, py in zip(x, y)], dtype=float)
    grads = [it.interpolate_with_gradient(px, py, field) for px, py in zip(x[:n_in], y[:n_in])]
    element = np.array([it.find_element(px, py) for px, py in zip(x, y)], dtype=np.int64)
    miss = np.zeros(len(x), dtype=bool)
    for i in range(n_in):
        _, lam_ref = it._quadtree.find_element(x[i], y[i], compute_barycentric=True)
        miss[i] = min(lam_ref) < -1e-10
    np.savez_compressed(HERE / "interp_p1.npz", nx=NX, ny=NY, Lx=LX, Ly=LY, field=field,
                        x=x, y=y, n_inside=n_in, value=value,
                        grad_x=np.array([g[1] for g in grads]),
                        grad_y=np.array([g[2] for g in grads]), element=element,
                        quadtree_miss=miss)
    print(f"wrote {HERE / 'interp_p1.npz'}: {n_in} inside ({miss.sum()} missed by the "
          f"quadtree), {n_out} outside points")


if __name__ == "__main__":
    main(*sys.argv[1:])

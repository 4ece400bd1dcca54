"""Build the reference's own Cython solver modules into ``oracle/_ref/``.

TEST INFRASTRUCTURE ONLY: the compiled reference modules pin the oracle's
reference-compatible formulas (tests/golden/make_ref_golden.py) and are never
part of the product path.  The sources are compiled where they lie under the
reference tree (read-only); generated C++ and objects go to oracle/_ref/.

Modules: qdsim_cython/core/mesh_minimal.pyx, qdsim_cython/solvers/
{schrodinger_solver, fixed_open_system_solver, poisson_solver}.pyx.
poisson_solver.pyx emits ``#include "Eigen/Dense"`` for a cimport it never
uses; empty stub headers stand in for Eigen.

Usage: python oracle/build_ref.py [reference_root]
The reference root comes from the argument, else the QDSIM_REFERENCE_ROOT
environment variable, else the location this recipe was written for.
"""
import os
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
OUT = HERE / "_ref"
# (short name, extension name, source); poisson_solver keeps its package name
# because of its relative ``cimport ..eigen``.
MODULES = [
    ("mesh_minimal", "mesh_minimal", "qdsim_cython/core/mesh_minimal.pyx"),
    ("schrodinger_solver", "schrodinger_solver", "qdsim_cython/solvers/schrodinger_solver.pyx"),
    ("fixed_open_system_solver", "fixed_open_system_solver",
     "qdsim_cython/solvers/fixed_open_system_solver.pyx"),
    ("poisson_solver", "qdsim_cython.solvers.poisson_solver",
     "qdsim_cython/solvers/poisson_solver.pyx"),
]


def default_root() -> str:
    """Reference tree: $QDSIM_REFERENCE_ROOT, else the recipe's default."""
    return os.environ.get("QDSIM_REFERENCE_ROOT", "/root/reference")


def _so(short):
    hits = sorted(OUT.rglob(f"{short}*.so"))
    return hits[0] if hits else None


def built() -> bool:
    return all(_so(short) is not None for short, _, _ in MODULES)


def build(ref_root: str | None = None, quiet: bool = True) -> bool:
    """Compile the modules; returns False if the reference tree is absent."""
    ref = Path(ref_root or default_root())
    if not (ref / "qdsim_cython").is_dir():
        return False
    import numpy
    from Cython.Build import cythonize
    from setuptools import Extension
    from setuptools.dist import Distribution

    OUT.mkdir(exist_ok=True)
    stub = OUT / "stub_include" / "Eigen"
    stub.mkdir(parents=True, exist_ok=True)
    for h in ("Dense", "Sparse"):
        (stub / h).write_text("// empty stand-in: the including module never uses Eigen\n")
    exts = [Extension(ext, [str(ref / src)], language="c++",
                      include_dirs=[numpy.get_include(), str(OUT / "stub_include")],
                      extra_compile_args=["-O2", "-w"])
            for _, ext, src in MODULES]
    exts = cythonize(exts, build_dir=str(OUT / "gen"), quiet=quiet, include_path=[str(ref)],
                     compiler_directives={"language_level": "3"})
    dist = Distribution({"ext_modules": exts})
    cmd = dist.get_command_obj("build_ext")
    cmd.build_lib = str(OUT)
    cmd.build_temp = str(OUT / "tmp")
    cmd.inplace = False
    cmd.ensure_finalized()
    cmd.run()
    return built()


def import_ref(short: str):
    """Load a compiled reference module by file (not through its package,
    whose __init__ needs the unbuildable C++ backend)."""
    import importlib.util
    path = _so(short)
    if path is None:
        raise ImportError(f"reference module {short} not built (run oracle/build_ref.py)")
    if short in sys.modules:
        return sys.modules[short]
    spec = importlib.util.spec_from_file_location(short, str(path))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    sys.modules[short] = mod
    return mod


if __name__ == "__main__":
    ok = build(sys.argv[1] if len(sys.argv) > 1 else None, quiet=False)
    print("reference modules built:" if ok else "reference not found", OUT)
    sys.exit(0 if ok else 1)

"""qdsim_b200: B200-native (sm_100a) finite-element quantum-dot hot path.

Drop-in replacement for QDSim's Cython solver API (``SimpleMesh``,
``CythonSchrodingerSolver``, ``FixedOpenSystemSolver``, ``CythonPoissonSolver``,
``CythonSelfConsistentSolver``) backed by hand-written CUDA kernels in
``libqdsim_b200.so`` (C ABI in ``include/qdsim_b200.h``).
"""
from .mesh import SimpleMesh, StructuredMesh  # noqa: F401

__version__ = "0.1.0"

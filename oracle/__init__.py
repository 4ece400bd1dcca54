"""FP64 CPU oracle for the QDSim finite-element hot path.

TEST INFRASTRUCTURE ONLY.  Nothing in ``qdsim_b200`` imports this package:
it is used by ``tests/``, ``__graft_entry__.smoke()`` (as the checker) and the
``cpu_baseline`` / ``--impl reference`` legs of ``bench.py``.  The product path
runs on the GPU through ``libqdsim_b200.so`` and fails loudly without it.

Modules
-------
fem        mesh generators, P1/P2/P3 shape functions and quadrature, element
           matrices, CSR assembly, CAP profile, Dirichlet elimination and the
           scipy shift-invert eigensolve (restating ``backend/src/fem.cpp`` and
           ``backend/src/fe_interpolator.cpp``).
refcompat  the reference Cython solvers' own element formulas (bug-compatible),
           pinned against the compiled reference modules.
poisson    P1 Poisson assembly / RHS / Dirichlet solve / E-field
           (``qdsim_cython/solvers/poisson_solver.pyx``).
sc         density and the self-consistent loop with Anderson mixing
           (``qdsim_cython/solvers/self_consistent_solver.pyx``,
           ``backend/src/self_consistent.cpp``).
adjoint    FP64 reference gradients dE/dV and dE/dc by the Hellmann-Feynman
           formula, checked against finite differences.
"""

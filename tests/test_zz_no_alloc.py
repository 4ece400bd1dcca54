"""The PCG entry point that allocates nothing (qd_pcg_solve_static).

Some callers cannot allocate device memory -- for instance a solver step run
inside another runtime that owns all device memory, or a loop that must not
call cudaMalloc between launches.  qd_pcg_solve_static serves them from a
scratch array the library reserves per GPU.  These checks call it through the
C ABI and compare it with qd_pcg_solve (caller-provided workspace) on two
calls in a row, so that scratch left over from the first call cannot change
the second answer.  The file sorts last so a stop-at-first-failure run has
already run every other test.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _system(cuda, seed):
    import torch
    from qdsim_b200 import mesh as Mh, poisson as P
    rng = np.random.default_rng(seed)
    m = Mh.StructuredMesh(1, 48, 16, 240.0, 80.0)
    prob = P.PoissonProblem(m, rng.uniform(10.0, 14.0, m.num_elements), device=cuda)
    nrhs = 3
    rho = 1.6e5 * rng.standard_normal((m.num_nodes, nrhs))
    b = prob.rhs(rho)
    x0 = torch.zeros_like(b)
    x0[torch.from_numpy(prob.right).to(cuda)] = torch.as_tensor(
        rng.uniform(0.0, 1.0, nrhs), device=cuda)
    return prob, b, x0


def _solve(prob, b, x0, static):
    import torch
    from qdsim_b200 import _native as N
    from qdsim_b200.fem import stream_ptr
    L = N.lib()
    n, nrhs = b.shape
    X = x0.clone()
    it, rel = C.c_int32(), C.c_double()
    args = (n, nrhs, N.ptr(prob.fem.d_rowptr), N.ptr(prob.fem.d_col), N.ptr(prob.K), N.ptr(b),
            N.ptr(X), N.ptr(prob.d_fixed), 1e-12, 20000, C.byref(it), C.byref(rel))
    if static:
        st = L.qd_pcg_solve_static(*args, stream_ptr())
    else:
        nb = C.c_size_t()
        N.check(L.qd_pcg_workspace_size(n, nrhs, C.byref(nb)), "ws")
        ws = torch.empty(nb.value, dtype=torch.uint8, device=b.device)
        st = L.qd_pcg_solve(*args, N.ptr(ws), ws.numel(), stream_ptr())
    N.check(st, "pcg")
    return X.cpu().numpy(), it.value, rel.value


def test_static_matches_workspace_entry_two_calls(cuda):
    for seed in (0, 1):          # two calls in a row with different systems
        prob, b, x0 = _system(cuda, seed)
        ref, it_ref, rel_ref = _solve(prob, b, x0, static=False)
        got, it_got, rel_got = _solve(prob, b, x0, static=True)
        err = np.abs(got - ref).max() / np.abs(ref).max()
        assert err < 1e-12, (seed, err)
        assert it_got == it_ref and rel_got <= 1e-12


def test_static_rejects_oversize(cuda):
    import torch
    from qdsim_b200 import _native as N
    from qdsim_b200.fem import stream_ptr
    L = N.lib()
    assert L.qd_pcg_static_scratch_bytes() == 16 << 20
    n, nrhs = 4_000_000, 4
    dummy = torch.zeros(8, dtype=torch.float64, device=cuda)
    idx = torch.zeros(8, dtype=torch.int32, device=cuda)
    it, rel = C.c_int32(), C.c_double()
    st = L.qd_pcg_solve_static(n, nrhs, N.ptr(idx), N.ptr(idx), N.ptr(dummy), N.ptr(dummy),
                               N.ptr(dummy), None, 1e-10, 10, C.byref(it), C.byref(rel),
                               stream_ptr())
    assert st == N.QD_ERR_LIMIT

"""Tensor-core DST preconditioner (qd_dst_precond_apply) vs its numpy
restatement with the same BF16 roundings, and vs the FP64 transform."""
import numpy as np
import pytest

from dst_emul import apply_bf16, apply_exact

pytestmark = pytest.mark.gpu

# (nx, ny): ragged tiles, a 5 x 3 lattice (one 16-row block, one K slab), a
# 600-wide lattice (three TMEM row blocks of 256 + 256 + 96 rows)
SHAPES = [(37, 21), (130, 65), (5, 3), (600, 7)]


@pytest.mark.parametrize("fp32", [0, 1])
def test_dst_apply_matches_restatement(cuda, fp32):
    import ctypes as C
    import torch
    from qdsim_b200 import _native as N, eigen as G, fem as F
    B = 12
    specs = [(nx, ny, 0.7, 0.9, 0.05 + 0.01 * i) for i, (nx, ny) in enumerate(SHAPES)]
    specs.append(None)           # a dot without preconditioner is left unchanged
    rows = [nx * ny for nx, ny in SHAPES] + [50]
    row_off = np.concatenate([[0], np.cumsum(rows)]).astype(np.int32)
    pre = G.DSTPreconditioner(specs, cuda)
    rng = np.random.default_rng(1)
    R = rng.standard_normal((row_off[-1], B))
    dt = torch.float32 if fp32 else torch.float64
    Rd = torch.from_numpy(R).to(cuda, dt).contiguous()
    Out = torch.empty_like(Rd)
    nbytes = C.c_size_t()
    L = N.lib()
    N.check(L.qd_dst_precond_workspace_size(len(specs), N.ptr(row_off), B, N.ptr(pre.desc),
                                            C.byref(nbytes)), "ws")
    ws = torch.empty(nbytes.value, dtype=torch.uint8, device=cuda)
    Out.copy_(Rd)
    N.check(L.qd_dst_precond_apply(len(specs), N.ptr(row_off), B, fp32, N.ptr(pre.desc),
                                   N.ptr(pre.d_mats), N.ptr(Rd), N.ptr(Out), N.ptr(ws),
                                   ws.numel(), F.stream_ptr()), "apply")
    got = Out.double().cpu().numpy()
    Rin = Rd.double().cpu().numpy()
    for d, s in enumerate(specs):
        sl = slice(row_off[d], row_off[d + 1])
        if s is None:
            assert np.array_equal(got[sl], Rin[sl])
            continue
        nx, ny, cx, cy, shift = s   # the descriptor stores cx, cy, shift as float32
        p = [float(np.float32(v)) for v in (cx, cy, shift)]
        emu = apply_bf16(Rin[sl], nx, ny, *p)
        ref = apply_exact(Rin[sl], nx, ny, *p)
        e_emu = np.linalg.norm(got[sl] - emu) / np.linalg.norm(emu)
        e_ref = np.linalg.norm(got[sl] - ref) / np.linalg.norm(ref)
        # FP32 accumulation order differs from the restatement's: rare 1-ulp
        # BF16 rounding flips in the intermediates, ~1e-4 in norm
        assert e_emu < 1e-3, (d, e_emu)
        # BF16 operands: ~5e-3 relative to the exact transform
        assert e_ref < 1e-2, (d, e_ref)


def test_dst_apply_in_place(cuda):
    """W <- T W with in == out (the solver's use) equals the out-of-place result."""
    import ctypes as C
    import torch
    from qdsim_b200 import _native as N, eigen as G, fem as F
    B = 8
    specs = [(63, 40, 1.1, 0.4, 0.02)]
    row_off = np.array([0, 63 * 40], np.int32)
    pre = G.DSTPreconditioner(specs, cuda)
    R = torch.randn(63 * 40, B, dtype=torch.float32, device=cuda)
    nbytes = C.c_size_t()
    L = N.lib()
    N.check(L.qd_dst_precond_workspace_size(1, N.ptr(row_off), B, N.ptr(pre.desc),
                                            C.byref(nbytes)), "ws")
    ws = torch.empty(nbytes.value, dtype=torch.uint8, device=cuda)
    out = torch.empty_like(R)
    N.check(L.qd_dst_precond_apply(1, N.ptr(row_off), B, 1, N.ptr(pre.desc), N.ptr(pre.d_mats),
                                   N.ptr(R), N.ptr(out), N.ptr(ws), ws.numel(),
                                   F.stream_ptr()), "apply")
    W = R.clone()
    N.check(L.qd_dst_precond_apply(1, N.ptr(row_off), B, 1, N.ptr(pre.desc), N.ptr(pre.d_mats),
                                   N.ptr(W), N.ptr(W), N.ptr(ws), ws.numel(),
                                   F.stream_ptr()), "apply")
    assert torch.equal(W, out)

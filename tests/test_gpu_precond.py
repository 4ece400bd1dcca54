"""DST preconditioner kernels vs scipy's fast sine transform."""
import numpy as np
import pytest
import scipy.fft as fft

pytestmark = pytest.mark.gpu


def _ref_apply(R, nx, ny, cx, cy, shift):
    kx = np.arange(1, nx + 1)
    ky = np.arange(1, ny + 1)
    lam = (cx * 4 * np.sin(np.pi * kx / (2 * (nx + 1)))[None, :] ** 2
           + cy * 4 * np.sin(np.pi * ky / (2 * (ny + 1)))[:, None] ** 2 + shift)
    out = np.empty_like(R)
    for j in range(R.shape[1]):
        g = R[:, j].reshape(ny, nx)
        out[:, j] = fft.idstn(fft.dstn(g, type=1, norm="ortho") / lam, type=1, norm="ortho").ravel()
    return out


@pytest.mark.parametrize("fp32", [0, 1])
def test_dst_apply_matches_scipy(cuda, fp32):
    import ctypes as C
    import torch
    from qdsim_b200 import _native as N, eigen as G, fem as F
    shapes = [(37, 21), (130, 65), (5, 3)]
    B = 12
    specs = [(nx, ny, 0.7, 0.9, 0.05 + 0.01 * i) for i, (nx, ny) in enumerate(shapes)]
    specs.append(None)           # a dot without preconditioner is left unchanged
    rows = [nx * ny for nx, ny in shapes] + [50]
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
        ref = _ref_apply(Rin[sl], nx, ny, *(float(np.float32(v)) for v in (cx, cy, shift)))
        err = np.abs(got[sl] - ref).max() / np.abs(ref).max()
        assert err < (2e-5 if fp32 else 1e-12), (d, err)

"""libqdsim_b200.so loads, exports every entry point include/qdsim_b200.h
declares, and validates arguments on the host (no GPU compute here)."""
import ctypes as C
import os
import re

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    txt = open(os.path.join(ROOT, "include", "qdsim_b200.h")).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(qd_[a-z0-9_]+)\s*\(", txt)))


def test_library_exports_all_declared_symbols():
    from qdsim_b200 import _native as N
    L = N.lib()
    names = _declared()
    assert len(names) >= 15
    for name in names:
        assert hasattr(L, name), name
        assert name in N.SIGNATURES, f"{name} has no ctypes signature"


def test_status_strings_and_version():
    from qdsim_b200 import _native as N
    L = N.lib()
    assert b"sm_100a" in L.qd_version()
    for st in (0, -1, -2, -3, -4, -5, -6, -7, -8):
        assert L.qd_status_string(st) and L.qd_status_string(st) != b"unknown status"


def test_invalid_arguments_rejected_without_gpu():
    from qdsim_b200 import _native as N
    L = N.lib()
    assert L.qd_assemble(4, 0, 10, 10, 5, *([None] * 16)) == N.QD_ERR_INVALID
    assert L.qd_assemble(2, N.QD_ASM_REF_FIXED, 10, 10, 5, *([None] * 16)) == N.QD_ERR_INVALID
    out = C.c_size_t()
    assert L.qd_lobpcg_workspace_size(1, 100, 900, 3, 0, None, None, C.byref(out)) == N.QD_ERR_INVALID
    assert L.qd_lobpcg_workspace_size(1, 100, 0, 12, 0, None, None, C.byref(out)) == N.QD_ERR_INVALID
    assert L.qd_lobpcg_workspace_size(1, 100, 900, 12, 0, None, None, C.byref(out)) == N.QD_OK
    assert out.value > 9 * 100 * 12 * 8
    fp64 = out.value
    # mixed precision: nine FP32 vector blocks, three FP64 ones (X, HX, MX) and
    # the FP32 (H, M) pairs instead of nine FP64 blocks
    assert L.qd_lobpcg_workspace_size(1, 100, 900, 12, 1, None, None, C.byref(out)) == N.QD_OK
    assert out.value >= fp64 - 6 * 100 * 12 * 8 + 9 * 100 * 12 * 4 + 900 * 8
    assert L.qd_pcg_workspace_size(100, 300, C.byref(out)) == N.QD_ERR_INVALID
    ro = np.array([0, 5], np.int32)
    info = np.zeros(4, np.int32)
    # n must exceed the block size
    assert L.qd_lobpcg_solve(1, N.ptr(ro), None, *([C.c_void_p(8)] * 4), None, None, 4, 8, 0,
                             1e-9, 10, 1, *([C.c_void_p(8)] * 4), N.ptr(info), None,
                             C.c_void_p(256), 1 << 20, None, None) == N.QD_ERR_INVALID
    assert L.qd_pcg_solve_static(0, 1, *([None] * 6), 1e-9, 10, None, None, None) == N.QD_ERR_INVALID


@pytest.mark.parametrize("n", [1, 5, 16, 63, 64, 65, 479, 600])
def test_dst_matrix_layout(n):
    """qd_dst_matrix_fill writes the BF16-rounded DST-I matrix in the
    tensor-core operand layout: undo the layout and compare element-wise."""
    from dst_emul import bf16, dst_matrix
    from qdsim_b200 import eigen as G
    m = G.dst_matrix_bf16(n)
    R, KS = (n + 15) // 16 * 16, (n + 63) // 64
    assert m.size == R * KS * 64
    full = np.zeros((R, KS * 64))
    pos = 0
    for m0 in range(0, R, 256):
        rows = min(256, R - m0)
        blk = m[pos:pos + rows * KS * 64].astype(np.uint32) << 16
        blk = blk.view(np.float32).astype(np.float64)
        # [slab][chunk][row group][row in group][k in chunk]
        a = blk.reshape(KS, 8, rows // 8, 8, 8).transpose(2, 3, 0, 1, 4)
        full[m0:m0 + rows] = a.reshape(rows, KS * 64)
        pos += rows * KS * 64
    want = np.zeros_like(full)
    want[:n, :n] = bf16(dst_matrix(n))
    # the fill reduces the sine's angle exactly (exact zeros where numpy's
    # sine leaves ~1e-16); a BF16 tie may round apart
    ulp = np.abs(want) * 2.0 ** -7 + 1e-12
    assert np.all(np.abs(full - want) <= ulp)
    assert np.mean(np.abs(full - want) <= 1e-12) > 0.999


@pytest.mark.parametrize("order", [1, 2, 3])
def test_pattern_builder_matches_oracle(order):
    from oracle import fem as O
    from qdsim_b200 import fem as F, mesh as Mh
    for nx, ny, dirichlet in ((5, 4, True), (9, 3, False), (1, 1, False)):
        m = Mh.StructuredMesh(order, nx, ny, float(nx), float(ny))
        om = O.structured_mesh(order, nx, ny, float(nx), float(ny))
        dm, n = F.dof_map_for(m, dirichlet)
        if n == 0:
            continue
        P = F.build_pattern(m.elems, dm, n, m.num_nodes)
        ip, ind, slot = O.csr_pattern(om.elems, O.dof_map(om, dirichlet), n)
        assert np.array_equal(P.rowptr, ip) and np.array_equal(P.col, ind)
        assert P.cptr[-1] == (slot >= 0).sum() == P.slotcnt.sum()
        # every row's contribution list covers each of its slots
        for r in range(0, n, max(1, n // 7)):
            L = P.rowptr[r + 1] - P.rowptr[r]
            assert (P.slotcnt[P.rowptr[r]:P.rowptr[r + 1]] > 0).all() and L > 0


def test_pattern_builder_rejects_bad_input():
    from qdsim_b200 import _native as N
    L = N.lib()
    elems = np.array([[0, 1, 7]], np.int32)      # node 7 out of range
    dm = np.arange(3, dtype=np.int32)
    nnz = C.c_int64()
    st = L.qd_pattern_build(3, 1, 3, N.ptr(elems), N.ptr(dm), 3, C.byref(nnz), None, None,
                            *([None] * 7))
    assert st == N.QD_ERR_INVALID


def test_node_adjacency_counts():
    from qdsim_b200 import fem as F, mesh as Mh
    m = Mh.StructuredMesh(2, 4, 3, 4.0, 3.0)
    ptr, adj = F.node_adjacency(m.elems, m.num_nodes)
    assert ptr[-1] == m.elems.size
    for g in (0, 5, m.num_nodes // 2):
        for packed in adj[ptr[g]:ptr[g + 1]]:
            assert m.elems[packed >> 4, packed & 15] == g


def test_open_system_and_dst_entry_points_reject_bad_arguments_without_gpu():
    """Argument checks of qd_cap_spmm and qd_dst_precond_apply return before
    any device work."""
    from qdsim_b200 import _native as N
    L = N.lib()
    p = C.c_void_p(256)   # never dereferenced: every call below is rejected or empty
    s = None

    def cap(n, b, ldx, ldy, rowptr, col, H, M, X, AX, MX):
        return L.qd_cap_spmm(n, b, 0, rowptr, col, H, None, M, X, ldx, AX, MX, ldy, s)

    full = (p, p, p, p, p, p, p)
    assert cap(10, 0, 4, 4, *full) == N.QD_ERR_INVALID       # b < 1
    assert cap(10, 65, 65, 65, *full) == N.QD_ERR_INVALID    # b > 64
    assert cap(10, 8, 4, 8, *full) == N.QD_ERR_INVALID       # ldx < b
    assert cap(10, 8, 8, 4, *full) == N.QD_ERR_INVALID       # ldy < b
    assert cap(10, 8, 8, 8, None, *full[1:]) == N.QD_ERR_INVALID
    assert cap(0, 8, 8, 8, *full) == N.QD_OK                  # nothing to do
    desc = np.zeros(1, dtype=N.DST_PREC_DTYPE)
    desc[0] = (4, 3, 0, 0, 1.0, 1.0, 0.1, 0)
    ro = np.array([0, 12], np.int32)
    apply = lambda b, din: L.qd_dst_precond_apply(1, N.ptr(ro), b, 1, N.ptr(desc), p, din, p, p,
                                                  1 << 20, s)
    assert apply(5, p) == N.QD_ERR_INVALID                    # odd column count
    assert apply(2, p) == N.QD_ERR_INVALID                    # fewer than 4 columns
    assert apply(4, C.c_void_p(264)) == N.QD_ERR_INVALID      # vectors not 16-byte aligned

"""ctypes binding of ``libqdsim_b200.so`` (declarations in ``include/qdsim_b200.h``).

The library is built in-tree by ``qdsim_b200.build``.  There is no fallback:
if the library is missing or cannot be loaded every entry point raises.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

_LIB_PATH = Path(__file__).resolve().parent / "libqdsim_b200.so"

QD_OK = 0
QD_ERR_INVALID = -1
QD_ERR_CUDA = -2
QD_ERR_NOT_CONVERGED = -3
QD_ERR_BREAKDOWN = -4
QD_ERR_WORKSPACE = -5
QD_ERR_DEGENERATE = -6
QD_ERR_LIMIT = -7
QD_ERR_TIMEOUT = -8

QD_ASM_FEM = 0
QD_ASM_REF_CYTHON = 1
QD_ASM_REF_FIXED = 2
QD_ASM_REF_CPP = 3

QD_PREC_FP64 = 0
QD_PREC_MIXED = 1

_p = C.c_void_p
_i32 = C.c_int32
_i64 = C.c_int64
_int = C.c_int
_dbl = C.c_double
_u64 = C.c_uint64
_sz = C.c_size_t

# name -> (restype, argtypes)
SIGNATURES = {
    "qd_version": (C.c_char_p, []),
    "qd_status_string": (C.c_char_p, [_int]),
    "qd_kernel_launch_count": (_u64, []),
    "qd_pattern_build": (_int, [_i64, _i64, _int, _p, _p, _i32, _p, _p, _p,
                                _p, _p, _p, _p, _p, _p, _p]),
    "qd_node_adjacency": (_int, [_i64, _i64, _int, _p, _p, _p, _p]),
    "qd_assemble": (_int, [_int, _int, _i64, _i64, _i32, _p, _p, _p, _p, _p,
                           _p, _p, _p, _p, _p, _p, _p, _p, _p, _p, _p]),
    "qd_spmm_dual": (_int, [_i32, _int, _int, _p, _p, _p, _p, _p, _p, _p, _p]),
    "qd_lobpcg_workspace_size": (_int, [_i32, _i64, _i64, _int, _int, _p, _p, _p]),
    "qd_lobpcg_solve": (_int, [_i32, _p, _p, _p, _p, _p, _p, _p, _p, _int, _int, _int, _dbl,
                               _int, _u64, _p, _p, _p, _p, _p, _p, _p, _sz, _p, _p]),
    "qd_dst_precond_workspace_size": (_int, [_i32, _p, _int, _p, _p]),
    "qd_dst_precond_apply": (_int, [_i32, _p, _int, _int, _p, _p, _p, _p, _p, _sz, _p]),
    "qd_dst_matrix_size": (_int, [_i32, _p]),
    "qd_dst_matrix_fill": (_int, [_i32, _p]),
    "qd_pcg_workspace_size": (_int, [_i32, _int, _p]),
    "qd_pcg_solve": (_int, [_i32, _int, _p, _p, _p, _p, _p, _p, _dbl, _int, _p, _p,
                            _p, _sz, _p]),
    "qd_pcg_static_scratch_bytes": (_sz, []),
    "qd_pcg_solve_static": (_int, [_i32, _int, _p, _p, _p, _p, _p, _p, _dbl, _int, _p, _p, _p]),
    "qd_csr_spmv": (_int, [_i32, _int, _p, _p, _p, _p, _p, _dbl, _p]),
    "qd_cap_spmm": (_int, [_i32, _int, _int, _p, _p, _p, _p, _p, _p, _int, _p, _p, _int, _p]),
    "qd_fe_interpolate": (_int, [_int, _i32, _i32, _dbl, _dbl, _int, _i64, _p, _i64, _p, _p,
                                 _p, _p, _p, _p, _int, _p]),
    "qd_bounded_wait_selftest": (_int, [_i64, _p, _int, _p, _p, _p]),
    "qd_fe_interpolate_tri": (_int, [_int, _i64, _i64, _p, _p, _i32, _i32, _dbl, _dbl, _p, _p,
                                     _p, _p, _int, _i64, _p, _i64, _p, _p, _p, _p, _p, _p, _int,
                                     _p]),
    "qd_prof_enable": (_int, [_int]),
    "qd_prof_read": (_int, [_p, _p, _int]),
    "qd_sc_potential": (_int, [_i32, _i64, _p, _p, _p, _p]),
    "qd_sc_density": (_int, [_i32, _i64, _int, _i64, _p, _p, _p, _dbl, _dbl, _dbl, _p, _p, _p,
                             _p, _p]),
    "qd_sc_mix": (_int, [_i32, _i64, _int, _int, _p, _p, _p, _p, _p, _p, _p, _p, _p]),
    "qd_adjoint": (_int, [_int, _i64, _i64, _int, _int, _p, _p, _p, _p, _p, _p, _p,
                          _p, _p, _p, _p]),
    "qd_cap_lobpcg_workspace_size": (_int, [_i32, _int, _int, _p, _p]),
    "qd_cap_lobpcg_solve": (_int, [_i32, _p, _p, _p, _p, _p, _p, _p, _p, _p, _p, _int, _int, _int,
                                   _dbl, _dbl, _dbl, _int, _int, _dbl, _u64, _p, _p, _p, _p, _p,
                                   _p, _sz, _p]),
    "qd_complex_schur": (_int, [_int, _p, _int, _p, _p, _int, _int, _p, _p]),
}


# struct qd_dst_prec (include/qdsim_b200.h)
import numpy as _np  # noqa: E402
DST_PREC_DTYPE = _np.dtype([("nx", _np.int32), ("ny", _np.int32), ("sx_off", _np.int64),
                            ("sy_off", _np.int64), ("cx", _np.float32), ("cy", _np.float32),
                            ("shift", _np.float32), ("pad", _np.int32)], align=True)
assert DST_PREC_DTYPE.itemsize == 40

# struct qd_lobpcg_opts (include/qdsim_b200.h)
LOBPCG_OPTS_DTYPE = _np.dtype([("tol32", _np.float64), ("stag_window", _np.int32),
                               ("graphs", _np.int32), ("x0", _np.uint64),
                               ("eig_scale", _np.float64), ("chunk_rows", _np.int32),
                               ("setup_cached", _np.int32)], align=True)
assert LOBPCG_OPTS_DTYPE.itemsize == 40

# struct qd_cap_info (include/qdsim_b200.h)
CAP_INFO_DTYPE = _np.dtype([("iters_fp32", _np.int32), ("iters_fp64", _np.int32),
                            ("converged", _np.int32), ("selected", _np.int32),
                            ("complete", _np.int32), ("schur_sweeps_max", _np.int32),
                            ("schur_unconverged", _np.int32), ("pad", _np.int32),
                            ("fp32_residual", _np.float64), ("kth_distance", _np.float64),
                            ("unconverged_bound", _np.float64), ("max_residual", _np.float64)],
                           align=True)
assert CAP_INFO_DTYPE.itemsize == 64


class QDError(RuntimeError):
    """A libqdsim_b200 entry point returned a negative status."""

    def __init__(self, status: int, what: str):
        self.status = status
        super().__init__(f"{what}: {status_string(status)} (status {status})")


_lib = None


def lib():
    """Load the library once; raise if it is missing (no CPU fallback)."""
    global _lib
    if _lib is None:
        if not _LIB_PATH.exists():
            raise RuntimeError(
                f"{_LIB_PATH.name} is not built; run `python -m qdsim_b200.build` "
                "(nvcc with sm_100a support is required)")
        L = C.CDLL(str(_LIB_PATH))
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def status_string(status: int) -> str:
    try:
        return lib().qd_status_string(int(status)).decode()
    except Exception:  # library missing while formatting an error
        return "unknown"


def check(status: int, what: str, allow=()):
    if status != QD_OK and status not in allow:
        raise QDError(status, what)
    return status


def ptr(t) -> int | None:
    """Raw pointer of a torch tensor or numpy array (None for None)."""
    if t is None:
        return None
    if hasattr(t, "data_ptr"):
        return t.data_ptr()
    return t.ctypes.data


def launch_count() -> int:
    return int(lib().qd_kernel_launch_count())


def exported_symbols():
    return list(SIGNATURES)

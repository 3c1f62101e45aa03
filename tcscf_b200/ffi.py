"""ctypes bindings of libtcscf_gpu.so (the C ABI declared in include/tcscf_gpu.h).

The library is built in-tree (tcscf_b200/libtcscf_gpu.so); there is no CPU fallback: when the
library is missing or no B200 is present the calls fail loudly.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "libtcscf_gpu.so"

# status codes (tcscf_status)
OK = 0
ERR_INVALID_ARGUMENT = 1
ERR_CUDA = 2
ERR_TIMEOUT = 3
ERR_NONFINITE = 4
ERR_NOT_CONVERGED = 5
ERR_LINALG = 6
ERR_UNSUPPORTED = 7
ERR_NO_DEVICE = 8

K_INV_R12, K_TC_SCALAR_SAME, K_TC_SCALAR_OPPO, K_GRAD_U_SAME, K_GRAD_U_OPPO = range(5)
PREC_FP64, PREC_BF16X3, PREC_TF32 = 0, 1, 2
BASIS_STO, BASIS_OCHI, BASIS_HYDROGEN = 0, 1, 2
MAP_NONE, MAP_LINEAR, MAP_X_OVER_1MX, MAP_TREUTLER_AHLRICHS_M4, MAP_ONE_PLUS_X = range(5)


class Sto(C.Structure):
    _fields_ = [("alpha", C.c_double), ("n", C.c_int32), ("l", C.c_int32), ("m", C.c_int32), ("family", C.c_int32)]


class Ochi(C.Structure):
    _fields_ = [("a", C.c_double), ("a12", C.c_double), ("nterms", C.c_int32), ("pad", C.c_int32),
                ("S", (C.c_int32 * 3) * 8), ("c", (C.c_double * 2) * 8)]


# every symbol include/tcscf_gpu.h declares, with (restype, argtypes)
_P = C.c_void_p
_D = C.POINTER(C.c_double)
_I = C.c_int
_I64 = C.c_int64
SIGNATURES: dict[str, tuple] = {
    "tcscf_ctx_create": (_I, [_I, C.POINTER(_P)]),
    "tcscf_ctx_destroy": (_I, [_P]),
    "tcscf_last_error": (C.c_char_p, [_P]),
    "tcscf_ctx_stream": (_I, [_P, C.POINTER(_P)]),
    "tcscf_selftest_bounded_wait": (_I, [_P, C.c_double]),
    "tcscf_near_coincident_pairs": (_I, [_P, _I, _I, C.POINTER(_I)]),
    "tcscf_synchronize": (_I, [_P]),
    "tcscf_last_timing": (_I, [_P, _D, _D, C.POINTER(_I)]),
    "tcscf_last_potentials": (_I, [_P, _D, _D]),
    "tcscf_grid_radial": (_I, [_I, _I, C.c_double, C.c_double, _D, _D]),
    "tcscf_grid_product": (_I, [_I, _D, _D, _I, _D, _D, _D]),
    "tcscf_grid_qmc": (_I, [_I, _I64, _D, _D, _D]),
    "tcscf_sobol": (_I, [_I, _I64, C.c_uint64, _D]),
    "tcscf_overlap_core_analytic": (_I, [C.POINTER(Sto), _I, _I, _D, _D]),
    "tcscf_set_scf_options": (_I, [_P, _I, _I]),
    "tcscf_load_sto": (_I, [C.c_char_p, C.c_char_p, C.c_char_p, _I, C.POINTER(Sto), _I, C.POINTER(_I)]),
    "tcscf_grid_create": (_I, [_P, _D, _D, _I64, _I, C.POINTER(_I)]),
    "tcscf_grid_destroy": (_I, [_P, _I]),
    "tcscf_grid_set_basis": (_I, [_P, _I, C.POINTER(Sto), _I, _I]),
    "tcscf_grid_basis_values": (_I, [_P, _I, _D, _D]),
    "tcscf_overlap_core_quadrature": (_I, [_P, _I, _I, _D, _D]),
    "tcscf_overlap_core_quadrature_static": (_I, [_P, _I, _I, _D, _D]),
    "tcscf_integrate_all_r1r2": (_I, [_P, _I, _I, _I, _I, C.POINTER(Ochi), _D]),
    "tcscf_three_electron_integrals": (_I, [_P, _I, _I, C.POINTER(Ochi), _D]),
    "tcscf_fock_build_batch": (_I, [_P, _I, C.POINTER(_I), C.POINTER(_I), C.POINTER(_D), C.POINTER(_D), _I, _I, _D, C.POINTER(_D)]),
    "tcscf_tc_fock_build": (_I, [_P, _I, _I, _I, _I, _I, _I, _I, _D, _D, _D, _D, _I, _D, _D, _D, _D]),
    "tcscf_batch_graph_stats": (_I, [_P, C.POINTER(_I), C.POINTER(_I)]),
    "tcscf_set_autotune": (_I, [_P, _I]),
    "tcscf_autotune_stats": (_I, [_P, C.POINTER(_I), C.POINTER(_I), C.POINTER(_I)]),
    "tcscf_autotune_split_candidates": (_I, [C.c_int64, C.c_int64, _I, C.POINTER(_I), _I, C.POINTER(_I)]),
    "tcscf_schedule_items": (_I, [C.c_int64, C.c_int64, _I, _I, _I, C.POINTER(_I), _I, C.POINTER(_I)]),
    "tcscf_tc_compute_q": (_I, [_P, _I, _I, _I, _D, _D, _D]),
    "tcscf_tc_assemble_g": (_I, [_P, _I, _D, _D, _D, _D, _D]),
    "tcscf_tc_scf": (_I, [_P, _I, _I, _I, _I, _I, _D, _D, _I, _I, _I, C.c_double, _I, _D, C.POINTER(_I), _D, _D]),
    "tcscf_compute_F": (_I, [_P, _I, _I, _I, C.POINTER(Ochi), _I, _D, _I, C.POINTER(_I)]),
    "tcscf_compute_V": (_I, [_P, _I, _I, _I, C.POINTER(Ochi), _I, _D, _I, C.POINTER(_I)]),
    "tcscf_tensor_destroy": (_I, [_P, _I]),
    "tcscf_fock_build": (_I, [_P, _I, _I, _I, _D, _D, _I, _I, _D, _D, _D]),
    "tcscf_fock_build_device": (_I, [_P, _I, _I, _I, _P, _P, _I, _I, _P, _P, _P]),
    "tcscf_fock_build_precomputed": (_I, [_P, _I, _I, _I, _D, _D, _I, _D, _D, _D]),
    "tcscf_scf": (_I, [_P, _I, _I, _I, _I, _I, _D, _D, _I, _I, C.c_double, _I, _D, C.POINTER(_I), _D, _D]),
    "tcscf_scf_graph": (_I, [_P, _I, _I, _I, _I, _D, _D, _I, _I, C.c_double, _I, _I, _D, C.POINTER(_I), _D, _D, C.POINTER(_I)]),
}

_lib: C.CDLL | None = None


def lib() -> C.CDLL:
    """Load libtcscf_gpu.so (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise RuntimeError(f"{LIB_PATH} is missing: run `python -m tcscf_b200.build` (no CPU fallback exists)")
        lib_ = C.CDLL(str(LIB_PATH))
        for name, (res, args) in SIGNATURES.items():
            f = getattr(lib_, name)
            f.restype = res
            f.argtypes = args
        _lib = lib_
    return _lib


def dptr(a: np.ndarray | None):
    if a is None:
        return None
    if a.dtype not in (np.float64, np.complex128) or not a.flags.c_contiguous:
        raise TypeError(f"expected a C-contiguous float64 or complex128 array, got {a.dtype} (contiguous={a.flags.c_contiguous})")
    return a.ctypes.data_as(_D)


class TcscfError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"tcscf error {code}: {msg}")
        self.code = code


def check(code: int, ctx=None) -> None:
    if code != OK:
        msg = lib().tcscf_last_error(ctx).decode() if ctx is not None else ""
        raise TcscfError(code, msg)


def sto_array(basis) -> "C.Array":
    """basis: (alpha, n, l, m) Slater-type orbitals, or (alpha, n, l, m, family) with family one of
    BASIS_STO, BASIS_OCHI, BASIS_HYDROGEN (alpha = Z for the hydrogen-like family)."""
    arr = (Sto * len(basis))()
    for i, b in enumerate(basis):
        arr[i].alpha, arr[i].n, arr[i].l, arr[i].m = float(b[0]), int(b[1]), int(b[2]), int(b[3])
        arr[i].family = int(b[4]) if len(b) > 4 else BASIS_STO
    return arr


def ochi_struct(a: float, a12: float, terms) -> Ochi:
    """terms: list of ((i, j, k), c_opposite, c_same)."""
    o = Ochi()
    o.a, o.a12, o.nterms = float(a), float(a12), len(terms)
    for t, (S, c_oppo, c_same) in enumerate(terms):
        for d in range(3):
            o.S[t][d] = int(S[d])
        o.c[t][0], o.c[t][1] = float(c_oppo), float(c_same)
    return o


def autotune_split_candidates(n1: int, n2: int, sms: int = 148) -> list[int]:
    """Candidate r2 split counts of a tensor-path launch over n1 x n2 points (host only, no device)."""
    buf = (C.c_int * 16)()
    n = C.c_int()
    check(lib().tcscf_autotune_split_candidates(int(n1), int(n2), int(sms), buf, 16, C.byref(n)))
    return list(buf[: n.value])


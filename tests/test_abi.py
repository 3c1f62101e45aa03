"""The C ABI library builds, loads without a GPU and exports every entry point include/*.h declares."""
import ctypes as C
import re
from pathlib import Path

import numpy as np
import pytest

from tcscf_b200 import build, ffi

ROOT = Path(__file__).resolve().parent.parent


def declared_functions():
    names = []
    for h in sorted((ROOT / "include").glob("*.h")):
        text = re.sub(r"/\*.*?\*/", "", h.read_text(), flags=re.S)
        names += re.findall(r"^\s*(?:const\s+)?\w+\s*\*?\s*(tcscf_\w+)\s*\(", text, flags=re.M)
    return sorted(set(names))


def test_library_builds_and_exports_every_declared_symbol():
    build.build()
    lib = C.CDLL(str(ffi.LIB_PATH))
    names = declared_functions()
    assert len(names) >= 20
    for n in names:
        assert hasattr(lib, n), n
    # the Python binding covers every declared entry point
    assert set(names) <= set(ffi.SIGNATURES), set(names) - set(ffi.SIGNATURES)


def test_struct_layouts_match_header():
    assert C.sizeof(ffi.Sto) == 24
    assert C.sizeof(ffi.Ochi) == 8 + 8 + 8 + 96 + 128


def test_host_entry_points_validate_arguments():
    lib = ffi.lib()
    u = np.empty(4)
    w = np.empty(4)
    assert lib.tcscf_grid_radial(0, 0, 0.0, 0.0, ffi.dptr(u), ffi.dptr(w)) == ffi.ERR_INVALID_ARGUMENT
    assert lib.tcscf_grid_radial(4, 9, 0.0, 0.0, ffi.dptr(u), ffi.dptr(w)) == ffi.ERR_INVALID_ARGUMENT
    assert lib.tcscf_sobol(4, 10, 1, ffi.dptr(np.empty(40))) == ffi.ERR_INVALID_ARGUMENT
    assert lib.tcscf_grid_qmc(1, 10, ffi.dptr(u), ffi.dptr(u), ffi.dptr(w)) == ffi.ERR_INVALID_ARGUMENT


def test_context_needs_a_device():
    import torch

    if torch.cuda.is_available():
        pytest.skip("a GPU is present; the no-device path is exercised on CPU-only hosts")
    h = C.c_void_p()
    assert ffi.lib().tcscf_ctx_create(0, C.byref(h)) == ffi.ERR_NO_DEVICE
    assert ffi.lib().tcscf_ctx_destroy(None) == ffi.OK


def _context_entry_points():
    """Names of the declared functions whose first parameter is the context."""
    out = []
    for h in sorted((ROOT / "include").glob("*.h")):
        text = re.sub(r"/\*.*?\*/", "", h.read_text(), flags=re.S)
        out += re.findall(r"^\s*(?:const\s+)?\w+\s*\*?\s*(tcscf_\w+)\s*\(\s*tcscf_ctx\s*\*\s*\w+\s*[,)]", text, flags=re.M)
    return sorted(set(out))


def test_every_context_entry_point_rejects_a_null_context():
    # the reference aborts on bad arguments (LVARRAY_ERROR_IF_*); the C ABI returns a status
    # instead, and a null context is refused before any device call, so this runs without a GPU
    lib = ffi.lib()
    names = _context_entry_points()
    assert len(names) >= 30
    assert set(names) <= set(ffi.SIGNATURES), set(names) - set(ffi.SIGNATURES)
    for n in names:
        res, argtypes = ffi.SIGNATURES[n]
        args = [None] + [0.0 if t is C.c_double else (0 if t in (C.c_int, C.c_int32, C.c_int64, C.c_uint64) else None)
                         for t in argtypes[1:]]
        r = getattr(lib, n)(*args)
        if n == "tcscf_ctx_destroy":
            assert r == ffi.OK
        elif n == "tcscf_last_error":
            assert r == b"null context"
        else:
            assert r == ffi.ERR_INVALID_ARGUMENT, n

"""Fixed-scratch S/H quadrature (tcscf_overlap_core_quadrature_static) through the C ABI.

The entry point allocates nothing: its block results live in a 2 MiB device array shared by every
call on the device, whose address the context looked up when it was created.  It must return what
the allocating entry point returns, on consecutive calls (the shared array is reused) and after
whatever the other test files left on the device, and the device's free memory must not drop
across its calls.
"""
import numpy as np
import pytest
import torch

from tcscf_b200 import api, ffi, grids
from tcscf_b200 import basis as wl

pytestmark = pytest.mark.gpu

# same kernel and summation order on both paths: identical up to launch-order effects (none)
TOL = 1e-13


def _rotated_grid(nrad, order):
    # a rotated product grid keeps every point off the z axis, where the gradient of an m != 0
    # function is not finite
    from scipy.spatial.transform import Rotation

    g = grids.product_grid(nrad, order)
    R = Rotation.from_euler("zyx", [0.3, 0.2, 0.1]).as_matrix()
    return grids.QuadratureGrid(np.ascontiguousarray(R @ g.points), g.weights)


def _allocating(lib, ctx, G, Z, nb):
    S = np.empty((nb, nb), dtype=np.complex128)
    H = np.empty((nb, nb), dtype=np.complex128)
    ffi.check(lib.tcscf_overlap_core_quadrature(ctx.handle, G.id, Z, ffi.dptr(S), ffi.dptr(H)), ctx.handle)
    return S, H


def _static(lib, ctx, G, Z, nb, with_h=True):
    S = np.full((nb, nb), np.nan, dtype=np.complex128)
    H = np.full((nb, nb), np.nan, dtype=np.complex128) if with_h else None
    ffi.check(lib.tcscf_overlap_core_quadrature_static(ctx.handle, G.id, Z, ffi.dptr(S), ffi.dptr(H)), ctx.handle)
    return S, H


def test_static_scratch_matches_allocating_entry_point(ctx):
    lib = ffi.lib()
    w = wl.ne()
    g = _rotated_grid(30, 17)
    G = api.QMCGrid(ctx, g)
    G.setBasisFunctions(w.basis, storeGradients=True)
    S0, H0 = _allocating(lib, ctx, G, w.Z, w.nb)
    assert np.isfinite(S0).all() and np.isfinite(H0).all()
    scale_s, scale_h = np.abs(S0).max(), np.abs(H0).max()
    free0 = torch.cuda.mem_get_info(0)[0]
    for _ in range(2):  # two calls in a row share the fixed array
        S1, H1 = _static(lib, ctx, G, w.Z, w.nb)
        assert np.abs(S1 - S0).max() <= TOL * scale_s
        assert np.abs(H1 - H0).max() <= TOL * scale_h
    # no device allocation: free memory cannot have dropped (a pool may only have returned memory)
    assert torch.cuda.mem_get_info(0)[0] >= free0


def test_static_scratch_smaller_basis_then_s_only(ctx):
    # a second grid and basis size reuse the same array; an S-only call (H NULL) returns the same S
    lib = ffi.lib()
    w = wl.he()
    g = _rotated_grid(w.nrad, w.order)
    G = api.QMCGrid(ctx, g)
    G.setBasisFunctions(w.basis, storeGradients=True)
    S0, H0 = _allocating(lib, ctx, G, w.Z, w.nb)
    S1, H1 = _static(lib, ctx, G, w.Z, w.nb)
    assert np.abs(S1 - S0).max() <= TOL * np.abs(S0).max()
    assert np.abs(H1 - H0).max() <= TOL * np.abs(H0).max()
    free0 = torch.cuda.mem_get_info(0)[0]
    S2, H2 = _static(lib, ctx, G, w.Z, w.nb, with_h=False)
    assert H2 is None
    assert np.abs(S2 - S0).max() <= TOL * np.abs(S0).max()
    assert torch.cuda.mem_get_info(0)[0] >= free0


def test_static_scratch_rejects_basis_beyond_limit(ctx):
    # 257 functions exceed the fixed array (nb <= 256): rejected before any launch
    lib = ffi.lib()
    basis = [(0.5 + 0.01 * k, 1, 0, 0) for k in range(257)]
    g = grids.product_grid(4, 7)
    G = api.QMCGrid(ctx, g)
    G.setBasisFunctions(basis, storeGradients=True)
    S = np.empty((257, 257), dtype=np.complex128)
    code = lib.tcscf_overlap_core_quadrature_static(ctx.handle, G.id, 2, ffi.dptr(S), None)
    assert code == ffi.ERR_UNSUPPORTED
    assert b"256" in lib.tcscf_last_error(ctx.handle)

"""Near-coincident pairs: the tensor-core paths follow the FP64 rule that only an exactly coincident pair
contributes 0 (the reference's r12Inv convention, IntegrationTest.cpp:298-309; HartreeFockTest.cpp:248-253
evaluates distinct grids without a guard).

Two distinct grids are built so that some r2 points sit within FP32 rounding of r1 points (relative
separations 1e-9 and 1e-6, below what FP32 coordinates resolve, 2^-16 |r1|) and others coincide
exactly.  The library finds the near pairs (tcscf_near_coincident_pairs) and the split-BF16 and TF32
builds then agree with the FP64 build, whose result those pairs dominate, within the tensor paths' usual
tolerances; the same holds for the tensor-core precompute form (computeF, 1/r12 and the TC scalar
kernel).  Without near pairs (one grid against itself) the list is empty.
"""
import numpy as np
import pytest

from tcscf_b200 import api, ffi, grids
from tcscf_b200 import basis as wl

pytestmark = pytest.mark.gpu


def _near_grids():
    w = wl.he()
    g = grids.product_grid(w.nrad, w.order)
    rng = np.random.default_rng(21)
    idx = np.sort(rng.choice(g.n, 400, replace=False))
    g1 = grids.subset(g, idx)
    # r2: a different product grid (radial 43, Lebedev 13), plus 6 points 1e-9 and 6 points 1e-6 (relative)
    # away from r1 points, plus 4 r1 points copied exactly
    h = grids.product_grid(43, 13)
    near9 = g1.points[:, :6] * (1 + 1e-9)
    near6 = g1.points[:, 6:12] * (1 + 1e-6)
    exact = g1.points[:, 12:16]
    pts = np.ascontiguousarray(np.concatenate([h.points, near9, near6, exact], axis=1))
    wts = np.concatenate([h.weights, np.full(16, h.weights.mean())])
    return w, g1, grids.QuadratureGrid(pts, wts)


def test_near_pairs_are_found_and_the_tensor_builds_follow_fp64(ctx):
    w, g1, g2 = _near_grids()
    G1 = api.QMCGrid(ctx, g1)
    G1.setBasisFunctions(w.basis)
    G2 = api.QMCGrid(ctx, g2)
    G2.setBasisFunctions(w.basis)
    assert G1.nearCoincidentPairs(G2) == 12           # the 4 exact copies are coincident, not near
    assert G1.nearCoincidentPairs(G1) == 0
    _, h = api.overlap_core(w.basis, w.Z)
    C = np.random.default_rng(22).normal(size=(w.nb, 1)) * 0.3
    D = (C @ C.T).astype(np.complex128)
    G64, _, E64 = api.fock_build(G1, G2, D, h, precision=ffi.PREC_FP64)
    scale = np.abs(G64).max()
    for prec, tol in ((ffi.PREC_BF16X3, 1e-6), (ffi.PREC_TF32, 2e-4)):
        Gm, _, Em = api.fock_build(G1, G2, D, h, precision=prec)
        assert np.abs(Gm - G64).max() <= tol * scale, (prec, np.abs(Gm - G64).max() / scale)
        assert abs(Em - E64) <= tol * abs(E64), (prec, Em, E64)
    G1.close()
    G2.close()


def test_near_pairs_in_the_tensor_core_precompute_form(ctx):
    w, g1, g2 = _near_grids()
    G1 = api.QMCGrid(ctx, g1)
    G1.setBasisFunctions(w.basis)
    G2 = api.QMCGrid(ctx, g2)
    G2.setBasisFunctions(w.basis)
    u = ffi.ochi_struct(1.0, 1.0, [((1, 0, 0), -0.5, -0.25)])
    for kern, jas in ((ffi.K_INV_R12, None), (ffi.K_TC_SCALAR_OPPO, u)):
        a = api.computeF(G1, G2, kern, jas, precision=ffi.PREC_BF16X3)
        b = api.computeF(G1, G2, kern, jas)
        assert np.abs(a - b).max() <= 2e-6 * np.abs(b).max(), kern
    G1.close()
    G2.close()

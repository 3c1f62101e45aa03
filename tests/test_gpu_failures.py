"""Failure detection on the device, with every failure made on the host or by a wait that runs out.

The reference's failure surface is an exception: ConvergenceError after the iteration limit
(HartreeFock.hpp:13-19), LvArray::dense::Error from a failed eigen-solve, which its driver maps to
+max and retries (HartreeFockTest.cpp:413-430).  Here every C-ABI call returns a status instead:

* a bounded device wait that nothing completes gives up after its limit and the call returns
  TCSCF_ERR_TIMEOUT, after which the same context still builds correctly;
* a non-finite grid point propagates to a non-finite energy, reported as TCSCF_ERR_NONFINITE by
  both the FP64 and the tensor-core build;
* a zero-weight grid gives a zero quadrature overlap, and that overlap or one with a zero-norm
  function makes the generalized eigen-solve fail: TCSCF_ERR_LINALG;
* an iteration limit that is too small: TCSCF_ERR_NOT_CONVERGED (ConvergenceError).
No test faults, traps or hangs the GPU: the inputs are ordinary finite-size arrays and the only
device wait that expires is bounded (20 ms).
"""
import numpy as np
import pytest

from tcscf_b200 import api, ffi, grids
from tcscf_b200 import basis as wl

pytestmark = pytest.mark.gpu


def _he_build(ctx, precision):
    w = wl.he()
    g = grids.product_grid(w.nrad, w.order)
    rng = np.random.default_rng(3)
    g1 = grids.subset(g, rng.choice(g.n, 256, replace=False))
    _, h = api.overlap_core(w.basis, w.Z)
    C = rng.normal(size=(w.nb, 1)) * 0.3
    D = (C @ C.T).astype(np.complex128)
    G1 = api.QMCGrid(ctx, g1)
    G1.setBasisFunctions(w.basis)
    G2 = api.QMCGrid(ctx, g)
    G2.setBasisFunctions(w.basis)
    try:
        return api.fock_build(G1, G2, D, h, precision=precision)
    finally:
        G1.close()
        G2.close()


def test_bounded_wait_gives_up_and_the_context_stays_usable(ctx):
    before = _he_build(ctx, ffi.PREC_BF16X3)
    code = ffi.lib().tcscf_selftest_bounded_wait(ctx.handle, 20.0)
    assert code == ffi.ERR_TIMEOUT
    assert b"bounded wait expired" in ffi.lib().tcscf_last_error(ctx.handle)
    # the same context: a tensor-core build (whose kernel uses the same waits) and an FP64 build
    after = _he_build(ctx, ffi.PREC_BF16X3)
    assert after[2] == before[2]
    np.testing.assert_array_equal(after[0], before[0])
    e64 = _he_build(ctx, ffi.PREC_FP64)[2]
    assert abs(e64 - after[2]) < 1e-6


def test_bounded_wait_limit_is_checked(ctx):
    assert ffi.lib().tcscf_selftest_bounded_wait(ctx.handle, 0.0) == ffi.ERR_INVALID_ARGUMENT
    assert ffi.lib().tcscf_selftest_bounded_wait(ctx.handle, 5000.0) == ffi.ERR_INVALID_ARGUMENT


@pytest.mark.parametrize("precision", [ffi.PREC_FP64, ffi.PREC_BF16X3])
def test_nonfinite_point_is_reported(ctx, precision):
    w = wl.he()
    g = grids.product_grid(w.nrad, w.order)
    pts = g.points.copy()
    pts[0, 17] = np.nan
    bad = grids.QuadratureGrid(pts, g.weights.copy())
    _, h = api.overlap_core(w.basis, w.Z)
    C = np.random.default_rng(4).normal(size=(w.nb, 1)) * 0.3
    D = (C @ C.T).astype(np.complex128)
    G = api.QMCGrid(ctx, bad)
    G.setBasisFunctions(w.basis)
    with pytest.raises(ffi.TcscfError) as e:
        api.fock_build(G, G, D, h, precision=precision)
    assert e.value.code == ffi.ERR_NONFINITE
    G.close()
    # the context is still usable
    assert np.isfinite(_he_build(ctx, precision)[2])


def test_zero_weight_grid_and_singular_overlap_fail_the_eigen_solve(ctx):
    w = wl.he()
    g = grids.product_grid(w.nrad, w.order)
    # quadrature S on a grid whose weights are all zero is the zero matrix (the grid is rotated off
    # the z axis, where the gradient of an m != 0 function is not finite)
    from scipy.spatial.transform import Rotation

    rot = Rotation.from_euler("zyx", [0.3, 0.2, 0.1]).as_matrix()
    zero = grids.QuadratureGrid(np.ascontiguousarray(rot @ g.points), np.zeros(g.n))
    Z0 = api.QMCGrid(ctx, zero)
    Z0.setBasisFunctions(w.basis, storeGradients=True)
    S0, H0 = api.overlap_core_quadrature(Z0, w.Z)
    assert np.abs(S0).max() == 0.0 and np.abs(H0).max() == 0.0
    Z0.close()
    G = api.QMCGrid(ctx, g)
    G.setBasisFunctions(w.basis)
    _, h = api.overlap_core(w.basis, w.Z)
    hf = api.RCSHartreeFock(1, 1, w.nb)
    with pytest.raises(api.LinearAlgebraError) as e:
        hf.compute(np.real(S0), h, G, G, precision=ffi.PREC_FP64, tol=1e-8, max_iter=5)
    assert e.value.code == ffi.ERR_LINALG
    # a singular overlap with one zero-norm function (a zero row and column): the Cholesky factor of S
    # inside the generalized eigen-solve meets a zero pivot
    S, _ = api.overlap_core(w.basis, w.Z)
    S[3, :] = 0.0
    S[:, 3] = 0.0
    hf = api.RCSHartreeFock(1, 1, w.nb)
    with pytest.raises(api.LinearAlgebraError):
        hf.compute(S, h, G, G, precision=ffi.PREC_FP64, tol=1e-8, max_iter=5)
    G.close()


def test_iteration_limit_raises_convergence_error(ctx):
    w = wl.he()
    g = grids.product_grid(w.nrad, w.order)
    G = api.QMCGrid(ctx, g)
    G.setBasisFunctions(w.basis)
    S, h = api.overlap_core(w.basis, w.Z)
    hf = api.RCSHartreeFock(1, 1, w.nb)
    with pytest.raises(api.ConvergenceError) as e:
        hf.compute(S, h, G, G, precision=ffi.PREC_FP64, tol=1e-12, max_iter=1)
    assert e.value.code == ffi.ERR_NOT_CONVERGED
    G.close()

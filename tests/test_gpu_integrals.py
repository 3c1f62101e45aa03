"""4- and 6-index r12 tensors (integrateAllR1R2, threeElectronIntegrals) on the GPU vs the oracle.

Both paths are FP64; the GPU sums r2 in the flash contraction and r1 in one GEMM, the oracle in
the reference's loop order, so they agree to rounding (1e-11 of the largest element here).
"""
import numpy as np
import pytest

import oracle
from tcscf_b200 import api, ffi, grids
from tcscf_b200 import basis as wl

pytestmark = pytest.mark.gpu

TOL = 1e-11
U = dict(a=1.0, a12=1.0, terms=[((1, 0, 0), -0.5, -0.25)])   # HartreeFockTest.cpp:351-360 sign convention
BASIS = wl.expand(0, [0.8, 1.9]) + wl.expand(1, [1.3])        # 5 functions: s, s, p(m=-1,0,1)


@pytest.fixture(scope="module")
def grids_12(ctx):
    g1 = grids.qmc_grid(3, 96, 31)
    g2 = grids.qmc_grid(2, 400, 32)
    G1 = api.QMCGrid(ctx, g1)
    G1.setBasisFunctions(BASIS)
    G2 = api.QMCGrid(ctx, g2)
    G2.setBasisFunctions(BASIS, storeGradients=True)
    vals1 = oracle.basis_values(g1.points, BASIS)
    vals2, grads2 = oracle.basis_values(g2.points, BASIS, gradients=True)
    return g1, g2, G1, G2, vals1, vals2, grads2


def _close(a, b):
    np.testing.assert_allclose(a, b, rtol=0, atol=TOL * np.abs(b).max())


@pytest.mark.parametrize("kernel", [ffi.K_INV_R12, ffi.K_TC_SCALAR_SAME])
def test_integrate_all_r1r2_value_form(ctx, grids_12, kernel):
    g1, g2, G1, G2, vals1, vals2, grads2 = grids_12
    u = ffi.ochi_struct(U["a"], U["a12"], U["terms"]) if kernel != ffi.K_INV_R12 else None
    uo = oracle.ochi(U["a"], U["a12"], U["terms"]) if kernel != ffi.K_INV_R12 else None
    got = api.integrateAllR1R2(G1, G2, kernel, u)
    ref = oracle.integrate_all_r1r2(False, g1.points, g1.weights, vals1, g2.points, g2.weights, vals2, None, len(BASIS), kernel, uo)
    _close(got, ref)


def test_integrate_all_r1r2_gradient_form(ctx, grids_12):
    g1, g2, G1, G2, vals1, vals2, grads2 = grids_12
    u = ffi.ochi_struct(U["a"], U["a12"], U["terms"])
    uo = oracle.ochi(U["a"], U["a12"], U["terms"])
    for k in (ffi.K_GRAD_U_SAME, ffi.K_GRAD_U_OPPO):
        got = api.integrateAllR1R2(G1, G2, k, u, use_gradient=True)
        ref = oracle.integrate_all_r1r2(True, g1.points, g1.weights, vals1, g2.points, g2.weights, vals2, grads2, len(BASIS), k, uo)
        _close(got, ref)


def test_three_electron_integrals(ctx):
    basis = wl.expand(0, [0.9]) + wl.expand(1, [1.4])   # 4 functions -> 4^6 outputs
    g1 = grids.qmc_grid(3, 80, 41)
    g2 = grids.qmc_grid(3, 300, 42)
    G1 = api.QMCGrid(ctx, g1)
    G1.setBasisFunctions(basis)
    G2 = api.QMCGrid(ctx, g2)
    G2.setBasisFunctions(basis)
    u = ffi.ochi_struct(U["a"], U["a12"], U["terms"])
    uo = oracle.ochi(U["a"], U["a12"], U["terms"])
    got = api.threeElectronIntegrals(G1, G2, u)
    ref = oracle.three_electron_integrals(g1.points, g1.weights, oracle.basis_values(g1.points, basis), g2.points, g2.weights,
                                          oracle.basis_values(g2.points, basis), len(basis), uo)
    _close(got, ref)


def test_tensor_argument_checks(ctx, grids_12):
    g1, g2, G1, G2, *_ = grids_12
    with pytest.raises(ffi.TcscfError) as e:
        api.integrateAllR1R2(G1, G1, ffi.K_INV_R12)          # r2 must be two dimensional
    assert e.value.code == ffi.ERR_INVALID_ARGUMENT
    with pytest.raises(ffi.TcscfError) as e:
        api.integrateAllR1R2(G1, G2, ffi.K_INV_R12, use_gradient=True)   # gradient form needs a vector kernel
    assert e.value.code == ffi.ERR_INVALID_ARGUMENT

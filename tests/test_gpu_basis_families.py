"""Ochi and hydrogen-like basis families (OchiBasis.hpp, HydrogenLikeBasis.hpp) on the GPU vs the oracle.

Basis values and gradients are FP64 on both sides (the device evaluates the generalised Laguerre
polynomials by their three-term recurrence, the oracle with std::assoc_laguerre as the reference
does): they agree to 1e-12 of the largest magnitude.  Fock builds and SCF with these bases go through
the same kernels as the Slater-type orbitals, with the same bars (FP64 1e-10 Eh, split BF16 1e-8 |E|).
"""
import numpy as np
import pytest

import oracle
from tcscf_b200 import api, ffi, grids
from tcscf_b200 import basis as wl

from .test_gpu_parity import real_density

pytestmark = pytest.mark.gpu

OCHI = wl.ochi_functions(3, 2, 1.7)          # 4 x (1 + 3 + 5) = 36 functions
HYDROGEN = wl.hydrogen_functions(3, 2, 2)    # 1s; 2s 2p; 3s 3p 3d = 14 functions


def _rotated_grid(nrad, order):
    # a rotated product grid keeps every point off the z axis, where the reference's gradient formula
    # (OchiBasis.hpp:76-77) divides by sin(theta) and tan(theta)
    from scipy.spatial.transform import Rotation

    g = grids.product_grid(nrad, order)
    R = Rotation.from_euler("zyx", [0.3, 0.2, 0.1]).as_matrix()
    return grids.QuadratureGrid(np.ascontiguousarray(R @ g.points), g.weights)


@pytest.fixture(scope="module")
def grid(ctx):
    return _rotated_grid(24, 17)


def _close(a, b, rel=1e-12):
    np.testing.assert_allclose(a, b, rtol=0, atol=rel * np.abs(b).max())


def test_ochi_values_and_gradients_match_oracle(ctx, grid):
    G = api.QMCGrid(ctx, grid)
    G.setBasisFunctions(OCHI, storeGradients=True)
    v, gr = oracle.basis_values(grid.points, OCHI, gradients=True)
    _close(G.basisValues, v)
    _close(G.basisGradients, gr)


def test_hydrogen_values_match_oracle_and_gradients_refused(ctx, grid):
    G = api.QMCGrid(ctx, grid)
    G.setBasisFunctions(HYDROGEN)
    _close(G.basisValues, oracle.basis_values(grid.points, HYDROGEN))
    with pytest.raises(ffi.TcscfError) as e:
        G.setBasisFunctions(HYDROGEN, storeGradients=True)    # the reference has no hydrogen-like gradient
    assert e.value.code == ffi.ERR_UNSUPPORTED
    with pytest.raises(ffi.TcscfError) as e:
        G.setBasisFunctions(OCHI[:1] + HYDROGEN[:1])         # one family per basis
    assert e.value.code == ffi.ERR_INVALID_ARGUMENT


def test_ochi_quadrature_overlap_core_matches_analytic(ctx):
    # S and H by quadrature of the device values and gradients on a fine product grid against the
    # orthonormal overlap and the reference's radial core formula
    b = wl.ochi_functions(3, 1, 1.7)
    G = api.QMCGrid(ctx, _rotated_grid(120, 17))
    G.setBasisFunctions(b, storeGradients=True)
    Sq, Hq = api.overlap_core_quadrature(G, 2)
    S, H = api.overlap_core(b, 2)
    np.testing.assert_allclose(Sq.real, S, atol=1e-9)
    # H from the gradients: the functions with m >= 0 (the reference's gradient formula, shared with
    # the STOs, is not the derivative for m < 0, SlaterTypeOrbital.hpp:73-75 / OchiBasis.hpp:74-76)
    keep = [i for i, f in enumerate(b) if f[3] >= 0]
    np.testing.assert_allclose(Hq.real[np.ix_(keep, keep)], H[np.ix_(keep, keep)], atol=1e-6)


@pytest.mark.parametrize("basis", [OCHI, HYDROGEN], ids=["ochi", "hydrogen"])
def test_family_fock_builds(ctx, grid, basis):
    G = api.QMCGrid(ctx, grid)
    G.setBasisFunctions(basis)
    S, h = api.overlap_core(basis, 2)
    D = real_density(basis, 2, np.random.default_rng(31))
    vals = oracle.basis_values(grid.points, basis)
    F = oracle.compute_F(grid.points, grid.points, grid.weights, vals, len(basis))
    Gr, Fr, Er = oracle.fock_build(F, vals, grid.weights, D, h)
    Gd, Fd, Ed = api.fock_build(G, G, D, h, precision=ffi.PREC_FP64)
    assert abs(Ed - Er) < 1e-10 * max(1.0, abs(Er)), (Ed, Er)
    np.testing.assert_allclose(Gd, Gr, rtol=0, atol=1e-10 * np.abs(Gr).max())
    # split BF16: the Fock matrix to 1e-6 of its largest element and the energy to 1e-8 Eh (the
    # hydrogen-like case's energy is a near-cancelling 4e-3 Eh, so the bar is absolute)
    Gm, Fm, Em = api.fock_build(G, G, D, h, precision=ffi.PREC_BF16X3)
    assert np.abs(Gm - Gd).max() < 1e-6 * np.abs(Gd).max()
    assert abs(Em - Ed) < 1e-8 * max(1.0, abs(Ed)), (Em, Ed)


def test_he_ochi_scf_matches_oracle(ctx, grid):
    b = wl.ochi_functions(5, 1, 1.9)
    S, h = api.overlap_core(b, 2)
    G = api.QMCGrid(ctx, grid)
    G.setBasisFunctions(b)
    vals = oracle.basis_values(grid.points, b)
    F = oracle.compute_F(grid.points, grid.points, grid.weights, vals, len(b))
    st, Er, itr, Dr, eig = oracle.scf(1, 1, 1, F, vals, grid.weights, S, h, tol=1e-8, max_iter=100)
    assert st == 0
    hf = api.RCSHartreeFock(1, 1, len(b))
    Eg = hf.compute(S, h, G, G, tol=1e-8)
    assert abs(Eg - Er) < 1e-10, (Eg, Er)
    assert -2.95 < Eg < -2.75

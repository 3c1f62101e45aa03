"""The symmetric contractions: with one grid as r1 and r2 and a positive semi-definite real density,
X = g rho is symmetric, so the split-BF16 and FP64 kernels compute only the r2 points on and above each
r1 tile's diagonal (the diagonal tile at half weight), the exchange matrix is sum W T' plus its
transpose, and the Coulomb rows they skip come from row-sum kernels over the points below the
diagonal.  A second grid object with the same points takes the full (unsymmetric) contraction, so the
two are compared on identical inputs, and both against the FP64 build (the reference's convention,
HartreeFock.cpp:144-213 with the r12 pair sum of HartreeFock.hpp:136-180).

Grids whose point count is not a multiple of the 128-point tile or the 64-point block leave partial
tiles; UOS builds take the symmetric path per spin; near-coincident pairs inside one grid are added
back with the weights of their blocks.
"""
import numpy as np
import pytest

from tcscf_b200 import api, ffi, grids
from tcscf_b200 import basis as wl

pytestmark = pytest.mark.gpu

TOL = 1e-6   # split BF16 against FP64, relative to the largest |G| (the tensor tests' bar)


def _real_density(basis, nocc, rng):
    nb = len(basis)
    U = wl.real_harmonic_unitary(basis)
    C = U.T @ (rng.normal(size=(nb, nocc)) * 0.3)
    return C @ C.conj().T


def _twins(ctx, g, basis):
    a = api.QMCGrid(ctx, g)
    a.setBasisFunctions(basis)
    b = api.QMCGrid(ctx, grids.QuadratureGrid(np.array(g.points, copy=True), np.array(g.weights, copy=True)))
    b.setBasisFunctions(basis)
    return a, b


@pytest.mark.parametrize("nrad,order", [(40, 17), (24, 13)])
def test_symmetric_matches_full_and_fp64_ne(ctx, nrad, order):
    w = wl.ne()
    g = grids.product_grid(nrad, order)
    assert g.n % 128 != 0
    G, Gb = _twins(ctx, g, w.basis)
    _, h = api.overlap_core(w.basis, w.Z)
    D = _real_density(w.basis, 5, np.random.default_rng(nrad))
    G64, _, E64 = api.fock_build(G, G, D, h, precision=ffi.PREC_FP64)
    Gs, _, Es = api.fock_build(G, G, D, h, precision=ffi.PREC_BF16X3)     # symmetric contraction
    Gf, _, Ef = api.fock_build(G, Gb, D, h, precision=ffi.PREC_BF16X3)    # two grid objects: full contraction
    scale = np.abs(G64).max()
    assert np.abs(Gs - G64).max() <= TOL * scale, np.abs(Gs - G64).max() / scale
    assert np.abs(Gf - G64).max() <= TOL * scale, np.abs(Gf - G64).max() / scale
    assert np.abs(Gs - Gf).max() <= TOL * scale
    assert abs(Es - E64) <= TOL * abs(E64) and abs(Ef - E64) <= TOL * abs(E64), (Es, Ef, E64)
    # the symmetric G is Hermitian up to rounding, as the FP64 one is
    assert np.abs(Gs - Gs.conj().transpose(0, 2, 1)).max() <= 1e-9 * scale
    # FP64: the symmetric contraction against the full one, to FP64 rounding
    G64f, _, E64f = api.fock_build(G, Gb, D, h, precision=ffi.PREC_FP64)
    assert np.abs(G64 - G64f).max() <= 1e-12 * scale, np.abs(G64 - G64f).max() / scale
    assert abs(E64 - E64f) <= 1e-10, (E64, E64f)
    # TF32 keeps the full contraction on one grid: the same bits as on the twin grid objects
    Gt, _, Et = api.fock_build(G, G, D, h, precision=ffi.PREC_TF32)
    Gtf, _, Etf = api.fock_build(G, Gb, D, h, precision=ffi.PREC_TF32)
    assert Et == Etf
    np.testing.assert_array_equal(Gt, Gtf)
    G.close()
    Gb.close()


def test_symmetric_fp64_kr_basis(ctx):
    # nb = 120, rank 18: the 128 x 128 FP64 tensor-core tile (warp-specialised), symmetric against the
    # full contraction on a grid with a partial last tile
    w = wl.kr()
    g = grids.product_grid(12, 77)
    assert g.n % 128 != 0
    G, Gb = _twins(ctx, g, w.basis)
    _, h = api.overlap_core(w.basis, w.Z)
    D = _real_density(w.basis, 18, np.random.default_rng(3))
    Gs, _, Es = api.fock_build(G, G, D, h, precision=ffi.PREC_FP64)
    Gf, _, Ef = api.fock_build(G, Gb, D, h, precision=ffi.PREC_FP64)
    scale = np.abs(Gf).max()
    assert np.abs(Gs - Gf).max() <= 1e-12 * scale, np.abs(Gs - Gf).max() / scale
    assert abs(Es - Ef) <= 1e-10 * abs(Ef), (Es, Ef)
    G.close()
    Gb.close()


def test_symmetric_uos(ctx):
    w = wl.ne()
    g = grids.product_grid(30, 17)
    G, Gb = _twins(ctx, g, w.basis)
    _, h = api.overlap_core(w.basis, w.Z)
    rng = np.random.default_rng(5)
    D = np.stack([_real_density(w.basis, 3, rng), _real_density(w.basis, 2, rng)])
    G64, _, E64 = api.fock_build(G, G, D, h, precision=ffi.PREC_FP64)
    Gs, _, Es = api.fock_build(G, G, D, h, precision=ffi.PREC_BF16X3)
    Gf, _, Ef = api.fock_build(G, Gb, D, h, precision=ffi.PREC_BF16X3)
    scale = np.abs(G64).max()
    assert np.abs(Gs - G64).max() <= TOL * scale and np.abs(Gf - G64).max() <= TOL * scale
    assert abs(Es - E64) <= TOL * abs(E64), (Es, E64)
    G.close()
    Gb.close()


def test_symmetric_with_near_pairs_inside_one_grid(ctx):
    # one grid holding 6 points 1e-9 and 6 points 1e-6 (relative) away from 12 of its other points: the
    # near list holds each such pair in both orders, added back with the weight of its block
    w = wl.he()
    base = grids.product_grid(w.nrad, w.order)
    rng = np.random.default_rng(31)
    idx = np.sort(rng.choice(base.n, 700, replace=False))
    g0 = grids.subset(base, idx)
    src = rng.choice(g0.n, 12, replace=False)
    near = np.concatenate([g0.points[:, src[:6]] * (1 + 1e-9), g0.points[:, src[6:]] * (1 + 1e-6)], axis=1)
    pts = np.ascontiguousarray(np.concatenate([g0.points, near], axis=1))
    wts = np.concatenate([g0.weights, g0.weights[src]])
    g = grids.QuadratureGrid(pts, wts)
    G, Gb = _twins(ctx, g, w.basis)
    assert G.nearCoincidentPairs(G) == 24
    _, h = api.overlap_core(w.basis, w.Z)
    D = _real_density(w.basis, 1, np.random.default_rng(32))
    G64, _, E64 = api.fock_build(G, G, D, h, precision=ffi.PREC_FP64)
    Gs, _, Es = api.fock_build(G, G, D, h, precision=ffi.PREC_BF16X3)
    Gf, _, Ef = api.fock_build(G, Gb, D, h, precision=ffi.PREC_BF16X3)
    scale = np.abs(G64).max()
    assert np.abs(Gs - G64).max() <= TOL * scale, np.abs(Gs - G64).max() / scale
    assert np.abs(Gf - G64).max() <= TOL * scale, np.abs(Gf - G64).max() / scale
    assert abs(Es - E64) <= TOL * abs(E64), (Es, E64)
    G.close()
    Gb.close()

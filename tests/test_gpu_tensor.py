"""Tensor-core (tcgen05, split-BF16) Fock build vs the FP64 GPU path and the oracle.

Tolerances stated here are the mixed path's accuracy claim on these small cases: energy within
1e-6 Eh of FP64 and every Fock element within 1e-6 of the largest |G| element.
"""
import numpy as np
import pytest

from tcscf_b200 import api, ffi, grids
from tcscf_b200 import basis as wl

from .test_gpu_parity import rand_density, real_density

pytestmark = pytest.mark.gpu

E_TOL_MIXED = 1e-6
G_REL_TOL = 1e-6


@pytest.fixture(scope="module")
def he(ctx):
    w = wl.he()
    g = grids.product_grid(w.nrad, w.order)
    G = api.QMCGrid(ctx, g)
    G.setBasisFunctions(w.basis)
    S, h = api.overlap_core(w.basis, w.Z)
    return w, g, G, h


def _compare(G1, G2, D, h, window=4):
    G1.ctx.set_flush_window(window)
    Gd, Fd, Ed = api.fock_build(G1, G2, D, h, precision=ffi.PREC_FP64)
    Gm, Fm, Em = api.fock_build(G1, G2, D, h, precision=ffi.PREC_BF16X3)
    scale = np.abs(Gd).max()
    return abs(Em - Ed), np.abs(Gm - Gd).max() / scale, Em, Ed


def test_single_tile_matches_fp64(ctx, he):
    w, g, G, h = he
    rng = np.random.default_rng(1)
    g1 = grids.subset(g, np.sort(rng.choice(g.n, 128, replace=False)))
    G1 = api.QMCGrid(ctx, g1)
    G1.setBasisFunctions(w.basis)
    D = real_density(w.basis, 1, rng)
    dE, dG, Em, Ed = _compare(G1, G, D, h)
    assert dE < E_TOL_MIXED, (Em, Ed)
    assert dG < G_REL_TOL


@pytest.mark.parametrize("window", [1, 4, 16])
def test_he_full_grid_flush_windows(ctx, he, window):
    w, g, G, h = he
    rng = np.random.default_rng(2)
    D = real_density(w.basis, 1, rng)
    dE, dG, Em, Ed = _compare(G, G, D, h, window)
    assert dE < E_TOL_MIXED, (window, Em, Ed)
    assert dG < G_REL_TOL


def test_ragged_sizes_complex_density_and_uos(ctx, he):
    # r1 / r2 counts that are not multiples of the 128 x 64 tiles, a density that is complex in the
    # real-harmonic basis (two tensor passes), and the two-spin build
    w, g, G, h = he
    rng = np.random.default_rng(3)
    g1 = grids.subset(g, np.sort(rng.choice(g.n, 333, replace=False)))
    g2 = grids.subset(g, np.sort(rng.choice(g.n, 1999, replace=False)))
    G1 = api.QMCGrid(ctx, g1)
    G1.setBasisFunctions(w.basis)
    G2 = api.QMCGrid(ctx, g2)
    G2.setBasisFunctions(w.basis)
    D = rand_density(w.nb, 2, rng)
    dE, dG, Em, Ed = _compare(G1, G2, D, h)
    assert dE < E_TOL_MIXED and dG < G_REL_TOL, (Em, Ed, dG)
    D2 = np.stack([real_density(w.basis, 2, rng), real_density(w.basis, 1, rng)])
    dE, dG, Em, Ed = _compare(G1, G2, D2, h)
    assert dE < E_TOL_MIXED and dG < G_REL_TOL, (Em, Ed, dG)


def test_ne_subset_accuracy(ctx):
    w = wl.ne()
    g = grids.product_grid(w.nrad, w.order)
    rng = np.random.default_rng(4)
    g1 = grids.subset(g, np.sort(rng.choice(g.n, 2048, replace=False)))
    G1 = api.QMCGrid(ctx, g1)
    G1.setBasisFunctions(w.basis)
    G2 = api.QMCGrid(ctx, g)
    G2.setBasisFunctions(w.basis)
    S, h = api.overlap_core(w.basis, w.Z)
    D = real_density(w.basis, 5, rng)
    dE, dG, Em, Ed = _compare(G1, G2, D, h)
    assert dE < E_TOL_MIXED, (Em, Ed)
    assert dG < G_REL_TOL


def test_tensor_path_rejects_unsupported_shapes(ctx, he):
    w, g, G, h = he
    rng = np.random.default_rng(5)
    # a complex density of rank 20 needs a 40-column factor: beyond the tensor path's rank 32
    D = rand_density(w.nb, 20, rng)
    with pytest.raises(ffi.TcscfError) as e:
        api.fock_build(G, G, D, h, precision=ffi.PREC_BF16X3)
    assert e.value.code == ffi.ERR_UNSUPPORTED

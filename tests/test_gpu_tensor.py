"""Tensor-core (tcgen05) Fock builds, fixed-point split-BF16 and TF32, vs the FP64 GPU path.

Tolerances stated here are the mixed path's accuracy on these cases: the energy within
max(1e-9 Eh, 1e-8 |E|) of FP64 (random test densities give energies of 1e0-1e4 Eh; the measured
relative errors are 4e-12 to 2.3e-9) and every Fock element within 1e-6 of the largest |G| element
(measured up to 1.5e-7).  The errors are the unbiased rounding of the 24-bit / 16-bit fixed-point
operand slices; the tensor-core accumulation itself is exact.
"""
import numpy as np
import pytest

from tcscf_b200 import api, ffi, grids
from tcscf_b200 import basis as wl

from .test_gpu_parity import rand_density, real_density

pytestmark = pytest.mark.gpu

G_REL_TOL = 1e-6
# TF32 (one operand rounding to 10 explicit mantissa bits, FP32 accumulation per 64-point block):
# measured |dE| / |E| 6.5e-6 (He), 6.4e-9 (Ne), 3.0e-7 (Kr, 406,000 points) and Fock elements within
# 1e-5 to 1.2e-4 of the largest |G| element (Kr basis on 660 to 406,000 points)
TF32_E_REL_TOL = 3e-5
TF32_G_REL_TOL = 3e-4


def e_tol(E):
    return max(1e-9, 1e-8 * abs(E))


@pytest.fixture(scope="module")
def he(ctx):
    w = wl.he()
    g = grids.product_grid(w.nrad, w.order)
    G = api.QMCGrid(ctx, g)
    G.setBasisFunctions(w.basis)
    S, h = api.overlap_core(w.basis, w.Z)
    return w, g, G, h


def _compare(G1, G2, D, h, precision=ffi.PREC_BF16X3):
    Gd, Fd, Ed = api.fock_build(G1, G2, D, h, precision=ffi.PREC_FP64)
    Gm, Fm, Em = api.fock_build(G1, G2, D, h, precision=precision)
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
    assert dE < e_tol(Ed), (Em, Ed)
    assert dG < G_REL_TOL


def test_he_full_grid(ctx, he):
    w, g, G, h = he
    rng = np.random.default_rng(2)
    D = real_density(w.basis, 1, rng)
    dE, dG, Em, Ed = _compare(G, G, D, h)
    assert dE < e_tol(Ed), (Em, Ed)
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
    assert dE < e_tol(Ed) and dG < G_REL_TOL, (Em, Ed, dG)
    D2 = np.stack([real_density(w.basis, 2, rng), real_density(w.basis, 1, rng)])
    dE, dG, Em, Ed = _compare(G1, G2, D2, h)
    assert dE < e_tol(Ed) and dG < G_REL_TOL, (Em, Ed, dG)


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
    assert dE < e_tol(Ed), (Em, Ed)
    assert dG < G_REL_TOL


def test_tensor_path_rank_chunks(ctx, he):
    w, g, G, h = he
    rng = np.random.default_rng(5)
    # a complex density of full rank 20 needs a 40-column factor (rank padding 64): one launch
    D = rand_density(w.nb, 20, rng)
    dE, dG, Em, Ed = _compare(G, G, D, h)
    assert dE < e_tol(Ed) and dG < G_REL_TOL, (Em, Ed, dG)
    # ranks above one launch's rank padding are contracted in column chunks whose T add up.
    # 120 functions with 36 real occupied orbitals: 32 + 4 columns (measured |dE|/|E| 5e-14, dG 2.6e-8,
    # the same as 32 orbitals in one launch)
    wk = wl.kr()
    q = grids.product_grid(6, 17)
    Q = api.QMCGrid(ctx, q)
    Q.setBasisFunctions(wk.basis)
    S, hk = api.overlap_core(wk.basis, wk.Z)
    dE, dG, Em, Ed = _compare(Q, Q, real_density(wk.basis, 36, rng), hk)
    assert dE < e_tol(Ed) and dG < G_REL_TOL, (Em, Ed, dG)
    # 40 functions with a random complex rank-40 density (80 columns: 64 + 16).  Random complex
    # densities of this rank (|E| ~ 1e6 Eh) sit at the 16-bit kernel tile's accuracy with or without
    # chunks: measured on 11,800 points |dE|/|E| 2.6e-8 and dG 2.8e-7 (a one-launch rank-30 density:
    # 1.5e-8 and 3.8e-7)
    wn = wl.ne()
    q = grids.product_grid(20, 41)
    Q = api.QMCGrid(ctx, q)
    Q.setBasisFunctions(wn.basis)
    S, hn = api.overlap_core(wn.basis, wn.Z)
    dE, dG, Em, Ed = _compare(Q, Q, rand_density(wn.nb, 40, np.random.default_rng(7)), hn)
    assert dE < 1e-7 * abs(Ed) and dG < 1e-6, (Em, Ed, dG)


def test_tf32_he_and_rank_chunks(ctx, he):
    w, g, G, h = he
    rng = np.random.default_rng(21)
    # a real rank-1 density (one launch) and a complex rank-20 density (40 factor columns: two TF32
    # launches of rank 32 + 8 whose T add up)
    for D in (real_density(w.basis, 1, rng), rand_density(w.nb, 20, rng)):
        dE, dG, Em, Ed = _compare(G, G, D, h, ffi.PREC_TF32)
        assert dE < TF32_E_REL_TOL * abs(Ed), (Em, Ed)
        assert dG < TF32_G_REL_TOL, dG


def test_tf32_nb128_tile(ctx):
    # 120 functions: the NB = 128 TF32 tile class, on a small grid
    wk = wl.kr()
    q = grids.product_grid(6, 17)
    Q = api.QMCGrid(ctx, q)
    Q.setBasisFunctions(wk.basis)
    S, hk = api.overlap_core(wk.basis, wk.Z)
    D = real_density(wk.basis, 18, np.random.default_rng(22))
    dE, dG, Em, Ed = _compare(Q, Q, D, hk, ffi.PREC_TF32)
    assert dE < TF32_E_REL_TOL * abs(Ed), (Em, Ed)
    assert dG < TF32_G_REL_TOL, dG

"""The Be transcorrelated configuration on the GPU: 24 STOs (s 12 + p 4 x 3, zeta = 0.4 * 1.8^k), three
independent 2^16-point scrambled-Sobol grids (r1; r2 for the TC scalar kernels; r3 for grad u) mapped
with the reference's QMC map, Jastrow u = r12 / (2 (1 + b r12)), b = 1, in the reference's sign
convention (HartreeFockTest.cpp:351-360).

* FP64 parity against the oracle on a sampled r1 subset (the oracle's precompute costs N2 nb^2 per
  row): computeF (same / opposite spin TC scalar kernels), computeV (same / opposite grad u) and the TC
  Fock build G2, G3, F, E built from those tensors (precomputeTranscorrelated,
  HartreeFockTest.cpp:261-319; TCHartreeFock, HartreeFock.cpp:1105-1261).  Bar: 1e-12 of the largest
  tensor element, 1e-10 of the largest G / F element and 1e-10 Eh.
* The split-BF16 tensor-core precompute against the FP64 one at full size (65,536 x 65,536 per
  kernel): every tensor within 2e-5 of its largest element (the FP32-coordinate limit for close
  QMC pairs, TENSOR_TOL), and the TC SCF energies built on each within 1 uEh (the mixed-precision
  bar).
* The tensor-core kernel-GEMM for 1/r12 (computeF) against FP64 on the He product grid, and an r12
  Jastrow with a second power, against FP64 on a small QMC case.
"""
import numpy as np
import pytest

import oracle
from tcscf_b200 import api, ffi, grids
from tcscf_b200 import basis as wl

pytestmark = pytest.mark.gpu

W = wl.be_tc()
J = wl.be_tc_jastrow(W)
SEED = W.extra["seed"]
N = W.qmc_points
ROWS = 64
KERNELS_F = (ffi.K_TC_SCALAR_SAME, ffi.K_TC_SCALAR_OPPO)
KERNELS_V = (ffi.K_GRAD_U_SAME, ffi.K_GRAD_U_OPPO)
# mixed-precision tensors against FP64, relative to the largest element: the kernel is generated from
# FP32 coordinates, whose rounding (2^-24 |r| per coordinate) gives a close pair (r12 ~ 1e-2 |r|) a
# relative error of ~1e-5; such pairs dominate a few tensor elements of the singular TC scalar kernel
TENSOR_TOL = 2e-5


@pytest.fixture(scope="module")
def be(ctx):
    g = [grids.qmc_grid(3, N, SEED + k) for k in range(3)]
    G = [api.QMCGrid(ctx, gk) for gk in g]
    G[0].setBasisFunctions(W.basis, storeGradients=True)
    G[1].setBasisFunctions(W.basis)
    G[2].setBasisFunctions(W.basis)
    rows = np.sort(np.random.default_rng(11).choice(N, ROWS, replace=False))
    g1s = grids.subset(g[0], rows)
    G1s = api.QMCGrid(ctx, g1s)
    G1s.setBasisFunctions(W.basis, storeGradients=True)
    yield g, G, g1s, G1s
    for x in G + [G1s]:
        x.close()


def _tensors(G1, G2, G3, u, precision, copy=False):
    Fs = api.computeF(G1, G2, ffi.K_TC_SCALAR_SAME, u, keep=True, copy=copy, precision=precision)
    Fo = api.computeF(G1, G2, ffi.K_TC_SCALAR_OPPO, u, keep=True, copy=copy, precision=precision)
    Vs = api.computeV(G1, G3, ffi.K_GRAD_U_SAME, u, keep=True, copy=copy, precision=precision)
    Vo = api.computeV(G1, G3, ffi.K_GRAD_U_OPPO, u, keep=True, copy=copy, precision=precision)
    return Fs, Fo, Vs, Vo


def _occupied(rng, nb):
    return [(rng.normal(size=(n, nb)) + 1j * rng.normal(size=(n, nb))) * 0.2 for n in (W.n_up, W.n_down)]


def test_be_tc_fp64_tensors_and_tc_build_match_oracle_on_sampled_rows(ctx, be):
    g, G, g1s, G1s = be
    u = ffi.ochi_struct(J["a"], J["a12"], J["terms"])
    uo = oracle.ochi(J["a"], J["a12"], J["terms"])
    gpu = _tensors(G1s, G[1], G[2], u, ffi.PREC_FP64, copy=True)
    vals2 = oracle.basis_values(g[1].points, W.basis)
    vals3 = oracle.basis_values(g[2].points, W.basis)
    ref = [oracle.compute_F(g1s.points, g[1].points, g[1].weights, vals2, W.nb, k, uo) for k in KERNELS_F]
    ref += [oracle.compute_V(g1s.points, g[2].points, g[2].weights, vals3, W.nb, k, uo) for k in KERNELS_V]
    for (arr, _), r in zip(gpu, ref):
        np.testing.assert_allclose(arr, r, rtol=0, atol=1e-12 * np.abs(r).max())
    # the TC Fock build on those tensors (random occupied orbitals of both spins)
    vals1, grads1 = oracle.basis_values(g1s.points, W.basis, gradients=True)
    _, h = api.overlap_core(W.basis, W.Z)
    occ = _occupied(np.random.default_rng(12), W.nb)
    D = np.stack([c.T @ c.conj() for c in occ])
    G2, G3, F, E = api.tc_fock_build(G1s, *(t for _, t in gpu), W.n_up, W.n_down, D, occ[0], occ[1], h)
    G2r, G3r, Fr, Er = oracle.tc_fock_build(*ref, vals1, grads1, g1s.weights, D, W.n_up, W.n_down, occ[0], occ[1], h)
    for a, b in ((G2, G2r), (G3, G3r), (F, Fr)):
        np.testing.assert_allclose(a, b, rtol=0, atol=1e-10 * max(1.0, np.abs(b).max()))
    assert abs(E - Er) < 1e-10 * max(1.0, abs(Er)), (E, Er)
    for _, t in gpu:
        t.close()


def test_be_tc_mixed_precompute_and_scf_match_fp64_at_full_size(ctx, be):
    g, G, _, _ = be
    u = ffi.ochi_struct(J["a"], J["a12"], J["terms"])
    S, h = api.overlap_core(W.basis, W.Z)
    res = {}
    for prec in (ffi.PREC_FP64, ffi.PREC_BF16X3):
        ts = _tensors(G[0], G[1], G[2], u, prec, copy=True)
        scf = api.TCHartreeFock(W.n_up, W.n_down)
        E = scf.compute(S, h, G[0], *(t for _, t in ts), tol=1e-9, max_iter=200)
        res[prec] = ([a for a, _ in ts], E, scf.iterations)
        for _, t in ts:
            t.close()
    for a, b in zip(res[ffi.PREC_BF16X3][0], res[ffi.PREC_FP64][0]):
        err = np.abs(a - b).max() / np.abs(b).max()
        assert err < TENSOR_TOL, err
    dE = res[ffi.PREC_BF16X3][1] - res[ffi.PREC_FP64][1]
    assert abs(dE) <= 1e-6, (dE, res[ffi.PREC_BF16X3][1:], res[ffi.PREC_FP64][1:])


def test_tensor_core_inv_r12_compute_f_matches_fp64(ctx):
    w = wl.he()
    g = grids.product_grid(w.nrad, w.order)
    rng = np.random.default_rng(13)
    g1 = grids.subset(g, rng.choice(g.n, 700, replace=False))
    G1 = api.QMCGrid(ctx, g1)
    G1.setBasisFunctions(w.basis)
    G2 = api.QMCGrid(ctx, g)
    G2.setBasisFunctions(w.basis)
    F64 = api.computeF(G1, G2, ffi.K_INV_R12)
    Fm = api.computeF(G1, G2, ffi.K_INV_R12, precision=ffi.PREC_BF16X3)
    assert np.abs(Fm - F64).max() <= 2e-6 * np.abs(F64).max()
    # the Fock build from each stored tensor (the reference's precompute form) agrees within 1 uEh
    C = rng.normal(size=(w.nb, 1)) * 0.3
    D = (C @ C.T).astype(np.complex128)
    _, h = api.overlap_core(w.basis, w.Z)
    _, t64 = api.computeF(G1, G2, ffi.K_INV_R12, keep=True, copy=False)
    _, tm = api.computeF(G1, G2, ffi.K_INV_R12, keep=True, copy=False, precision=ffi.PREC_BF16X3)
    E64 = api.fock_build_precomputed(G1, t64, D, h)[2]
    Em = api.fock_build_precomputed(G1, tm, D, h)[2]
    assert abs(Em - E64) <= 1e-6, (Em, E64)
    t64.close()
    tm.close()
    G1.close()
    G2.close()


def test_tensor_core_tc_kernels_with_a_second_r12_power(ctx):
    # u = c1 r12T + c2 r12T^2: the polynomial of u' has two coefficients per spin kind
    basis = wl.expand(0, [0.6, 1.5, 3.6, 8.5]) + wl.expand(1, [1.2])
    u = ffi.ochi_struct(0.8, 0.8, [((1, 0, 0), -0.4, -0.2), ((2, 0, 0), 0.15, 0.05)])
    g1, g2 = grids.qmc_grid(3, 640, 61), grids.qmc_grid(3, 4096, 62)
    G1 = api.QMCGrid(ctx, g1)
    G1.setBasisFunctions(basis)
    G2 = api.QMCGrid(ctx, g2)
    G2.setBasisFunctions(basis)
    for k in KERNELS_F:
        a = api.computeF(G1, G2, k, u, precision=ffi.PREC_BF16X3)
        b = api.computeF(G1, G2, k, u)
        assert np.abs(a - b).max() <= TENSOR_TOL * np.abs(b).max(), k
    for k in KERNELS_V:
        a = api.computeV(G1, G2, k, u, precision=ffi.PREC_BF16X3)
        b = api.computeV(G1, G2, k, u)
        assert np.abs(a - b).max() <= TENSOR_TOL * np.abs(b).max(), k
    G1.close()
    G2.close()


def test_tensor_core_tc_kernels_refuse_r1_dependent_jastrow(ctx):
    basis = wl.expand(0, [0.6, 1.5])
    u = ffi.ochi_struct(1.0, 1.0, [((1, 1, 0), -0.5, -0.25)])
    g1 = grids.qmc_grid(3, 128, 71)
    G1 = api.QMCGrid(ctx, g1)
    G1.setBasisFunctions(basis)
    with pytest.raises(ffi.TcscfError) as e:
        api.computeF(G1, G1, ffi.K_TC_SCALAR_SAME, u, precision=ffi.PREC_BF16X3)
    assert e.value.code == ffi.ERR_UNSUPPORTED
    G1.close()

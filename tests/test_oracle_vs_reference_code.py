"""The oracle pinned to the reference's own code.

oracle/_ref/libtcscf_ref.so is the reference's hot path compiled from its sources (HartreeFock.cpp,
HartreeFock.hpp, the integration headers, SlaterTypeOrbital.hpp, jastrowFunctions.hpp) over the
LvArray / RAJA / Caliper / qmc stand-ins in oracle/ref_shim/, built by `make -C oracle ref` where the
reference sources are present.  Each test runs the same inputs through the reference's function and
the oracle's restatement of it and asserts agreement at the level of FP64 rounding, so the oracle,
against which every GPU path is checked, computes what the reference computes:
  * the QMC map (QMCGrid constructor, integrateAll.hpp:21-63) on given unit-cube points;
  * STO values and gradients, m < 0 gradient quirk included (QMCGrid::setBasisFunctions,
    integrateAll.hpp:88-137; SlaterTypeOrbital.hpp:51-105), and the analytic S / H
    (SlaterTypeOrbital.hpp:118-176);
  * precomputeIntegrand + computeF (HartreeFock.hpp:23-180) with 1/r12 on 2-D real and 3-D complex r2
    grids and with the TC scalar kernels, and computeV with grad u (HartreeFock.hpp:185-229), the
    kernels being those of the reference's tests (HartreeFockTest.cpp:248-317);
  * the RCS, UOS and TC SCF drivers (HartreeFock.cpp:785-1362): iteration count, energy and density;
  * the Ochi and hydrogen-like families (OchiBasis.hpp, HydrogenLikeBasis.hpp): values, Ochi
    gradients, S and core H on the reference driver's core grid;
  * the 4- and 6-index tensors integrateAllR1R2 (value and gradient forms) and threeElectronIntegrals
    (integrateAll.hpp:152-442), and the 3-body verification route computeQ / assembleG
    (HartreeFock.cpp:613-752).
The reference's drivers call LAPACK through LvArray; the build gives them the LAPACK the oracle uses.
"""
from __future__ import annotations

import numpy as np
import pytest

import oracle
from tcscf_b200 import basis as wl
from tcscf_b200 import ffi, grids

if oracle.ref_lib() is None:
    pytest.skip("the reference's sources are not present to build oracle/_ref", allow_module_level=True)

RNG_SEED = 20261204
# He-like s / p functions and d / f functions with every m, so the gradient quirk for m < 0 is covered
BASIS_SP = [(0.9 * 1.8 ** k, 1, 0, 0) for k in range(6)] + [(1.0 * 2.0 ** k, 2, 1, 0) for k in range(2)]
BASIS_LM = ([(0.9 * 1.8 ** k, 1, 0, 0) for k in range(3)] + [(1.1, 2, 1, m) for m in (-1, 0, 1)]
            + [(0.7, 3, 2, m) for m in (-2, -1, 0, 1, 2)] + [(1.3, 4, 3, -3), (1.3, 4, 3, 2)])
JASTROW = oracle.ochi(1.0, 1.0, [((1, 0, 0), 0.5, 0.25), ((0, 1, 1), 0.1, -0.05), ((2, 0, 0), -0.2, 0.1)])


def _rel(a, b):
    return np.abs(a - b).max() / np.abs(b).max()


@pytest.fixture(scope="module")
def setting():
    """r1: 30 radial x Lebedev 17 product grid, rotated off the z axis (the reference's STO gradient
    divides by sin(theta)); r2: 3,000 QMC points in (r, theta), r3: 1,500 QMC points in 3-D."""
    from scipy.spatial.transform import Rotation

    rng = np.random.default_rng(RNG_SEED)
    r, wr = oracle.radial_grid(30, ffi.MAP_ONE_PLUS_X)
    p1, w1 = oracle.product_grid(r, wr, grids.lebedev_table(17))
    p1 = np.ascontiguousarray(Rotation.from_euler("zyx", [0.3, 0.2, 0.1]).as_matrix() @ p1)
    p2, w2 = oracle.qmc_grid(np.ascontiguousarray(rng.random((2, 3000))))
    p3, w3 = oracle.qmc_grid(np.ascontiguousarray(rng.random((3, 1500))))
    return p1, w1, p2, w2, p3, w3


@pytest.mark.parametrize("ndim", [2, 3])
def test_qmc_map_matches_reference(ndim):
    u = np.ascontiguousarray(np.random.default_rng(RNG_SEED + ndim).random((ndim, 4000)))
    po, wo = oracle.qmc_grid(u)
    pr, wr = oracle.ref_qmc_grid(u)
    assert _rel(po, pr) < 1e-15
    assert _rel(wo, wr) < 1e-14


@pytest.mark.parametrize("ndim", [2, 3])
def test_sto_values_and_gradients_match_reference(ndim):
    pts, _ = oracle.qmc_grid(np.ascontiguousarray(np.random.default_rng(RNG_SEED + 10 + ndim).random((ndim, 600))))
    if ndim == 3:
        vo, go = oracle.basis_values(pts, BASIS_LM, gradients=True)
        vr, gr = oracle.ref_sto_values(pts, BASIS_LM, gradients=True)
        assert _rel(go, gr) < 1e-14
    else:
        vo = oracle.basis_values(pts, BASIS_LM)
        vr = oracle.ref_sto_values(pts, BASIS_LM)
    assert _rel(vo, vr) < 1e-14


def test_analytic_overlap_and_core_match_reference():
    S, H = oracle.overlap_core(BASIS_LM, 5)
    Sr, Hr = oracle.ref_overlap_core(BASIS_LM, 5)
    assert _rel(S, Sr) < 1e-14 and _rel(H, Hr) < 1e-14


def test_compute_F_matches_reference(setting):
    """1/r12 on the 2-D real r2 grid (F real, scaled by 2 pi) and on the 3-D complex r3 grid."""
    p1, w1, p2, w2, p3, w3 = setting
    nb = len(BASIS_SP)
    v1 = oracle.basis_values(p1, BASIS_SP)
    for p, w in ((p2, w2), (p3, w3)):
        v = oracle.basis_values(p, BASIS_SP)
        F = oracle.compute_F(p1, p, w, v, nb)
        Fr = oracle.ref_compute_F(p1, w1, v1, p, w, v, nb)
        assert F.dtype == Fr.dtype
        assert _rel(F, Fr) < 1e-14


def test_tc_kernels_match_reference(setting):
    """computeF with the TC scalar kernels 2/r12 - |grad_12 u|^2 - |grad_21 u|^2 and computeV with
    grad u, same and opposite spin, for a three-term Ochi Jastrow factor."""
    p1, w1, p2, w2, p3, w3 = setting
    nb = len(BASIS_SP)
    v1 = oracle.basis_values(p1, BASIS_SP)
    v2 = oracle.basis_values(p2, BASIS_SP)
    v3 = oracle.basis_values(p3, BASIS_SP)
    for k in (ffi.K_TC_SCALAR_SAME, ffi.K_TC_SCALAR_OPPO):
        assert _rel(oracle.compute_F(p1, p2, w2, v2, nb, k, JASTROW), oracle.ref_compute_F(p1, w1, v1, p2, w2, v2, nb, k, JASTROW)) < 1e-14
    for k in (ffi.K_GRAD_U_SAME, ffi.K_GRAD_U_OPPO):
        assert _rel(oracle.compute_V(p1, p3, w3, v3, nb, k, JASTROW), oracle.ref_compute_V(p1, w1, v1, p3, w3, v3, nb, k, JASTROW)) < 1e-14


@pytest.mark.parametrize("nspin,n_up,n_down,Z,sym", [(1, 1, 1, 2, True), (2, 1, 1, 2, True), (2, 2, 1, 3, True), (1, 1, 1, 2, False),
                                                     (2, 2, 1, 3, False)])
def test_rcs_uos_scf_match_reference(setting, nspin, n_up, n_down, Z, sym):
    """RCS He, UOS He and UOS Li (two spin-up electrons, one spin-down) through the reference's
    drivers (their own 1e-5 stopping rule) and the oracle's restatement of them, with and without the
    one-electron symmetry mask of the two-electron terms."""
    p1, w1, p2, w2, _, _ = setting
    nb = len(BASIS_SP)
    v1 = oracle.basis_values(p1, BASIS_SP)
    F = oracle.compute_F(p1, p2, w2, oracle.basis_values(p2, BASIS_SP), nb)
    S, h = oracle.overlap_core(BASIS_SP, Z)
    st, E, it, D, _ = oracle.scf(nspin, n_up, n_down, F, v1, w1, S, h, respect_symmetry=sym)
    loops, Er, Dr = oracle.ref_scf(nspin, n_up, n_down, F, p1, w1, v1, S, h, respect_symmetry=sym)
    assert st == 0 and loops == it
    assert abs(E - Er) < 1e-12 * abs(Er), (E, Er)
    assert np.abs(D - Dr).max() < 1e-12


@pytest.mark.parametrize("n_up,n_down,Z", [(1, 1, 2), (2, 1, 3)])
def test_tc_scf_matches_reference(setting, n_up, n_down, Z):
    """TCHartreeFock::compute (zggev, the sort by real part, the S-metric MGS with its quirk) on the
    TC tensors of a nonzero Jastrow factor: He with one electron of each spin, and Li with two
    spin-up electrons and one spin-down."""
    p1, w1, p2, w2, p3, w3 = setting
    nb = len(BASIS_SP)
    v1, g1 = oracle.basis_values(p1, BASIS_SP, gradients=True)
    v2 = oracle.basis_values(p2, BASIS_SP)
    v3 = oracle.basis_values(p3, BASIS_SP)
    Fs = oracle.compute_F(p1, p2, w2, v2, nb, ffi.K_TC_SCALAR_SAME, JASTROW)
    Fo = oracle.compute_F(p1, p2, w2, v2, nb, ffi.K_TC_SCALAR_OPPO, JASTROW)
    Vs = oracle.compute_V(p1, p3, w3, v3, nb, ffi.K_GRAD_U_SAME, JASTROW)
    Vo = oracle.compute_V(p1, p3, w3, v3, nb, ffi.K_GRAD_U_OPPO, JASTROW)
    S, h = oracle.overlap_core(BASIS_SP, Z)
    st, E, it, D, _ = oracle.tc_scf(Fs, Fo, Vs, Vo, v1, g1, w1, S, h, n_up, n_down)
    loops, Er, Dr = oracle.ref_tc_scf(Fs, Fo, Vs, Vo, p1, w1, v1, g1, S, h, n_up, n_down)
    assert st == 0 and loops == it
    assert abs(E - Er) < 1e-12 * abs(Er), (E, Er)
    assert np.abs(D - Dr).max() < 1e-12


@pytest.mark.parametrize("family", ["ochi", "hydrogen"])
def test_basis_families_match_reference(family):
    """Values on 2-D and 3-D points (Ochi gradients too: the reference has no hydrogen-like gradient),
    and S / core H as the reference's driver fills them (HartreeFockTest.cpp:363-378); the
    hydrogen-like overlap, which the reference integrates numerically in 3-D, is compared in the
    GPU tests against the analytic orthonormality instead."""
    basis, Z = (wl.ochi_functions(3, 2, 1.7), 2) if family == "ochi" else (wl.hydrogen_functions(3, 2, 2), 2)
    rng = np.random.default_rng(RNG_SEED + 20)
    for ndim in (2, 3):
        pts, _ = oracle.qmc_grid(np.ascontiguousarray(rng.random((ndim, 400))))
        grads = family == "ochi" and ndim == 3
        if grads:
            vo, go = oracle.basis_values(pts, basis, gradients=True)
            vr, gr = oracle.ref_family_values(pts, basis, gradients=True)
            assert _rel(go, gr) < 1e-13
        else:
            vo = oracle.basis_values(pts, basis)
            vr = oracle.ref_family_values(pts, basis)
        assert _rel(vo, vr) < 1e-13
    S, H = oracle.overlap_core(basis, Z)
    Sr, Hr = oracle.ref_family_overlap_core(basis, Z)
    assert _rel(H, Hr) < 1e-13
    if family == "ochi":
        assert np.array_equal(S, Sr)


@pytest.fixture(scope="module")
def tensor_grids():
    """r1: 96 QMC points in 3-D; r2: 400 in (r, theta) with gradients; the basis of the GPU tensor tests."""
    rng = np.random.default_rng(RNG_SEED + 30)
    basis = wl.expand(0, [0.8, 1.9]) + wl.expand(1, [1.3])
    p1, w1 = oracle.qmc_grid(np.ascontiguousarray(rng.random((3, 96))))
    p2, w2 = oracle.qmc_grid(np.ascontiguousarray(rng.random((2, 400))))
    v1 = oracle.basis_values(p1, basis)
    v2, g2 = oracle.basis_values(p2, basis, gradients=True)
    return basis, p1, w1, v1, p2, w2, v2, g2


@pytest.mark.parametrize("kernel", [ffi.K_INV_R12, ffi.K_TC_SCALAR_SAME, ffi.K_GRAD_U_SAME, ffi.K_GRAD_U_OPPO])
def test_integrate_all_r1r2_matches_reference(tensor_grids, kernel):
    basis, p1, w1, v1, p2, w2, v2, g2 = tensor_grids
    grad = kernel >= ffi.K_GRAD_U_SAME
    u = JASTROW if kernel != ffi.K_INV_R12 else None
    ours = oracle.integrate_all_r1r2(grad, p1, w1, v1, p2, w2, v2, g2 if grad else None, len(basis), kernel, u)
    ref = oracle.ref_integrate_all_r1r2(grad, p1, w1, v1, p2, w2, v2, g2 if grad else None, len(basis), kernel, u)
    assert _rel(ours, ref) < 1e-13


def test_three_electron_integrals_match_reference():
    rng = np.random.default_rng(RNG_SEED + 40)
    basis = wl.expand(0, [0.9]) + wl.expand(1, [1.4])
    p1, w1 = oracle.qmc_grid(np.ascontiguousarray(rng.random((3, 60))))
    p2, w2 = oracle.qmc_grid(np.ascontiguousarray(rng.random((3, 200))))
    v1, v2 = oracle.basis_values(p1, basis), oracle.basis_values(p2, basis)
    ours = oracle.three_electron_integrals(p1, w1, v1, p2, w2, v2, len(basis), JASTROW)
    ref = oracle.ref_three_electron_integrals(p1, w1, v1, p2, w2, v2, len(basis), JASTROW)
    assert _rel(ours, ref) < 1e-13


def test_compute_q_and_assemble_g_match_reference():
    """computeQ / assembleG on grad-u tensors of a Jastrow factor with c_same = c_opposite / 2 in every
    term, the convention assembleG itself asserts (Q_so = 2 Q_ss, HartreeFock.cpp:722)."""
    jastrow = oracle.ochi(1.0, 1.0, [((1, 0, 0), 0.5, 0.25), ((0, 1, 1), 0.1, 0.05), ((2, 0, 0), -0.2, -0.1)])
    rng = np.random.default_rng(RNG_SEED + 50)
    basis = wl.expand(0, [0.9, 2.0]) + wl.expand(1, [1.4])
    nb = len(basis)
    p1, w1 = oracle.qmc_grid(np.ascontiguousarray(rng.random((3, 50))))
    p3, w3 = oracle.qmc_grid(np.ascontiguousarray(rng.random((3, 300))))
    v1, v3 = oracle.basis_values(p1, basis), oracle.basis_values(p3, basis)
    Vs = oracle.compute_V(p1, p3, w3, v3, nb, ffi.K_GRAD_U_SAME, jastrow)
    Vo = oracle.compute_V(p1, p3, w3, v3, nb, ffi.K_GRAD_U_OPPO, jastrow)
    Q = oracle.compute_q(w1, v1, Vs, Vo)
    Qr = oracle.ref_compute_q(w1, v1, Vs, Vo)
    for a, b in zip(Q, Qr):
        assert _rel(a, b) < 1e-13
    C = [rng.normal(size=(n, nb)) + 1j * rng.normal(size=(n, nb)) for n in (2, 1)]
    D = np.stack([c.T @ c.conj() for c in C])
    assert _rel(oracle.assemble_g(*Q, D), oracle.ref_assemble_g(*Q, D)) < 1e-13


def test_load_sto_matches_reference_on_its_library():
    """The product's loadSTO (host code, no GPU) against the reference's (SlaterTypeOrbital.cpp:24-75)
    on every file of the reference's basis-set library, for each basis set and several l cut-offs:
    identical function lists (exponents parsed to the same doubles, m expanded -l..l in file order).
    Files the reference's loader rejects (a shell type beyond f, as in Gd, Th and Ra) and an unknown
    basis set are rejected by both."""
    from tcscf_b200 import api

    lib = oracle.ref_basis_library()
    if lib is None:
        pytest.skip("the reference build was not given its basis-set library")
    checked = rejected = 0
    for basis_set in ("TZ3P", "QZ6P", "ATZ3P", "AQZ6P"):
        for element in sorted(p.name for p in (lib / basis_set).iterdir() if p.is_file()):
            for max_l in (0, 1, 3, 99):
                ref = oracle.ref_load_sto(lib, basis_set, element, max_l)
                if ref is None:
                    with pytest.raises(ffi.TcscfError):
                        api.loadSTO(lib, basis_set, element, max_l)
                    rejected += 1
                else:
                    assert [tuple(f) for f in api.loadSTO(lib, basis_set, element, max_l)] == ref, (basis_set, element, max_l)
                checked += 1
    assert checked > 1000 and rejected < checked // 10
    assert oracle.ref_load_sto(lib, "XZ9P", "He", 3) is None
    with pytest.raises(ffi.TcscfError):
        api.loadSTO(lib, "XZ9P", "He", 3)


# ---- the product's host code against the reference's, directly ---------------------------------------

@pytest.mark.parametrize("map_,p0,p1", [(ffi.MAP_NONE, 0.0, 0.0), (ffi.MAP_LINEAR, 2.5, 0.0), (ffi.MAP_X_OVER_1MX, 0.0, 0.0),
                                        (ffi.MAP_TREUTLER_AHLRICHS_M4, 1.0, 0.9)])
def test_product_radial_grids_match_reference(map_, p0, p1):
    """tcscf_grid_radial against createGrid(ChebyshevGauss(n), map) of the reference: identical doubles
    (r = (1+x)/(1-x), the fifth map, is not in the reference)."""
    for n in (7, 50, 200):
        u, w = grids.radial_grid(n, map_, p0, p1)
        ur, wr = oracle.ref_radial_grid(n, map_, p0, p1)
        assert np.array_equal(u, ur) and np.array_equal(w, wr)


@pytest.mark.parametrize("ndim", [2, 3])
def test_product_qmc_map_matches_reference(ndim):
    """tcscf_grid_qmc (the map under grids.qmc_grid) against the reference's QMCGrid on the same points."""
    u = np.ascontiguousarray(np.random.default_rng(RNG_SEED + 60 + ndim).random((ndim, 3000)))
    pts, w = np.empty_like(u), np.empty(u.shape[1])
    ffi.check(ffi.lib().tcscf_grid_qmc(ndim, u.shape[1], ffi.dptr(u), ffi.dptr(pts), ffi.dptr(w)))
    pr, wr = oracle.ref_qmc_grid(u)
    assert _rel(pts, pr) < 1e-15 and _rel(w, wr) < 1e-14


def test_product_analytic_overlap_core_matches_reference():
    """The product's analytic S and core H (tcscf_overlap_core_analytic) for the STO family, and for the
    Ochi and hydrogen-like families on the reference driver's core grid (S of the hydrogen-like family
    is the reference's numerical 3-D overlap, not compared)."""
    from tcscf_b200 import api

    S, H = api.overlap_core(BASIS_LM, 5)
    Sr, Hr = oracle.ref_overlap_core(BASIS_LM, 5)
    assert _rel(S, Sr) < 1e-14 and _rel(H, Hr) < 1e-14
    for basis in (wl.ochi_functions(3, 2, 1.7), wl.hydrogen_functions(3, 2, 2)):
        S, H = api.overlap_core(basis, 2)
        Sr, Hr = oracle.ref_family_overlap_core(basis, 2)
        assert _rel(H, Hr) < 1e-13
        if basis[0][4] == 1:
            assert np.array_equal(S, Sr)

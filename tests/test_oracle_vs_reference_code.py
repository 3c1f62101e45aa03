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
  * the RCS, UOS and TC SCF drivers (HartreeFock.cpp:785-1362): iteration count, energy and density.
The reference's drivers call LAPACK through LvArray; the build gives them the LAPACK the oracle uses.
"""
from __future__ import annotations

import numpy as np
import pytest

import oracle
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


@pytest.mark.parametrize("nspin,n_up,n_down,Z", [(1, 1, 1, 2), (2, 1, 1, 2), (2, 2, 1, 3)])
def test_rcs_uos_scf_match_reference(setting, nspin, n_up, n_down, Z):
    """RCS He, UOS He and UOS Li (two spin-up electrons, one spin-down) through the reference's
    drivers (their own 1e-5 stopping rule) and the oracle's restatement of them."""
    p1, w1, p2, w2, _, _ = setting
    nb = len(BASIS_SP)
    v1 = oracle.basis_values(p1, BASIS_SP)
    F = oracle.compute_F(p1, p2, w2, oracle.basis_values(p2, BASIS_SP), nb)
    S, h = oracle.overlap_core(BASIS_SP, Z)
    st, E, it, D, _ = oracle.scf(nspin, n_up, n_down, F, v1, w1, S, h)
    loops, Er, Dr = oracle.ref_scf(nspin, n_up, n_down, F, p1, w1, v1, S, h)
    assert st == 0 and loops == it
    assert abs(E - Er) < 1e-12 * abs(Er), (E, Er)
    assert np.abs(D - Dr).max() < 1e-12


def test_tc_scf_matches_reference(setting):
    """TCHartreeFock::compute (zggev, the sort by real part, the S-metric MGS with its quirk) on the
    TC tensors of a nonzero Jastrow factor, He with one electron of each spin."""
    p1, w1, p2, w2, p3, w3 = setting
    nb = len(BASIS_SP)
    v1, g1 = oracle.basis_values(p1, BASIS_SP, gradients=True)
    v2 = oracle.basis_values(p2, BASIS_SP)
    v3 = oracle.basis_values(p3, BASIS_SP)
    Fs = oracle.compute_F(p1, p2, w2, v2, nb, ffi.K_TC_SCALAR_SAME, JASTROW)
    Fo = oracle.compute_F(p1, p2, w2, v2, nb, ffi.K_TC_SCALAR_OPPO, JASTROW)
    Vs = oracle.compute_V(p1, p3, w3, v3, nb, ffi.K_GRAD_U_SAME, JASTROW)
    Vo = oracle.compute_V(p1, p3, w3, v3, nb, ffi.K_GRAD_U_OPPO, JASTROW)
    S, h = oracle.overlap_core(BASIS_SP, 2)
    st, E, it, D, _ = oracle.tc_scf(Fs, Fo, Vs, Vo, v1, g1, w1, S, h, 1, 1)
    loops, Er, Dr = oracle.ref_tc_scf(Fs, Fo, Vs, Vo, p1, w1, v1, g1, S, h, 1, 1)
    assert st == 0 and loops == it
    assert abs(E - Er) < 1e-12 * abs(Er), (E, Er)
    assert np.abs(D - Dr).max() < 1e-12

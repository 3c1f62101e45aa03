"""Host grid generation: the scipy-sourced Lebedev rules are the reference's tables, and the library's
product / QMC grids equal the oracle's restatement point for point."""
import json
from pathlib import Path

import numpy as np
import pytest

import oracle
from tcscf_b200 import basis as wl
from tcscf_b200 import grids

LEB = json.loads((Path(__file__).parent / "golden" / "lebedev_reference.json").read_text())


@pytest.mark.parametrize("order", sorted(int(k) for k in LEB))
def test_lebedev_rule_equals_reference_table(order):
    ref = LEB[str(order)]
    ang = grids.lebedev_table(order)
    assert ang.shape[0] == ref["npoints"] == wl.lebedev_npoints(order)
    np.testing.assert_allclose(sorted(set(np.round(ang[:, 2], 12))), np.round(ref["distinct_weights"], 12), rtol=0, atol=2e-12)
    np.testing.assert_allclose(np.sort(ang[:, 0]), ref["sorted_theta"], rtol=0, atol=1e-12)
    assert abs(ang[:, 2].sum() - 4 * np.pi) < 1e-12


def test_product_grid_matches_oracle():
    g = grids.product_grid(12, 11)
    r, wr = oracle.radial_grid(12, 4)
    pts, w = oracle.product_grid(r, wr, grids.lebedev_table(11))
    np.testing.assert_allclose(g.points, pts, rtol=1e-15, atol=1e-300)
    np.testing.assert_allclose(g.weights, w, rtol=1e-15, atol=0)


@pytest.mark.parametrize("ndim", [2, 3])
def test_qmc_mapping_matches_oracle(ndim):
    u = grids.sobol(ndim, 4096, 7)
    g = grids.qmc_grid(ndim, 4096, 7)
    pts, w = oracle.qmc_grid(u)
    np.testing.assert_allclose(g.points, pts, rtol=1e-14, atol=1e-14)
    np.testing.assert_allclose(g.weights, w, rtol=1e-13, atol=0)


def test_sobol_points_are_a_scrambled_net():
    u = grids.sobol(3, 1 << 12, 20261203)
    assert u.min() > 0 and u.max() < 1
    # (0, m, s)-net-like stratification of the first dimension: every 1/4096 interval holds one point
    assert np.all(np.bincount((u[0] * 4096).astype(int), minlength=4096) == 1)
    # 2-D stratification of dimensions 1 and 2 on a 64 x 64 grid
    h = np.histogram2d(u[1], u[2], bins=64, range=[[0, 1], [0, 1]])[0]
    assert h.min() >= 1
    # different seeds give different point sets; same seed reproduces
    assert not np.allclose(u, grids.sobol(3, 1 << 12, 1))
    np.testing.assert_array_equal(u, grids.sobol(3, 1 << 12, 20261203))


def test_qmc_grid_integrates_a_normalised_density():
    # sum_g w rho(r) for a normalised 1s density ~ 1 (QMC estimate)
    g = grids.qmc_grid(3, 1 << 16, 3)
    r = np.linalg.norm(g.points, axis=0)
    rho = np.exp(-2 * r) / np.pi
    assert abs(np.sum(g.weights * rho) - 1.0) < 5e-3


def test_workload_sizes():
    assert wl.he().nb == 20 and wl.he().npoints == 2500
    assert wl.ne().nb == 40 and wl.ne().npoints == 59000
    assert wl.kr().nb == 120 and wl.kr().npoints == 406000
    assert wl.be_tc().nb == 24
    b = wl.batch()
    assert len(b) == 64 and all(10 <= x.nb <= 80 for x in b)


def test_coincident_pairs_are_counted():
    """Exact r1 == r2 pairs (dropped by every r12 kernel) and pairs equal up to rounding (where 1/r12
    explodes): Chebyshev rules of 6 and 21 nodes (n + 1 = 6, 21) share two radii up to rounding, and
    the Lebedev rules of orders 11 and 17 share 14 directions; rules of 10 and 15 nodes share four
    radii exactly, orders 3 and 5 the six octahedral directions."""
    g = grids.product_grid(12, 11)
    assert grids.coincident_pairs(g, g) == (g.n, 0)
    assert grids.coincident_pairs(grids.product_grid(5, 11), grids.product_grid(20, 17)) == (0, 28)
    assert grids.coincident_pairs(grids.product_grid(9, 3), grids.product_grid(14, 5)) == (24, 0)
    assert grids.coincident_pairs(grids.product_grid(8, 11), grids.product_grid(9, 17)) == (0, 0)
    # a 2-D (x, z) grid is compared in the y = 0 plane
    g2 = grids.QuadratureGrid(np.ascontiguousarray(g.points[[0, 2]]), g.weights)
    assert grids.coincident_pairs(g, g2)[0] >= 1

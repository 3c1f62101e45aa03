"""Host-side quadrature grids (thin wrappers over the library's host grid generators).

Lebedev angular rules come from scipy.integrate.lebedev_rule (the published Lebedev-Laikov
quadratures; the same rules as the reference's src/integration/data tables, which
tests/test_golden_grids.py pins); radial rules, product grids, the QMC point mapping and the Sobol
source are the library's C functions.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from . import ffi


@dataclass
class QuadratureGrid:
    """integration::QuadratureGrid (src/integration/quadrature.hpp:25-35): points [ndim][N], weights [N]."""

    points: np.ndarray
    weights: np.ndarray

    @property
    def ndim(self) -> int:
        return self.points.shape[0]

    @property
    def n(self) -> int:
        return self.weights.shape[0]


def lebedev_table(order: int) -> np.ndarray:
    """Lebedev rule of the given order as rows {theta, phi, weight} with weights summing to 4 pi
    (the column layout of the reference's LebedevData_*.hpp tables)."""
    from scipy.integrate import lebedev_rule

    x, w = lebedev_rule(order)
    theta = np.arccos(np.clip(x[2], -1.0, 1.0))
    phi = np.arctan2(x[1], x[0])
    return np.ascontiguousarray(np.stack([theta, phi, w], axis=1))


def radial_grid(n: int, map_: int = ffi.MAP_ONE_PLUS_X, p0: float = 0.0, p1: float = 0.0):
    u = np.empty(n)
    w = np.empty(n)
    ffi.check(ffi.lib().tcscf_grid_radial(n, map_, p0, p1, ffi.dptr(u), ffi.dptr(w)))
    return u, w


def product_grid(nrad: int, order: int, map_: int = ffi.MAP_ONE_PLUS_X, p0: float = 0.0, p1: float = 0.0) -> QuadratureGrid:
    r, wr = radial_grid(nrad, map_, p0, p1)
    ang = lebedev_table(order)
    N = nrad * ang.shape[0]
    pts = np.empty((3, N))
    w = np.empty(N)
    ffi.check(ffi.lib().tcscf_grid_product(nrad, ffi.dptr(r), ffi.dptr(wr), ang.shape[0], ffi.dptr(ang), ffi.dptr(pts), ffi.dptr(w)))
    return QuadratureGrid(pts, w)


def sobol(ndim: int, n: int, seed: int) -> np.ndarray:
    u = np.empty((ndim, n))
    ffi.check(ffi.lib().tcscf_sobol(ndim, n, seed, ffi.dptr(u)))
    return u


def qmc_grid(ndim: int, n: int, seed: int) -> QuadratureGrid:
    u = sobol(ndim, n, seed)
    pts = np.empty((ndim, n))
    w = np.empty(n)
    ffi.check(ffi.lib().tcscf_grid_qmc(ndim, n, ffi.dptr(u), ffi.dptr(pts), ffi.dptr(w)))
    return QuadratureGrid(pts, w)


def subset(grid: QuadratureGrid, idx) -> QuadratureGrid:
    idx = np.asarray(idx)
    return QuadratureGrid(np.ascontiguousarray(grid.points[:, idx]), np.ascontiguousarray(grid.weights[idx]))


def _cartesian(grid: QuadratureGrid) -> np.ndarray:
    """Points as [N][3]; a 2-D grid's rows are (x, z) with y = 0."""
    p = grid.points
    if grid.ndim == 2:
        return np.stack([p[0], np.zeros_like(p[0]), p[1]], axis=1)
    return np.ascontiguousarray(p.T)


def coincident_pairs(r1: QuadratureGrid, r2: QuadratureGrid, rel_tol: float = 1e-10) -> tuple[int, int]:
    """(exact, near): the r1 / r2 point pairs with r1 == r2, which every r12 kernel drops (contributes 0,
    the reference's r12Inv convention, src/unitTests/IntegrationTest.cpp:298-309), and the pairs
    with 0 < |r1 - r2| <= rel_tol |r1|, where 1/r12 exceeds 1/(rel_tol |r1|) and swamps the quadrature.
    Near pairs arise when two grids share angular directions and radial nodes up to rounding, e.g.
    Chebyshev radial rules of n and m points with (n + 1) and (m + 1) sharing a factor."""
    from scipy.spatial import cKDTree

    a, b = _cartesian(r1), _cartesian(r2)
    tree = cKDTree(b)
    radius = rel_tol * np.linalg.norm(a, axis=1)
    exact = near = 0
    for i, hits in enumerate(tree.query_ball_point(a, np.maximum(radius, 0.0))):
        for j in hits:
            if np.array_equal(a[i], b[j]):
                exact += 1
            else:
                near += 1
    # a point at the origin has radius 0: query_ball_point returns only exact matches there
    return exact, near

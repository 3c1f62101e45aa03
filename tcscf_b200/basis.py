"""Even-tempered STO basis sets and the synthetic atomic workloads (He, Ne, Be, Kr, 64-atom batch).

Basis-count rule: for a per-l budget B, floor(B/(2l+1)) exponents per l (l <= 3), each expanded over
m = -l..l in the order of loadSTO (src/SlaterTypeOrbital.cpp:57-62), n = l+1, with the remainder
padded by further s exponents continuing k; exponents zeta_k = z0 * ratio**k per l.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

Basis = list  # list of (alpha, n, l, m) Slater-type orbitals, or (alpha, n, l, m, family)


def expand(l: int, zetas) -> Basis:
    return [(float(z), l + 1, l, m) for z in zetas for m in range(-l, l + 1)]


def ochi_functions(n_max: int, l_max: int, alpha: float) -> Basis:
    """Ochi functions (family 1) for n = 0..n_max, l = 0..l_max, m = -l..l in the order of
    createBasisFunctions (src/unitTests/HartreeFockTest.cpp:153-172)."""
    return [(float(alpha), n, l, m, 1) for n in range(n_max + 1) for l in range(l_max + 1) for m in range(-l, l + 1)]


def hydrogen_functions(n_max: int, l_max: int, Z: int) -> Basis:
    """Hydrogen-like functions (family 2, alpha = Z) for n = 1..n_max, l = 0..min(l_max, n - 1),
    m = -l..l.  createBasisFunctions (src/unitTests/HartreeFockTest.cpp:178-198) runs l up to
    min(l_max, n), which the constructor's l < n check (HydrogenLikeBasis.hpp:33) rejects at l = n."""
    return [(float(Z), n, l, m, 2) for n in range(1, n_max + 1) for l in range(min(l_max, n - 1) + 1) for m in range(-l, l + 1)]


def even_tempered(counts: dict[int, int], z0: float, ratio: float) -> Basis:
    out: Basis = []
    for l in sorted(counts):
        out += expand(l, [z0 * ratio ** k for k in range(counts[l])])
    return out


def budget_counts(budget: int, total: int, lmax: int = 3) -> dict[int, int]:
    counts = {l: budget // (2 * l + 1) for l in range(lmax + 1)}
    nb = sum(c * (2 * l + 1) for l, c in counts.items())
    counts[0] += max(0, total - nb)
    return counts


def real_harmonic_unitary(basis: Basis) -> np.ndarray:
    """U with phi^R = U phi: m > 0 -> (phi_m + phi_-m)/sqrt2, m < 0 -> (phi_|m| - phi_-|m|)/(i sqrt2)
    (the reference's Y_l^m = P_l^|m| e^{i m phi} convention, mathFunctions.hpp:126-139)."""
    nb = len(basis)
    key = lambda b: (b[0], b[1], b[2], b[3], b[4] if len(b) > 4 else 0)
    idx = {key(b): i for i, b in enumerate(basis)}
    U = np.zeros((nb, nb), dtype=complex)
    h = 1 / np.sqrt(2)
    for k, b in enumerate(basis):
        a, n, l, m, fam = key(b)
        if m == 0:
            U[k, k] = 1
            continue
        p = idx[(a, n, l, -m, fam)]
        if m > 0:
            U[k, k], U[k, p] = h, h
        else:
            U[k, p], U[k, k] = -1j * h, 1j * h
    return U


@dataclass
class Workload:
    name: str
    Z: int
    basis: Basis
    nrad: int = 0           # radial points (Gauss-Chebyshev, r = (1+x)/(1-x))
    order: int = 0          # Lebedev order
    n_up: int = 0
    n_down: int = 0
    qmc_points: int = 0     # scrambled-Sobol points per electron coordinate (QMC workloads)
    extra: dict = field(default_factory=dict)

    @property
    def nb(self) -> int:
        return len(self.basis)

    @property
    def npoints(self) -> int:
        return self.qmc_points or self.nrad * lebedev_npoints(self.order)


_LEB_N = {3: 6, 5: 14, 7: 26, 9: 38, 11: 50, 13: 74, 15: 86, 17: 110, 19: 146, 21: 170, 23: 194, 25: 230, 27: 266,
          29: 302, 31: 350, 35: 434, 41: 590, 47: 770, 53: 974, 59: 1202, 65: 1454, 71: 1730, 77: 2030, 83: 2354,
          89: 2702, 95: 3074, 101: 3470, 107: 3890, 113: 4334, 119: 4802, 125: 5294, 131: 5810}


def lebedev_npoints(order: int) -> int:
    return _LEB_N[order]


def he() -> Workload:
    """He, Z=2, RCS: 8 s (n=1, 0.5*1.8^k) + 4 p (n=2, 1.0*2^k); 50 radial x Lebedev-11 (50 points)."""
    basis = expand(0, [0.5 * 1.8 ** k for k in range(8)]) + expand(1, [1.0 * 2.0 ** k for k in range(4)])
    return Workload("He", 2, basis, nrad=50, order=11, n_up=1, n_down=1)


def ne() -> Workload:
    """Ne, Z=10, closed shell: 40 STOs zeta = 0.3*1.7^k (s 14, p 3x3, d 2x5, f 1x7); 100 x Lebedev-41 (590)."""
    basis = even_tempered(budget_counts(10, 40), 0.3, 1.7)
    return Workload("Ne", 10, basis, nrad=100, order=41, n_up=5, n_down=5)


def be_tc() -> Workload:
    """Be, Z=4, transcorrelated: 12 s (0.4*1.8^k) + 4 p x 3 (0.4*1.8^k); 2^16 Sobol points per coordinate
    on three independent grids (seeds seed, seed+1, seed+2: r1, r2 for the scalar kernels, r3 for grad u)."""
    basis = expand(0, [0.4 * 1.8 ** k for k in range(12)]) + expand(1, [0.4 * 1.8 ** k for k in range(4)])
    return Workload("Be-TC", 4, basis, n_up=2, n_down=2, qmc_points=1 << 16,
                    extra={"b": 1.0, "seed": 20261203})


def be_tc_jastrow(w: Workload) -> dict:
    """u(r12) = r12 / (2 (1 + b r12)) as an Ochi factor of r12 alone: S = {(1, 0, 0)}, a12 = 1/b, in the
    sign convention of the reference's TC driver (HartreeFockTest.cpp:351-360): c = -a12/2 for opposite
    spins and -a12/4 for equal spins.  a (the r1 / r2 scale) does not enter; it is set to a12."""
    a12 = 1.0 / w.extra["b"]
    return dict(a=a12, a12=a12, terms=[((1, 0, 0), -a12 / 2, -a12 / 4)])


def kr() -> Workload:
    """Kr, Z=36, closed shell: 120 STOs zeta = 0.2*1.45^k (s 32, p 10x3, d 6x5, f 4x7); 200 x Lebedev-77."""
    basis = even_tempered(budget_counts(30, 120), 0.2, 1.45)
    return Workload("Kr", 36, basis, nrad=200, order=77, n_up=18, n_down=18)


_BATCH_ORDERS = [17, 19, 21, 23, 25, 27, 29, 31, 35, 41, 47, 53, 59]


def batch(seed: int = 20261203, count: int = 64) -> list[Workload]:
    """64 closed-shell atoms/ions: Z ~ U{2..36} (odd Z -> cation with Z-1 electrons), nb ~ U{10..80},
    zeta_k = 0.3*1.7^k, radial ~ U{40..200}, Lebedev order ~ U{17..59}."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(count):
        Z = int(rng.integers(2, 37))
        ne_ = Z if Z % 2 == 0 else Z - 1
        target = int(rng.integers(10, 81))
        target = max(target, ne_ // 2 + 1)
        basis = even_tempered(budget_counts(max(target // 4, 1), target), 0.3, 1.7)
        nrad = int(rng.integers(40, 201))
        order = int(rng.choice(_BATCH_ORDERS))
        out.append(Workload(f"batch{i}-Z{Z}", Z, basis, nrad=nrad, order=order, n_up=ne_ // 2, n_down=ne_ // 2))
    return out

"""Generates tests/golden/*.json from the reference sources (run in a container where the reference
checkout is mounted; GPU test runs only read the committed fixtures).

  python tests/golden/make_golden.py /path/to/tcscf

* lebedev_reference.json: for the Lebedev orders the workloads use, the point count, the sorted
  distinct weights and the sorted polar angles of the reference tables
  (src/integration/data/LebedevData_<order>.hpp); the library's scipy-sourced rules are checked
  against them.
* known_answers.json: the asserted known answers of the reference's unit tests, with their
  tolerances and file:line.
"""
from __future__ import annotations

import json
import re
import sys
from pathlib import Path

ORDERS = [3, 11, 17, 41, 59, 77]


def _threej(j1, j2, j3, m1, m2, m3):
    """Wigner 3j symbol by the Racah formula (integer arguments)."""
    from math import factorial as f, sqrt
    if m1 + m2 + m3 != 0 or not abs(j1 - j2) <= j3 <= j1 + j2 or abs(m1) > j1 or abs(m2) > j2 or abs(m3) > j3:
        return 0.0
    pre = (-1) ** (j1 - j2 - m3) * sqrt(f(j1 + j2 - j3) * f(j1 - j2 + j3) * f(-j1 + j2 + j3) / f(j1 + j2 + j3 + 1)
                                        * f(j1 + m1) * f(j1 - m1) * f(j2 + m2) * f(j2 - m2) * f(j3 + m3) * f(j3 - m3))
    total = 0.0
    for k in range(j1 + j2 + j3 + 1):
        d = [k, j1 + j2 - j3 - k, j1 - m1 - k, j2 + m2 - k, j3 - j2 + m1 + k, j3 - j1 - m2 + k]
        if min(d) >= 0:
            den = 1
            for x in d:
                den *= f(x)
            total += (-1) ** k / den
    return pre * total


def hydrogen_coulomb(na, la, ma, nb, lb, mb):
    """Coulomb integral J = <a b|1/r12|a b> of hydrogen-like Z = 1 functions by the Slater-Condon
    expansion J = sum_k c^k(la ma, la ma) c^k(lb mb, lb mb) F^k(a, b), the radial F^k on a dense
    trapezoid grid with Richardson extrapolation (about 1e-10 absolute)."""
    import numpy as np
    from math import factorial as f, sqrt
    from scipy import special

    def radial(n, l, r):
        beta = 1.0 / n
        norm = sqrt((2 * beta) ** (2 * l + 3) * f(n - l - 1) / (2 * n * f(n + l)))
        return norm * r ** l * special.eval_genlaguerre(n - l - 1, 2 * l + 1, 2 * beta * r) * np.exp(-beta * r)

    def ck(l, m, k):
        return (-1) ** m * (2 * l + 1) * _threej(l, k, l, 0, 0, 0) * _threej(l, k, l, -m, 0, m)

    def fk(k, npts):
        r = np.linspace(0.0, 400.0, npts)[1:]
        h = r[1] - r[0]
        pa = (radial(na, la, r) * r) ** 2
        pb = (radial(nb, lb, r) * r) ** 2
        inner = np.cumsum(pb * r ** k) * h - 0.5 * h * pb * r ** k
        outer = (np.cumsum((pb / r ** (k + 1))[::-1]) * h)[::-1] - 0.5 * h * pb / r ** (k + 1)
        return float(np.sum(pa * (inner / r ** (k + 1) + outer * r ** k)) * h)

    total = 0.0
    for k in range(0, 2 * min(la, lb) + 1, 2):
        coeff = ck(la, ma, k) * ck(lb, mb, k)
        if coeff != 0.0:
            coarse, fine = fk(k, 1_000_001), fk(k, 2_000_001)
            total += coeff * (fine + (fine - coarse) / 3)
    return total


def parse_table(path: Path):
    rows = re.findall(r"\{\s*([-0-9.eE]+)L,\s*([-0-9.eE]+)L,\s*([-0-9.eE]+)L\s*\}", path.read_text())
    return [(float(a), float(b), float(c)) for a, b, c in rows]


def main(ref: Path) -> None:
    here = Path(__file__).resolve().parent
    out = {}
    for order in ORDERS:
        rows = parse_table(ref / "src/integration/data" / f"LebedevData_{order}.hpp")
        weights = sorted({round(r[2], 15) for r in rows})
        thetas = sorted(round(r[0], 15) for r in rows)
        out[str(order)] = {"npoints": len(rows), "distinct_weights": weights, "sorted_theta": thetas,
                           "weight_sum": sum(r[2] for r in rows)}
    (here / "lebedev_reference.json").write_text(json.dumps(out, indent=1))
    known = {
        "chebyshev_linear": {"n": 100, "value": 0.0, "tol": 3e-16, "src": "src/unitTests/IntegrationTest.cpp:19-29"},
        "chebyshev_quadratic": {"n": 1000, "value": 2.0 / 3.0, "tol": 1e-5, "src": "src/unitTests/IntegrationTest.cpp:32-43"},
        "chebyshev_cubic": {"n": 1000, "value": 2.0, "tol": 1e-5, "src": "src/unitTests/IntegrationTest.cpp:46-57"},
        "radial_exponential": {"n": 100, "value": 1.0, "tol": 1e-7, "src": "src/unitTests/IntegrationTest.cpp:76-89"},
        "radial_exp_polynomial": {"n": 100, "value": -20.0 / 27.0, "tol": 1e-10, "src": "src/unitTests/IntegrationTest.cpp:92-105"},
        "lebedev_constant": {"order": 3, "value": 12.566370614359172, "tol": 3e-14, "src": "src/unitTests/IntegrationTest.cpp:142-154"},
        "lebedev_ylm_tol_per_degree": {"value": 3e-15, "src": "src/unitTests/IntegrationTest.cpp:157-197"},
        "sto_overlap": {"radial": 1000, "order": 11, "epsilon": 1.0, "alpha1": 1.524, "alpha2": 2.532, "tol": 1e-14,
                        "src": "src/unitTests/SlaterTypeOrbitalTest.cpp:14-47"},
        "ochi_gradient": {"a": 1.5, "c_oppo": 0.75, "c_same": 0.375, "h": 2.0 ** -15, "tol": 1e-8, "r1": [1, 1, 1],
                          "range": [-5, 5], "samples": 100, "src": "src/unitTests/gradientsTest.cpp:59-93"},
        "he_literature": {"hf": -2.861700, "exact": -2.903700, "src": "src/unitTests/HartreeFockTest.cpp:591-602"},
    }
    # r12 Coulomb integrals of hydrogen-like Z = 1 functions (n, l, m): the reference's printed expected
    # values and error bars (never asserted there) and the exact values by Slater-Condon
    cases = [("first", (2, 1, 0), (2, 1, 0), 0.196207, 0.0018, "src/unitTests/IntegrationTest.cpp:369-399"),
             ("second", (2, 1, 0), (2, 1, 1), 0.174825, 0.000862, "src/unitTests/IntegrationTest.cpp:402-447"),
             ("third", (4, 3, 2), (3, 2, -1), 0.000451565, 0.000064, "src/unitTests/IntegrationTest.cpp:450-483"),
             ("fourth", (4, 2, -2), (5, 3, 1), 0.0317012, 0.0001, "src/unitTests/IntegrationTest.cpp:485-520"),
             ("s_p", (1, 0, 0), (2, 1, 0), None, None, "closed form F0(1s,2p) = 59/243")]
    # the reference's recorded He study (convergence.sh: RCS, Ochi s functions n = 0..nMax with
    # -n 1..9 -l 0 -a 1.355, QMC grids --r1 2000 --r2 1000; data.txt: mean and standard deviation
    # over ten grid draws per basis size)
    rows = []
    for line in (ref / "data.txt").read_text().splitlines()[1:]:
        f = [x.strip() for x in line.split(",")]
        if len(f) >= 5:
            rows.append([int(f[0]), float(f[3]), float(f[4])])
    script = (ref / "convergence.sh").read_text()
    alpha = float(re.search(r"-a\s+([0-9.]+)", script).group(1))
    known["he_ochi_study"] = {"Z": 2, "alpha": alpha, "l_max": 0, "rows_nbasis_energy_std": rows,
                              "src": "data.txt:1-10 (settings convergence.sh:3-6)"}
    known["r12_hydrogen"] = [{"name": n, "a": list(a), "b": list(b), "reference_value": v, "reference_error": e,
                              "exact": hydrogen_coulomb(*a, *b), "src": src} for n, a, b, v, e, src in cases]
    (here / "known_answers.json").write_text(json.dumps(known, indent=1))


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/make_golden.py /path/to/tcscf")
    main(Path(sys.argv[1]))

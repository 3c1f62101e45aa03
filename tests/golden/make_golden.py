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
    (here / "known_answers.json").write_text(json.dumps(known, indent=1))


if __name__ == "__main__":
    main(Path(sys.argv[1] if len(sys.argv) > 1 else "/root/reference"))

"""The C++ host layer's device paths on the GPU: include/tcscf_gpu.hpp compiled with g++ against
libtcscf_gpu.so (tests/cpp/shim_host.cpp) and run with the device visible.  Its He SCF through
RCSHartreeFock::compute and its device-loop form, the FP64 and split-BF16 fockBuild at the converged
density and the UOS SCF are
checked against the oracle's SCF on the same grid and basis (RCSHartreeFock::compute,
HartreeFock.cpp:785-882): the energies within 1e-8 Eh (the two sides use different eigen-solvers and
converge to 1e-10)."""
import os
import shutil
import subprocess
from pathlib import Path

import numpy as np
import pytest

import oracle
from tcscf_b200 import build, ffi

from .test_load_sto import HE_FILE

pytestmark = pytest.mark.gpu

ROOT = Path(__file__).resolve().parent.parent


def _octahedron():
    w = 4 * np.pi / 6
    return np.array([[np.pi / 2, 0, w], [np.pi / 2, np.pi, w], [np.pi / 2, np.pi / 2, w], [np.pi / 2, 3 * np.pi / 2, w],
                     [0, 0, w], [np.pi, 0, w]])


@pytest.mark.skipif(shutil.which("g++") is None, reason="needs g++")
def test_cpp_host_layer_device_paths_match_oracle(tmp_path):
    lib = build.build()
    exe = tmp_path / "shim_host"
    cmd = ["g++", "-std=c++17", "-O1", "-Wall", "-Wextra", "-Werror", "-I", str(ROOT / "include"), str(ROOT / "tests/cpp/shim_host.cpp"),
           "-L", str(lib.parent), "-ltcscf_gpu", f"-Wl,-rpath,{lib.parent}", "-o", str(exe)]
    res = subprocess.run(cmd, capture_output=True, text=True)
    assert res.returncode == 0, res.stderr[-4000:]
    d = tmp_path / "basis" / "TZ3P"
    d.mkdir(parents=True)
    (d / "He").write_text(HE_FILE)
    run = subprocess.run([str(exe), str(tmp_path / "basis")], capture_output=True, text=True, timeout=600, env=dict(os.environ))
    assert run.returncode == 0, run.stdout + run.stderr
    assert "0 failure(s)" in run.stdout and "no device" not in run.stdout, run.stdout
    vals = {}
    for line in run.stdout.splitlines():
        parts = line.split()
        if len(parts) == 2 and parts[0].isupper():
            vals[parts[0]] = float(parts[1])
    # the oracle on the same grid (40 radial points, r = (1+x)/(1-x), octahedral angular rule) and basis
    basis = [(0.9 * 1.8 ** k, 1, 0, 0) for k in range(6)]
    r, wr = oracle.radial_grid(40, ffi.MAP_ONE_PLUS_X)
    pts, w = oracle.product_grid(r, wr, _octahedron())
    vals1 = oracle.basis_values(pts, basis)
    F = oracle.compute_F(pts, pts, w, vals1, len(basis))
    S, h = oracle.overlap_core(basis, 2)
    st, E, it, D, eig = oracle.scf(1, 1, 1, F, vals1, w, S, h, tol=1e-10, max_iter=50)
    assert st == 0
    assert abs(vals["E_SCF"] - E) < 1e-8, (vals["E_SCF"], E)
    assert abs(vals["E_FOCK_FP64"] - E) < 1e-8
    assert abs(vals["E_FOCK_BF16X3"] - E) < 1e-6
    assert abs(vals["E_UOS"] - E) < 1e-8
    assert abs(vals["E_GRAPH"] - E) < 1e-8
    assert vals["S_QUAD_ERR"] < 1e-6

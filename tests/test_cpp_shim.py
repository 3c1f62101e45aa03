"""The C++ host layer include/tcscf_gpu.hpp compiles with g++ against libtcscf_gpu.so, and its
host-side paths (grids, loadSTO, analytic S / H, the error mapping) run and give the known answers
(tests/cpp/shim_host.cpp).  Without a device the program checks that Context throws
Error(TCSCF_ERR_NO_DEVICE); its device paths are compiled in every run and run only where a
context can be created (devices are hidden here)."""
import os
import shutil
import subprocess
from pathlib import Path

import pytest

from tcscf_b200 import build

from .test_load_sto import HE_FILE

ROOT = Path(__file__).resolve().parent.parent


@pytest.mark.skipif(shutil.which("g++") is None, reason="needs g++")
def test_cpp_host_layer_compiles_and_runs(tmp_path):
    lib = build.build()
    exe = tmp_path / "shim_host"
    cmd = ["g++", "-std=c++17", "-O1", "-Wall", "-Wextra", "-Werror", "-I", str(ROOT / "include"), str(ROOT / "tests/cpp/shim_host.cpp"),
           "-L", str(lib.parent), "-ltcscf_gpu", f"-Wl,-rpath,{lib.parent}", "-o", str(exe)]
    res = subprocess.run(cmd, capture_output=True, text=True)
    assert res.returncode == 0, res.stderr[-4000:]
    d = tmp_path / "basis" / "TZ3P"
    d.mkdir(parents=True)
    (d / "He").write_text(HE_FILE)
    # devices hidden: this test covers the host layer (the device paths are compiled, not run)
    env = dict(os.environ, CUDA_VISIBLE_DEVICES="")
    run = subprocess.run([str(exe), str(tmp_path / "basis")], capture_output=True, text=True, timeout=300, env=env)
    assert run.returncode == 0, run.stdout + run.stderr
    assert "0 failure(s)" in run.stdout

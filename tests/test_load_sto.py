"""loadSTO (SlaterTypeOrbital.cpp:24-75) on basis-set files written here in the ADF library format
(the reference's own library is not copied: the files below hold made-up exponents)."""
import numpy as np
import pytest

from tcscf_b200 import api, ffi

HE_FILE = """Helium (made-up exponents for the loader tests)

BASIS
1S  2.90
1S  1.40
2S  0.80
2P  2.10
2P  1.00

3D  1.50
4F  2.20
END

CORE    0  0  0  0
END
"""


def _library(tmp_path, name="TZ3P", element="He", text=HE_FILE):
    d = tmp_path / name
    d.mkdir(parents=True)
    (d / element).write_text(text)
    return tmp_path


def test_load_sto_expands_m_and_filters_l(tmp_path):
    lib = _library(tmp_path)
    b = api.loadSTO(lib, "TZ3P", "He", 3)
    # 3 s + 2 x 3 p + 5 d + 7 f, in file order, m = -l..l (SlaterTypeOrbital.cpp:57-62)
    assert len(b) == 3 + 6 + 5 + 7
    assert b[:3] == [(2.9, 1, 0, 0), (1.4, 1, 0, 0), (0.8, 2, 0, 0)]
    assert b[3:6] == [(2.1, 2, 1, -1), (2.1, 2, 1, 0), (2.1, 2, 1, 1)]
    assert [f[3] for f in b[9:14]] == [-2, -1, 0, 1, 2] and b[9][:3] == (1.5, 3, 2)
    assert len(api.loadSTO(lib, "TZ3P", "He", 1)) == 9     # d and f dropped
    assert len(api.loadSTO(lib, "TZ3P", "He", 0)) == 3


def test_load_sto_errors(tmp_path):
    lib = _library(tmp_path)
    with pytest.raises(ffi.TcscfError) as e:
        api.loadSTO(lib, "DZ", "He", 3)                    # not one of TZ3P, QZ6P, ATZ3P, AQZ6P
    assert e.value.code == ffi.ERR_INVALID_ARGUMENT
    with pytest.raises(ffi.TcscfError) as e:
        api.loadSTO(lib, "QZ6P", "He", 3)                  # basis-set directory missing
    assert e.value.code == ffi.ERR_INVALID_ARGUMENT
    assert api.loadSTO(lib, "TZ3P", "Ne", 3) == []         # missing element file: empty, as the reference
    bad = _library(tmp_path / "x", element="Li", text="BASIS\n1S 3.0\nnot a line\nEND\n")
    with pytest.raises(ffi.TcscfError) as e:
        api.loadSTO(bad, "TZ3P", "Li", 3)
    assert e.value.code == ffi.ERR_INVALID_ARGUMENT


@pytest.mark.gpu
def test_loaded_basis_runs_scf(ctx, tmp_path):
    # the loaded basis through the device grid, the analytic S / H and the FP64 RCS SCF
    from tcscf_b200 import grids
    import oracle
    b = api.loadSTO(_library(tmp_path), "TZ3P", "He", 1)
    g = grids.product_grid(40, 11)
    G = api.QMCGrid(ctx, g)
    G.setBasisFunctions(b)
    S, h = api.overlap_core(b, 2)
    vals = oracle.basis_values(g.points, b)
    F = oracle.compute_F(g.points, g.points, g.weights, vals, len(b))
    st, Er, itr, Dr, eig = oracle.scf(1, 1, 1, F, vals, g.weights, S, h, tol=1e-8, max_iter=50)
    assert st == 0
    Eg = api.RCSHartreeFock(1, 1, len(b)).compute(S, h, G, G, tol=1e-8)
    assert abs(Eg - Er) < 1e-10, (Eg, Er)

"""ORACLE — test infrastructure only.

ctypes bindings of the CPU restatement in oracle/tcscf_oracle.cpp (built into
oracle/_build/liboracle.so by oracle/Makefile).  Only tests/, __graft_entry__.smoke() and bench.py's
cpu_baseline / reference arm may import this package, and only as the parity reference or the timed
CPU baseline; the product library never touches it.
"""
from __future__ import annotations

import ctypes as C
import glob
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "_build" / "liboracle.so"
_lib = None

_D = C.POINTER(C.c_double)


class Sto(C.Structure):
    _fields_ = [("alpha", C.c_double), ("n", C.c_int32), ("l", C.c_int32), ("m", C.c_int32), ("family", C.c_int32)]


class Ochi(C.Structure):
    _fields_ = [("a", C.c_double), ("a12", C.c_double), ("nterms", C.c_int32), ("pad", C.c_int32),
                ("S", (C.c_int32 * 3) * 8), ("c", (C.c_double * 2) * 8)]


def build() -> Path:
    src = HERE / "tcscf_oracle.cpp"
    if not LIB.exists() or LIB.stat().st_mtime < src.stat().st_mtime:
        subprocess.run(["make", "-s", "-C", str(HERE)], check=True)
    return LIB


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        build()
        _lib = C.CDLL(str(LIB))
        _lib.oracle_product_grid.restype = None
        _lib.oracle_kernel_values.restype = None
        for name in ("oracle_fock_build", "oracle_tc_fock_build", "oracle_ochi_value", "oracle_ochi_laplacian", "oracle_sto_normalization"):
            getattr(_lib, name).restype = C.c_double
        _lib.oracle_ochi_value.argtypes = [C.POINTER(Ochi), C.c_double, C.c_double, C.c_double, C.c_int]
        _lib.oracle_sto_normalization.argtypes = [C.c_double, C.c_int]
        _lib.oracle_sph_harmonic.argtypes = [C.c_int, C.c_int, C.c_double, C.c_double, _D]
        paths = sorted(glob.glob(os.path.join(os.path.dirname(np.__file__), "..", "scipy.libs", "libscipy_openblas*.so")))
        if paths:
            _lib.oracle_set_lapack(paths[0].encode())
    return _lib


def _p(a):
    if a is None:
        return None
    assert a.flags.c_contiguous and a.dtype in (np.float64, np.complex128), (a.dtype, a.flags)
    return a.ctypes.data_as(_D)


def _sto(basis):
    arr = (Sto * len(basis))()
    for i, b in enumerate(basis):
        arr[i].alpha, arr[i].n, arr[i].l, arr[i].m = float(b[0]), int(b[1]), int(b[2]), int(b[3])
        arr[i].family = int(b[4]) if len(b) > 4 else 0
    return arr


def ochi(a: float, a12: float, terms) -> Ochi:
    o = Ochi()
    o.a, o.a12, o.nterms = float(a), float(a12), len(terms)
    for t, (S, c_oppo, c_same) in enumerate(terms):
        for d in range(3):
            o.S[t][d] = int(S[d])
        o.c[t][0], o.c[t][1] = float(c_oppo), float(c_same)
    return o


def set_threads(n: int) -> None:
    lib().oracle_set_threads(int(n))


def threads() -> int:
    return lib().oracle_get_threads()


def radial_grid(n: int, map_: int, p0: float = 0.0, p1: float = 0.0):
    u, w = np.empty(n), np.empty(n)
    lib().oracle_radial_grid(n, map_, C.c_double(p0), C.c_double(p1), _p(u), _p(w))
    return u, w


def product_grid(r, wr, ang):
    nrad, nang = len(r), ang.shape[0]
    N = nrad * nang
    pts, w = np.empty((3, N)), np.empty(N)
    lib().oracle_product_grid(nrad, _p(np.ascontiguousarray(r)), _p(np.ascontiguousarray(wr)), nang,
                              _p(np.ascontiguousarray(ang)), _p(pts), _p(w))
    return pts, w


def qmc_grid(u: np.ndarray):
    ndim, N = u.shape
    pts, w = np.empty((ndim, N)), np.empty(N)
    lib().oracle_qmc_grid(ndim, C.c_int64(N), _p(np.ascontiguousarray(u)), _p(pts), _p(w))
    return pts, w


def basis_values(points: np.ndarray, basis, gradients: bool = False):
    ndim, N = points.shape
    nb = len(basis)
    vals = np.empty((N, nb), dtype=np.complex128 if ndim == 3 else np.float64)
    grads = np.empty((N, nb, 3), dtype=np.complex128) if gradients else None
    lib().oracle_basis_values(_p(np.ascontiguousarray(points)), C.c_int64(N), ndim, _sto(basis), nb, _p(vals), _p(grads))
    return (vals, grads) if gradients else vals


def sph_harmonic(l: int, m: int, theta: float, phi: float) -> complex:
    out = np.empty(2)
    lib().oracle_sph_harmonic(l, m, theta, phi, _p(out))
    return complex(out[0], out[1])


def sto_normalization(alpha: float, n: int) -> float:
    return lib().oracle_sto_normalization(alpha, n)


def overlap_core(basis, Z: int):
    nb = len(basis)
    S, H = np.empty((nb, nb)), np.empty((nb, nb))
    lib().oracle_overlap_core(_sto(basis), nb, Z, _p(S), _p(H))
    return S, H


def quadrature_overlap_core(points, weights, vals, grads, Z: int):
    N, nb = vals.shape
    S = np.empty((nb, nb), dtype=np.complex128)
    H = np.empty((nb, nb), dtype=np.complex128) if grads is not None else None
    lib().oracle_quadrature_overlap_core(_p(np.ascontiguousarray(points)), _p(np.ascontiguousarray(weights)), C.c_int64(N),
                                         _p(vals), _p(grads), nb, Z, _p(S), _p(H))
    return S, H


def ochi_value(u: Ochi, r1, r2, r12, same: bool) -> float:
    return lib().oracle_ochi_value(C.byref(u), r1, r2, r12, int(same))


def ochi_gradient(u: Ochi, p1, p2, same: bool) -> np.ndarray:
    out = np.empty(3)
    lib().oracle_ochi_gradient(C.byref(u), _p(np.asarray(p1, dtype=np.float64)), _p(np.asarray(p2, dtype=np.float64)), int(same), _p(out))
    return out


def kernel_values(kernel: int, u: Ochi | None, p1: np.ndarray, p2: np.ndarray) -> np.ndarray:
    N1, N2 = p1.shape[1], p2.shape[1]
    out = np.empty((N1, N2, 3)) if kernel >= 3 else np.empty((N1, N2))
    lib().oracle_kernel_values(kernel, C.byref(u) if u else None, _p(np.ascontiguousarray(p1)), C.c_int64(N1),
                               _p(np.ascontiguousarray(p2)), C.c_int64(N2), p2.shape[0], _p(out))
    return out


def compute_F(p1, p2, w2, vals2, basis_n: int, kernel: int = 0, u: Ochi | None = None):
    N1, N2 = p1.shape[1], p2.shape[1]
    cx = p2.shape[0] == 3
    F = np.empty((N1, basis_n, basis_n), dtype=np.complex128 if cx else np.float64)
    lib().oracle_compute_F(_p(np.ascontiguousarray(p1)), C.c_int64(N1), _p(np.ascontiguousarray(p2)), _p(np.ascontiguousarray(w2)),
                           C.c_int64(N2), p2.shape[0], _p(np.ascontiguousarray(vals2)), basis_n, kernel, C.byref(u) if u else None, _p(F))
    return F


def compute_V(p1, p2, w2, vals2, basis_n: int, kernel: int, u: Ochi):
    N1, N2 = p1.shape[1], p2.shape[1]
    V = np.empty((N1, basis_n, basis_n, 3), dtype=np.complex128)
    lib().oracle_compute_V(_p(np.ascontiguousarray(p1)), C.c_int64(N1), _p(np.ascontiguousarray(p2)), _p(np.ascontiguousarray(w2)),
                           C.c_int64(N2), _p(np.ascontiguousarray(vals2)), basis_n, kernel, C.byref(u), _p(V))
    return V


def integrate_all_r1r2(use_gradient: bool, p1, w1, vals1, p2, w2, vals2, grads2, nb: int, kernel: int, u: Ochi | None):
    """integrateAllR1R2 (r1 3-D complex values, r2 2-D real values / complex gradients): [nb]^4 complex."""
    out = np.empty((nb,) * 4, dtype=np.complex128)
    lib().oracle_integrate_all_r1r2(int(use_gradient), _p(np.ascontiguousarray(p1)), _p(np.ascontiguousarray(w1)),
                                    C.c_int64(p1.shape[1]), _p(np.ascontiguousarray(vals1)), _p(np.ascontiguousarray(p2)),
                                    _p(np.ascontiguousarray(w2)), C.c_int64(p2.shape[1]), _p(np.ascontiguousarray(vals2)),
                                    _p(None if grads2 is None else np.ascontiguousarray(grads2)), nb, kernel,
                                    C.byref(u) if u else None, _p(out))
    return out


def three_electron_integrals(p1, w1, vals1, p2, w2, vals2, nb: int, u: Ochi):
    """threeElectronIntegrals (same-spin grad u): [nb]^6 complex."""
    out = np.empty((nb,) * 6, dtype=np.complex128)
    lib().oracle_three_electron_integrals(_p(np.ascontiguousarray(p1)), _p(np.ascontiguousarray(w1)), C.c_int64(p1.shape[1]),
                                          _p(np.ascontiguousarray(vals1)), _p(np.ascontiguousarray(p2)), _p(np.ascontiguousarray(w2)),
                                          C.c_int64(p2.shape[1]), _p(np.ascontiguousarray(vals2)), nb, C.byref(u), _p(out))
    return out


def fock_build(F, vals1, w1, D, h, respect_symmetry: bool = True):
    D = np.ascontiguousarray(D, dtype=np.complex128)
    if D.ndim == 2:
        D = D[None]
    nspin, nb = D.shape[0], D.shape[1]
    N1 = vals1.shape[0]
    G = np.empty((nspin, nb, nb), dtype=np.complex128)
    Fock = np.empty((nspin, nb, nb), dtype=np.complex128)
    e = lib().oracle_fock_build(nspin, int(np.iscomplexobj(F)), _p(np.ascontiguousarray(F)), C.c_int64(N1), nb, _p(vals1),
                                _p(np.ascontiguousarray(w1)), _p(D), _p(np.ascontiguousarray(h, dtype=np.float64)),
                                int(respect_symmetry), _p(G), _p(Fock))
    return G, Fock, e


def scf(nspin: int, n_up: int, n_down: int, F, vals1, w1, S, h, respect_symmetry=True, tol=1e-5, max_iter=50):
    nb = vals1.shape[1]
    N1 = vals1.shape[0]
    e = C.c_double()
    it = C.c_int()
    D = np.empty((nspin, nb, nb), dtype=np.complex128)
    eig = np.empty((nspin, nb))
    st = lib().oracle_scf(nspin, n_up, n_down, int(np.iscomplexobj(F)), _p(np.ascontiguousarray(F)), C.c_int64(N1), nb, _p(vals1),
                          _p(np.ascontiguousarray(w1)), _p(np.ascontiguousarray(S, dtype=np.float64)),
                          _p(np.ascontiguousarray(h, dtype=np.float64)), int(respect_symmetry), C.c_double(tol), max_iter,
                          C.byref(e), C.byref(it), _p(D), _p(eig))
    return st, e.value, it.value, D, eig


def tc_fock_build(Fs, Fo, Vs, Vo, vals1, grads1, w1, D, n_up, n_down, occ_up, occ_down, h, respect_symmetry=True):
    nb = vals1.shape[1]
    N1 = vals1.shape[0]
    G2 = np.empty((2, nb, nb), dtype=np.complex128)
    G3 = np.empty((2, nb, nb), dtype=np.complex128)
    Fock = np.empty((2, nb, nb), dtype=np.complex128)
    e = lib().oracle_tc_fock_build(int(np.iscomplexobj(Fs)), _p(Fs), _p(Fo), _p(Vs), _p(Vo), C.c_int64(N1), nb, _p(vals1), _p(grads1),
                                   _p(np.ascontiguousarray(w1)), _p(np.ascontiguousarray(D, dtype=np.complex128)), n_up, n_down,
                                   _p(np.ascontiguousarray(occ_up, dtype=np.complex128)), _p(np.ascontiguousarray(occ_down, dtype=np.complex128)),
                                   _p(np.ascontiguousarray(h, dtype=np.float64)), int(respect_symmetry), _p(G2), _p(G3), _p(Fock))
    return G2, G3, Fock, e


def tc_scf(Fs, Fo, Vs, Vo, vals1, grads1, w1, S, h, n_up, n_down, respect_symmetry=True, tol=1e-5, max_iter=200):
    nb = vals1.shape[1]
    N1 = vals1.shape[0]
    e = C.c_double()
    it = C.c_int()
    D = np.empty((2, nb, nb), dtype=np.complex128)
    pe = np.zeros((2, nb))
    st = lib().oracle_tc_scf(int(np.iscomplexobj(Fs)), _p(Fs), _p(Fo), _p(Vs), _p(Vo), C.c_int64(N1), nb, _p(vals1), _p(grads1),
                             _p(np.ascontiguousarray(w1)), _p(np.ascontiguousarray(S, dtype=np.float64)),
                             _p(np.ascontiguousarray(h, dtype=np.float64)), n_up, n_down, int(respect_symmetry), C.c_double(tol),
                             max_iter, C.byref(e), C.byref(it), _p(D), _p(pe))
    return st, e.value, it.value, D, pe


def mgs(vectors: np.ndarray, metric_col_major: np.ndarray | None = None) -> np.ndarray:
    v = np.ascontiguousarray(vectors, dtype=np.complex128).copy()
    lib().oracle_mgs(_p(v), v.shape[0], v.shape[1], _p(None if metric_col_major is None else np.ascontiguousarray(metric_col_major, dtype=np.complex128)))
    return v


def compute_q(w1, vals1, Vs, Vo):
    """computeQ (HartreeFock.cpp:613-683): (Qss, Qso, Qoo), each complex [nb]^6."""
    N1, nb = vals1.shape
    out = [np.empty((nb,) * 6, dtype=np.complex128) for _ in range(3)]
    lib().oracle_compute_q(C.c_int64(N1), nb, _p(np.ascontiguousarray(w1)), _p(np.ascontiguousarray(vals1, dtype=np.complex128)),
                           _p(np.ascontiguousarray(Vs)), _p(np.ascontiguousarray(Vo)), _p(out[0]), _p(out[1]), _p(out[2]))
    return tuple(out)


def assemble_g(Qss, Qso, Qoo, D):
    """assembleG (HartreeFock.cpp:687-752): G3 [2][nb][nb] from the Q tensors and the spin densities."""
    nb = Qss.shape[0]
    G3 = np.empty((2, nb, nb), dtype=np.complex128)
    lib().oracle_assemble_g(nb, _p(np.ascontiguousarray(Qss)), _p(np.ascontiguousarray(Qso)), _p(np.ascontiguousarray(Qoo)),
                            _p(np.ascontiguousarray(D, dtype=np.complex128)), _p(G3))
    return G3


# ---- the reference's own hot-path code (oracle/_ref, built by `make -C oracle ref`) ----------------
# oracle/ref_hot_path.cpp compiles the reference's HartreeFock.cpp / HartreeFock.hpp, integration
# headers, SlaterTypeOrbital.hpp and jastrowFunctions.hpp where they lie, over the LvArray / RAJA /
# Caliper / qmc stand-ins in oracle/ref_shim/.  The tests pin the restatement above to it.
REF_LIB = HERE / "_ref" / "libtcscf_ref.so"
_ref = None


def build_ref() -> Path | None:
    """Builds oracle/_ref/libtcscf_ref.so when the reference sources are present; returns its path,
    or None when it is neither built nor buildable here."""
    sources = [HERE / "ref_hot_path.cpp", *HERE.glob("ref_shim/**/*.hpp")]
    stale = not REF_LIB.exists() or any(s.stat().st_mtime > REF_LIB.stat().st_mtime for s in sources)
    if stale:
        res = subprocess.run(["make", "-s", "-C", str(HERE), "ref"], capture_output=True, text=True)
        if res.returncode != 0 and not REF_LIB.exists():
            return None
    return REF_LIB if REF_LIB.exists() else None


def ref_lib() -> C.CDLL | None:
    global _ref
    if _ref is None:
        if build_ref() is None:
            return None
        _ref = C.CDLL(str(REF_LIB))
        paths = sorted(glob.glob(os.path.join(os.path.dirname(np.__file__), "..", "scipy.libs", "libscipy_openblas*.so")))
        if not paths or _ref.tcscf_ref_set_lapack(paths[0].encode()) != 0:
            raise RuntimeError("no LAPACK (scipy's bundled OpenBLAS) for the reference build")
    return _ref


def _c(a):
    return _p(np.ascontiguousarray(a))


def ref_compute_F(p1, w1, vals1, p2, w2, vals2, nb: int, kernel: int = 0, u: Ochi | None = None):
    """precomputeIntegrand + computeF of the reference (HartreeFock.hpp:23-180)."""
    N1, N2, ndim2 = p1.shape[1], p2.shape[1], p2.shape[0]
    F = np.empty((N1, nb, nb), dtype=np.complex128 if ndim2 == 3 else np.float64)
    st = ref_lib().tcscf_ref_compute_F(_c(p1), _c(w1), C.c_int64(N1), _c(vals1), _c(p2), _c(w2), C.c_int64(N2), ndim2, _c(vals2), nb,
                                       kernel, C.byref(u) if u else None, _p(F))
    assert st == 0, st
    return F


def ref_compute_V(p1, w1, vals1, p2, w2, vals2, nb: int, kernel: int, u: Ochi):
    """precomputeIntegrand + computeV of the reference (HartreeFock.hpp:185-229)."""
    N1, N2 = p1.shape[1], p2.shape[1]
    V = np.empty((N1, nb, nb, 3), dtype=np.complex128)
    st = ref_lib().tcscf_ref_compute_V(_c(p1), _c(w1), C.c_int64(N1), _c(vals1), _c(p2), _c(w2), C.c_int64(N2), _c(vals2), nb, kernel,
                                       C.byref(u), _p(V))
    assert st == 0, st
    return V


def ref_scf(nspin: int, n_up: int, n_down: int, F, p1, w1, vals1, S, h, respect_symmetry=True):
    """RCSHartreeFock (nspin 1) / UOSHartreeFock (nspin 2) ::compute of the reference on a real F:
    (convergence loops or -1, energy, density)."""
    nb = vals1.shape[1]
    e = C.c_double()
    D = np.empty((nspin, nb, nb), dtype=np.complex128)
    loops = ref_lib().tcscf_ref_scf(nspin, n_up, n_down, _c(F), _c(p1), _c(w1), C.c_int64(vals1.shape[0]), nb, _c(vals1), _c(S), _c(h),
                                    int(respect_symmetry), C.byref(e), _p(D))
    return loops, e.value, D


def ref_tc_scf(Fs, Fo, Vs, Vo, p1, w1, vals1, grads1, S, h, n_up, n_down, respect_symmetry=True):
    """TCHartreeFock::compute of the reference: (convergence loops or -1, energy, density)."""
    nb = vals1.shape[1]
    e = C.c_double()
    D = np.empty((2, nb, nb), dtype=np.complex128)
    loops = ref_lib().tcscf_ref_tc_scf(_c(Fs), _c(Fo), _c(Vs), _c(Vo), _c(p1), _c(w1), C.c_int64(vals1.shape[0]), nb, _c(vals1), _c(grads1),
                                       _c(S), _c(h), n_up, n_down, int(respect_symmetry), C.byref(e), _p(D))
    return loops, e.value, D


def ref_qmc_grid(u: np.ndarray):
    """Points and weights of the reference's QMCGrid built on the unit-cube points u [ndim][N]."""
    ndim, N = u.shape
    pts, w = np.empty((ndim, N)), np.empty(N)
    assert ref_lib().tcscf_ref_qmc_grid(ndim, C.c_int64(N), _c(u), _p(pts), _p(w)) == 0
    return pts, w


def ref_sto_values(points: np.ndarray, basis, gradients: bool = False):
    """QMCGrid::setBasisFunctions of the reference with SlaterTypeOrbital functions."""
    ndim, N = points.shape
    nb = len(basis)
    vals = np.empty((N, nb), dtype=np.complex128 if ndim == 3 else np.float64)
    grads = np.empty((N, nb, 3), dtype=np.complex128) if gradients else None
    assert ref_lib().tcscf_ref_sto_values(ndim, C.c_int64(N), _c(points), _sto(basis), nb, _p(vals), _p(grads)) == 0
    return (vals, grads) if gradients else vals


def ref_overlap_core(basis, Z: int):
    """The reference's analytic STO overlap and core-Hamiltonian matrices."""
    nb = len(basis)
    S, H = np.empty((nb, nb)), np.empty((nb, nb))
    assert ref_lib().tcscf_ref_overlap_core(_sto(basis), nb, Z, _p(S), _p(H)) == 0
    return S, H


def ref_family_values(points: np.ndarray, basis, gradients: bool = False):
    """QMCGrid::setBasisFunctions of the reference with Ochi (family 1) or hydrogen-like (family 2) functions."""
    ndim, N = points.shape
    nb = len(basis)
    vals = np.empty((N, nb), dtype=np.complex128 if ndim == 3 else np.float64)
    grads = np.empty((N, nb, 3), dtype=np.complex128) if gradients else None
    assert ref_lib().tcscf_ref_family_values(ndim, C.c_int64(N), _c(points), _sto(basis), nb, _p(vals), _p(grads)) == 0
    return (vals, grads) if gradients else vals


def ref_family_overlap_core(basis, Z: int):
    """S and core H of an Ochi / hydrogen-like basis as the reference's driver fills them (S NaN for
    the hydrogen-like family, whose overlap the reference integrates numerically)."""
    nb = len(basis)
    S, H = np.empty((nb, nb)), np.empty((nb, nb))
    assert ref_lib().tcscf_ref_family_overlap_core(_sto(basis), nb, Z, _p(S), _p(H)) == 0
    return S, H


def ref_integrate_all_r1r2(use_gradient: bool, p1, w1, vals1, p2, w2, vals2, grads2, nb: int, kernel: int, u: Ochi | None):
    """integrateAllR1R2 of the reference: [nb]^4 complex."""
    out = np.empty((nb,) * 4, dtype=np.complex128)
    st = ref_lib().tcscf_ref_integrate_all_r1r2(int(use_gradient), _c(p1), _c(w1), C.c_int64(p1.shape[1]), _c(vals1), _c(p2), _c(w2),
                                                C.c_int64(p2.shape[1]), _c(vals2), _p(None if grads2 is None else np.ascontiguousarray(grads2)),
                                                nb, kernel, C.byref(u) if u else None, _p(out))
    assert st == 0, st
    return out


def ref_three_electron_integrals(p1, w1, vals1, p2, w2, vals2, nb: int, u: Ochi):
    """threeElectronIntegrals of the reference: [nb]^6 complex."""
    out = np.empty((nb,) * 6, dtype=np.complex128)
    st = ref_lib().tcscf_ref_three_electron_integrals(_c(p1), _c(w1), C.c_int64(p1.shape[1]), _c(vals1), _c(p2), _c(w2), C.c_int64(p2.shape[1]),
                                                      _c(vals2), nb, C.byref(u), _p(out))
    assert st == 0, st
    return out


def ref_compute_q(w1, vals1, Vs, Vo):
    """internal::computeQ of the reference: (Qss, Qso, Qoo), each complex [nb]^6."""
    N1, nb = vals1.shape
    out = [np.empty((nb,) * 6, dtype=np.complex128) for _ in range(3)]
    st = ref_lib().tcscf_ref_compute_q(C.c_int64(N1), nb, _c(w1), _c(np.asarray(vals1, dtype=np.complex128)), _c(Vs), _c(Vo), _p(out[0]),
                                       _p(out[1]), _p(out[2]))
    assert st == 0, st
    return tuple(out)


def ref_assemble_g(Qss, Qso, Qoo, D):
    """internal::assembleG of the reference: G3 [2][nb][nb]."""
    nb = Qss.shape[0]
    G3 = np.empty((2, nb, nb), dtype=np.complex128)
    st = ref_lib().tcscf_ref_assemble_g(nb, _c(Qss), _c(Qso), _c(Qoo), _c(np.asarray(D, dtype=np.complex128)), _p(G3))
    assert st == 0, st
    return G3


def ref_load_sto(directory, basis_set: str, element: str, max_l: int):
    """loadSTO of the reference: [(alpha, n, l, m)], or None when the reference's loader rejects the arguments."""
    out = (Sto * 4096)()
    n = ref_lib().tcscf_ref_load_sto(str(directory).encode(), basis_set.encode(), element.encode(), max_l, out, 4096)
    if n < 0:
        return None
    assert n <= 4096
    return [(out[i].alpha, out[i].n, out[i].l, out[i].m) for i in range(n)]


def ref_basis_library() -> Path | None:
    """The reference's basis-set library directory the reference build was given (None if absent)."""
    f = ref_lib().tcscf_ref_basis_library
    f.restype = C.c_char_p
    p = Path(f().decode())
    return p if str(p) and p.is_dir() else None


def ref_radial_grid(n: int, map_: int, p0: float = 0.0, p1: float = 0.0):
    """createGrid(ChebyshevGauss(n), map) of the reference (maps 0-3: None, Linear, XOver1mX, TreutlerAhlrichsM4)."""
    u, w = np.empty(n), np.empty(n)
    assert ref_lib().tcscf_ref_radial_grid(n, map_, C.c_double(p0), C.c_double(p1), _p(u), _p(w)) == 0
    return u, w

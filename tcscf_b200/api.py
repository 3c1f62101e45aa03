"""Host-side mirror of tcscf's integral / SCF interface, driving libtcscf_gpu.so.

Names follow the reference: QMCGrid.setBasisFunctions (src/integration/integrateAll.hpp:88-137),
computeF / computeV (src/HartreeFock.hpp:88-229), RCSHartreeFock / UOSHartreeFock::compute
(src/HartreeFock.hpp:233-349), overlap / coreMatrixElement (src/SlaterTypeOrbital.hpp:134-181).
Errors are raised as ffi.TcscfError carrying the C status; ConvergenceError mirrors
tcscf::ConvergenceError (src/HartreeFock.hpp:13-19).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import ffi
from .grids import QuadratureGrid


class ConvergenceError(ffi.TcscfError):
    pass


class LinearAlgebraError(ffi.TcscfError):
    pass


def _raise(code: int, ctx) -> None:
    if code == ffi.OK:
        return
    msg = ffi.lib().tcscf_last_error(ctx).decode()
    if code == ffi.ERR_NOT_CONVERGED:
        raise ConvergenceError(code, msg)
    if code == ffi.ERR_LINALG:
        raise LinearAlgebraError(code, msg)
    raise ffi.TcscfError(code, msg)


class Context:
    """One tcscf_ctx (device, stream, cuSOLVER handle, device-resident grids)."""

    def __init__(self, device: int = 0):
        self._h = C.c_void_p()
        code = ffi.lib().tcscf_ctx_create(device, C.byref(self._h))
        if code != ffi.OK:
            raise ffi.TcscfError(code, "tcscf_ctx_create failed (a B200 / sm_100 device is required)")

    @property
    def handle(self):
        return self._h

    def close(self) -> None:
        if self._h:
            ffi.lib().tcscf_ctx_destroy(self._h)
            self._h = C.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def stream(self) -> int:
        s = C.c_void_p()
        _raise(ffi.lib().tcscf_ctx_stream(self._h, C.byref(s)), self._h)
        return s.value or 0

    def synchronize(self) -> None:
        _raise(ffi.lib().tcscf_synchronize(self._h), self._h)

    def batch_graph_stats(self) -> tuple[int, int]:
        """(captures, replays) of the batched builds' CUDA graph on this context."""
        a, b = C.c_int(), C.c_int()
        _raise(ffi.lib().tcscf_batch_graph_stats(self._h, C.byref(a), C.byref(b)), self._h)
        return a.value, b.value

    def set_autotune(self, enable: bool = True) -> None:
        """Measure the tensor-path launch schedule (tile class, then r2 split) per build shape and the
        split policy per batch signature on first use and keep the fastest (off by default)."""
        _raise(ffi.lib().tcscf_set_autotune(self._h, int(bool(enable))), self._h)

    def autotune_stats(self) -> tuple[int, int, int]:
        """(shapes tuned, batch signatures tuned, candidate measurements) on this context."""
        a, b, c = C.c_int(), C.c_int(), C.c_int()
        _raise(ffi.lib().tcscf_autotune_stats(self._h, C.byref(a), C.byref(b), C.byref(c)), self._h)
        return a.value, b.value, c.value

    def last_timing(self) -> tuple[float, float, int]:
        a, b, n = C.c_double(), C.c_double(), C.c_int()
        _raise(ffi.lib().tcscf_last_timing(self._h, C.byref(a), C.byref(b), C.byref(n)), self._h)
        return a.value, b.value, n.value

    def last_potentials(self, n1: int, nb: int):
        """(VH [n1], T [n1][nb]) of the most recent direct Fock build (diagnostics)."""
        VH = np.empty(n1)
        T = np.empty((n1, nb))
        _raise(ffi.lib().tcscf_last_potentials(self._h, ffi.dptr(VH), ffi.dptr(T)), self._h)
        return VH, T


class QMCGrid:
    """Device-resident integration::QMCGrid built from a host QuadratureGrid (points already Cartesian)."""

    def __init__(self, ctx: Context, grid: QuadratureGrid):
        self.ctx = ctx
        self.quadratureGrid = grid
        self._id = C.c_int()
        pts = np.ascontiguousarray(grid.points, dtype=np.float64)
        w = np.ascontiguousarray(grid.weights, dtype=np.float64)
        _raise(ffi.lib().tcscf_grid_create(ctx.handle, ffi.dptr(pts), ffi.dptr(w), grid.n, grid.ndim, C.byref(self._id)), ctx.handle)
        self.basis: list = []
        self.gradients = False

    @property
    def id(self) -> int:
        return self._id.value

    def nGrid(self) -> int:
        return self.quadratureGrid.n

    def nBasis(self) -> int:
        return len(self.basis)

    def setBasisFunctions(self, basis, storeGradients: bool = False) -> None:
        arr = ffi.sto_array(basis)
        _raise(ffi.lib().tcscf_grid_set_basis(self.ctx.handle, self.id, arr, len(basis), int(storeGradients)), self.ctx.handle)
        self.basis = list(basis)
        self.gradients = bool(storeGradients)

    @property
    def basisValues(self) -> np.ndarray:
        n, nb = self.nGrid(), self.nBasis()
        out = np.empty((n, nb), dtype=np.complex128 if self.quadratureGrid.ndim == 3 else np.float64)
        _raise(ffi.lib().tcscf_grid_basis_values(self.ctx.handle, self.id, ffi.dptr(out), None), self.ctx.handle)
        return out

    @property
    def basisGradients(self) -> np.ndarray:
        n, nb = self.nGrid(), self.nBasis()
        out = np.empty((n, nb, 3), dtype=np.complex128)
        _raise(ffi.lib().tcscf_grid_basis_values(self.ctx.handle, self.id, None, ffi.dptr(out)), self.ctx.handle)
        return out

    def close(self) -> None:
        if self._id.value:
            ffi.lib().tcscf_grid_destroy(self.ctx.handle, self.id)
            self._id = C.c_int()

    def nearCoincidentPairs(self, r2Grid: "QMCGrid") -> int:
        """Pairs with this grid as r1 and r2Grid as r2 that are closer than 2^-16 |r1| without being
        identical (tcscf_near_coincident_pairs): the tensor-core paths evaluate them in FP64."""
        n = C.c_int()
        _raise(ffi.lib().tcscf_near_coincident_pairs(self.ctx.handle, self.id, r2Grid.id, C.byref(n)), self.ctx.handle)
        return n.value


def loadSTO(directory: str, basisSet: str, element: str, maxL: int) -> list:
    """loadSTO (SlaterTypeOrbital.cpp:24-75): the (alpha, n, l, m) Slater-type orbitals of `element`
    in the basis-set library `directory`/`basisSet` (TZ3P, QZ6P, ATZ3P or AQZ6P), l <= maxL."""
    n = C.c_int()
    args = (str(directory).encode(), basisSet.encode(), element.encode(), int(maxL))
    ffi.check(ffi.lib().tcscf_load_sto(*args, None, 0, C.byref(n)))
    arr = (ffi.Sto * max(1, n.value))()
    ffi.check(ffi.lib().tcscf_load_sto(*args, arr, n.value, C.byref(n)))
    return [(arr[i].alpha, arr[i].n, arr[i].l, arr[i].m) for i in range(n.value)]


def overlap_core(basis, Z: int) -> tuple[np.ndarray, np.ndarray]:
    """Analytic overlap and core-Hamiltonian matrices (SlaterTypeOrbital.hpp:134-181)."""
    nb = len(basis)
    S = np.empty((nb, nb))
    H = np.empty((nb, nb))
    ffi.check(ffi.lib().tcscf_overlap_core_analytic(ffi.sto_array(basis), nb, Z, ffi.dptr(S), ffi.dptr(H)))
    return S, H


def overlap_core_quadrature(grid: QMCGrid, Z: int) -> tuple[np.ndarray, np.ndarray | None]:
    nb = grid.nBasis()
    S = np.empty((nb, nb), dtype=np.complex128)
    H = np.empty((nb, nb), dtype=np.complex128) if grid.gradients else None
    _raise(ffi.lib().tcscf_overlap_core_quadrature(grid.ctx.handle, grid.id, Z, ffi.dptr(S), ffi.dptr(H)), grid.ctx.handle)
    return S, H


class DeviceTensor:
    def __init__(self, ctx: Context, handle: int):
        self.ctx, self.handle = ctx, handle

    def close(self) -> None:
        if self.handle:
            ffi.lib().tcscf_tensor_destroy(self.ctx.handle, self.handle)
            self.handle = 0


def computeF(r1Grid: QMCGrid, r2Grid: QMCGrid, kernel: int = ffi.K_INV_R12, jastrow: ffi.Ochi | None = None,
             keep: bool = False, copy: bool = True, precision: int = ffi.PREC_FP64):
    """precomputeIntegrand + computeF: Fji [N1][nb][nb] (complex for a 3-D r2 grid, real x 2 pi for 2-D).
    precision: PREC_FP64 or PREC_BF16X3 (tensor-core kernel-GEMM; TC kernels need a Jastrow factor of
    r12 alone)."""
    ctx = r1Grid.ctx
    n1, nb = r1Grid.nGrid(), r1Grid.nBasis()
    F = None
    if copy:
        F = np.empty((n1, nb, nb), dtype=np.complex128 if r2Grid.quadratureGrid.ndim == 3 else np.float64)
    h = C.c_int()
    _raise(ffi.lib().tcscf_compute_F(ctx.handle, r1Grid.id, r2Grid.id, kernel, C.byref(jastrow) if jastrow else None,
                                     int(precision), ffi.dptr(F), int(keep), C.byref(h)), ctx.handle)
    return (F, DeviceTensor(ctx, h.value)) if keep else F


def computeV(r1Grid: QMCGrid, r2Grid: QMCGrid, kernel: int, jastrow: ffi.Ochi, keep: bool = False, copy: bool = True,
             precision: int = ffi.PREC_FP64):
    """precomputeIntegrand + computeV: Vji [N1][nb][nb][3] complex (precision as for computeF)."""
    ctx = r1Grid.ctx
    n1, nb = r1Grid.nGrid(), r1Grid.nBasis()
    V = np.empty((n1, nb, nb, 3), dtype=np.complex128) if copy else None
    h = C.c_int()
    _raise(ffi.lib().tcscf_compute_V(ctx.handle, r1Grid.id, r2Grid.id, kernel, C.byref(jastrow), int(precision), ffi.dptr(V),
                                     int(keep), C.byref(h)), ctx.handle)
    return (V, DeviceTensor(ctx, h.value)) if keep else V


def integrateAllR1R2(r1Grid: QMCGrid, r2Grid: QMCGrid, kernel: int, jastrow: ffi.Ochi | None = None,
                     use_gradient: bool = False) -> np.ndarray:
    """integrateAllR1R2<USE_GRADIENT> (integrateAll.hpp:221-317): r1 a 3-D grid, r2 a 2-D grid.
    Value form: answer[b1][b2][b3][b4]; gradient form (vector kernel . r2 basis gradients):
    answer[b2][b1][b4][b3].  Complex [nb]^4."""
    ctx = r1Grid.ctx
    nb = r1Grid.nBasis()
    out = np.empty((nb,) * 4, dtype=np.complex128)
    _raise(ffi.lib().tcscf_integrate_all_r1r2(ctx.handle, r1Grid.id, r2Grid.id, int(use_gradient), kernel,
                                              C.byref(jastrow) if jastrow is not None else None, ffi.dptr(out)), ctx.handle)
    return out


def threeElectronIntegrals(r1Grid: QMCGrid, r2Grid: QMCGrid, jastrow: ffi.Ochi) -> np.ndarray:
    """threeElectronIntegrals (integrateAll.hpp:361-442): complex [nb]^6, answer[p][q][r][s][t][u]."""
    ctx = r1Grid.ctx
    nb = r1Grid.nBasis()
    out = np.empty((nb,) * 6, dtype=np.complex128)
    _raise(ffi.lib().tcscf_three_electron_integrals(ctx.handle, r1Grid.id, r2Grid.id, C.byref(jastrow), ffi.dptr(out)), ctx.handle)
    return out


def fock_build_batch(r1Grids, r2Grids, densities, hs, respect_symmetry: bool = True, precision: int = ffi.PREC_BF16X3,
                     want_fock: bool = False):
    """Batched RCS Fock builds (one persistent tensor-core launch per tile class for the whole batch).
    Returns the energies [count] (and the Fock matrices when want_fock)."""
    count = len(r1Grids)
    ctx = r1Grids[0].ctx
    D = [np.ascontiguousarray(d, dtype=np.complex128).reshape(g.nBasis(), g.nBasis()) for d, g in zip(densities, r1Grids)]
    H = [np.ascontiguousarray(h, dtype=np.float64) for h in hs]
    F = [np.empty_like(d) for d in D] if want_fock else None
    r1 = (C.c_int * count)(*[g.id for g in r1Grids])
    r2 = (C.c_int * count)(*[g.id for g in r2Grids])
    dp = (ffi._D * count)(*[ffi.dptr(d) for d in D])
    hp = (ffi._D * count)(*[ffi.dptr(h) for h in H])
    fp = (ffi._D * count)(*[ffi.dptr(f) for f in F]) if F else None
    e = np.empty(count)
    _raise(ffi.lib().tcscf_fock_build_batch(ctx.handle, count, r1, r2, dp, hp, int(respect_symmetry), precision, ffi.dptr(e), fp),
           ctx.handle)
    return (e, F) if want_fock else e


def tc_fock_build(r1Grid: QMCGrid, Fs: DeviceTensor, Fo: DeviceTensor, Vs: DeviceTensor, Vo: DeviceTensor, n_up: int, n_down: int,
                  density: np.ndarray, occ_up: np.ndarray, occ_down: np.ndarray, h: np.ndarray, respect_symmetry: bool = True):
    """One transcorrelated Fock build (HartreeFock.cpp:1150-1224) from device tensors.
    occ_up / occ_down: occupied orbitals as [n_occ][nb] rows (column-major nb x n_occ).
    Returns (G2, G3, Fock, energy)."""
    ctx = r1Grid.ctx
    nb = r1Grid.nBasis()
    D = np.ascontiguousarray(density, dtype=np.complex128)
    cu = np.ascontiguousarray(occ_up, dtype=np.complex128).reshape(n_up, nb) if n_up else None
    cd = np.ascontiguousarray(occ_down, dtype=np.complex128).reshape(n_down, nb) if n_down else None
    hh = np.ascontiguousarray(h, dtype=np.float64)
    G2, G3, F = (np.empty((2, nb, nb), dtype=np.complex128) for _ in range(3))
    e = C.c_double()
    _raise(ffi.lib().tcscf_tc_fock_build(ctx.handle, r1Grid.id, Fs.handle, Fo.handle, Vs.handle, Vo.handle, n_up, n_down,
                                         ffi.dptr(D), ffi.dptr(cu), ffi.dptr(cd), ffi.dptr(hh), int(respect_symmetry),
                                         ffi.dptr(G2), ffi.dptr(G3), ffi.dptr(F), C.byref(e)), ctx.handle)
    return G2, G3, F, e.value


def tc_compute_q(r1Grid: QMCGrid, Vs: DeviceTensor, Vo: DeviceTensor):
    """computeQ (HartreeFock.cpp:613-683): (Qss, Qso, Qoo), complex [nb]^6 each, from computeV tensors."""
    ctx = r1Grid.ctx
    nb = r1Grid.nBasis()
    out = [np.empty((nb,) * 6, dtype=np.complex128) for _ in range(3)]
    _raise(ffi.lib().tcscf_tc_compute_q(ctx.handle, r1Grid.id, Vs.handle, Vo.handle, *(ffi.dptr(o) for o in out)), ctx.handle)
    return tuple(out)


def tc_assemble_g(ctx: Context, Qss: np.ndarray, Qso: np.ndarray, Qoo: np.ndarray, density: np.ndarray) -> np.ndarray:
    """assembleG (HartreeFock.cpp:687-752): G3 [2][nb][nb] from the Q tensors and the spin densities."""
    nb = Qss.shape[0]
    D = np.ascontiguousarray(density, dtype=np.complex128)
    G3 = np.empty((2, nb, nb), dtype=np.complex128)
    args = [ffi.dptr(np.ascontiguousarray(q, dtype=np.complex128)) for q in (Qss, Qso, Qoo)]
    _raise(ffi.lib().tcscf_tc_assemble_g(ctx.handle, nb, *args, ffi.dptr(D), ffi.dptr(G3)), ctx.handle)
    return G3


class TCHartreeFock:
    """TCHartreeFock::compute (HartreeFock.hpp:386-394, HartreeFock.cpp:1007-1362) on device tensors."""

    def __init__(self, n_up: int, n_down: int):
        self.n_up, self.n_down = n_up, n_down
        self.energy = None
        self.iterations = 0
        self.density = None
        self.pseudo_energies = None

    def compute(self, overlap: np.ndarray, h: np.ndarray, r1Grid: QMCGrid, Fs: DeviceTensor, Fo: DeviceTensor, Vs: DeviceTensor,
                Vo: DeviceTensor, respect_symmetry: bool = True, tol: float = 1e-5, max_iter: int = 200) -> float:
        ctx = r1Grid.ctx
        nb = r1Grid.nBasis()
        D = np.empty((2, nb, nb), dtype=np.complex128)
        pe = np.zeros((2, nb))
        e, it = C.c_double(), C.c_int()
        code = ffi.lib().tcscf_tc_scf(ctx.handle, r1Grid.id, Fs.handle, Fo.handle, Vs.handle, Vo.handle,
                                      ffi.dptr(np.ascontiguousarray(overlap, dtype=np.float64)),
                                      ffi.dptr(np.ascontiguousarray(h, dtype=np.float64)), self.n_up, self.n_down, int(respect_symmetry),
                                      float(tol), int(max_iter), C.byref(e), C.byref(it), ffi.dptr(D), ffi.dptr(pe))
        self.energy, self.iterations, self.density, self.pseudo_energies = e.value, it.value, D, pe
        if code == ffi.ERR_NOT_CONVERGED:
            raise ConvergenceError(ffi.lib().tcscf_last_error(ctx.handle).decode())
        _raise(code, ctx.handle)
        return self.energy


def _check_shapes(D: np.ndarray, h: np.ndarray, nb: int) -> None:
    """CHECK_BOUNDS_3(density, nSpin, nBasis, nBasis) / CHECK_BOUNDS_2(oneElectronTerms, nBasis, nBasis)."""
    if D.ndim != 3 or D.shape[0] not in (1, 2) or D.shape[1:] != (nb, nb) or h.shape != (nb, nb):
        raise ffi.TcscfError(ffi.ERR_INVALID_ARGUMENT, f"density {D.shape} / h {h.shape} do not match nBasis {nb}")


def fock_build(r1Grid: QMCGrid, r2Grid: QMCGrid, density: np.ndarray, h: np.ndarray, respect_symmetry: bool = True,
               precision: int = ffi.PREC_FP64):
    """Direct-form Fock build: density [nspin][nb][nb] complex -> (G, Fock, energy)."""
    ctx = r1Grid.ctx
    D = np.ascontiguousarray(density, dtype=np.complex128)
    if D.ndim == 2:
        D = D[None]
    nspin, nb = D.shape[0], r1Grid.nBasis()
    hh = np.ascontiguousarray(h, dtype=np.float64)
    _check_shapes(D, hh, nb)
    G = np.empty((nspin, nb, nb), dtype=np.complex128)
    F = np.empty((nspin, nb, nb), dtype=np.complex128)
    e = C.c_double()
    _raise(ffi.lib().tcscf_fock_build(ctx.handle, r1Grid.id, r2Grid.id, nspin, ffi.dptr(D), ffi.dptr(hh), int(respect_symmetry),
                                      precision, ffi.dptr(G), ffi.dptr(F), C.byref(e)), ctx.handle)
    return G, F, e.value


def fock_build_precomputed(r1Grid: QMCGrid, Fji: DeviceTensor, density: np.ndarray, h: np.ndarray, respect_symmetry: bool = True):
    ctx = r1Grid.ctx
    D = np.ascontiguousarray(density, dtype=np.complex128)
    if D.ndim == 2:
        D = D[None]
    nspin, nb = D.shape[0], r1Grid.nBasis()
    hh = np.ascontiguousarray(h, dtype=np.float64)
    _check_shapes(D, hh, nb)
    G = np.empty((nspin, nb, nb), dtype=np.complex128)
    F = np.empty((nspin, nb, nb), dtype=np.complex128)
    e = C.c_double()
    _raise(ffi.lib().tcscf_fock_build_precomputed(ctx.handle, r1Grid.id, Fji.handle, nspin, ffi.dptr(D), ffi.dptr(hh),
                                                  int(respect_symmetry), ffi.dptr(G), ffi.dptr(F), C.byref(e)), ctx.handle)
    return G, F, e.value


class _SCF:
    nspin = 1

    def __init__(self, numSpinUp: int, numSpinDown: int, numBasisFunctions: int):
        self.nElectrons = (numSpinUp, numSpinDown)
        self.basisSize = numBasisFunctions
        self.density = np.zeros((self.nspin, numBasisFunctions, numBasisFunctions), dtype=np.complex128)
        self.eigenvalues = np.zeros((self.nspin, numBasisFunctions))
        self._iter = 0

    def numberOfConvergenceLoops(self) -> int:
        return self._iter

    def compute(self, overlap: np.ndarray, oneElectronTerms: np.ndarray, r1Grid: QMCGrid, r2Grid: QMCGrid,
                respectOneElectronSymmetry: bool = True, precision: int = ffi.PREC_FP64, tol: float = 1e-5,
                max_iter: int | None = None, diis: int = 0, real_eigensolve: bool = False) -> float:
        """diis: Pulay DIIS history length; real_eigensolve: diagonalise a Fock matrix that is real in the
        real-harmonic basis there (real densities when a degenerate shell is partly occupied).  The
        defaults (0, False) iterate plain Roothaan steps with the complex solver, as the reference."""
        ctx = r1Grid.ctx
        S = np.ascontiguousarray(np.real(overlap), dtype=np.float64)
        hh = np.ascontiguousarray(oneElectronTerms, dtype=np.float64)
        nb = r1Grid.nBasis()
        if S.shape != (nb, nb) or hh.shape != (nb, nb) or nb != self.basisSize:
            raise ffi.TcscfError(ffi.ERR_INVALID_ARGUMENT, "overlap / oneElectronTerms do not match nBasis")
        e = C.c_double()
        it = C.c_int()
        _raise(ffi.lib().tcscf_set_scf_options(ctx.handle, int(diis), int(real_eigensolve)), ctx.handle)
        try:
            code = ffi.lib().tcscf_scf(ctx.handle, r1Grid.id, r2Grid.id, self.nspin, self.nElectrons[0], self.nElectrons[1],
                                       ffi.dptr(S), ffi.dptr(hh), int(respectOneElectronSymmetry), precision, tol,
                                       max_iter or self.max_iter, C.byref(e), C.byref(it), ffi.dptr(self.density),
                                       ffi.dptr(self.eigenvalues))
        finally:
            ffi.lib().tcscf_set_scf_options(ctx.handle, 0, 0)
        self._iter = it.value
        _raise(code, ctx.handle)
        return e.value


class RCSHartreeFock(_SCF):
    """RCSHartreeFock (HartreeFock.hpp:233-293): restricted closed shell, at most 50 iterations."""

    nspin = 1
    max_iter = 50

    def highestOccupiedOrbitalEnergy(self) -> float:
        return float(self.eigenvalues[0, sum(self.nElectrons) // 2 - 1])

    def computeOnDevice(self, overlap: np.ndarray, oneElectronTerms: np.ndarray, r1Grid: QMCGrid, r2Grid: QMCGrid,
                        respectOneElectronSymmetry: bool = True, precision: int = ffi.PREC_FP64, tol: float = 1e-5,
                        max_iter: int | None = None, capture: bool = True) -> float:
        """compute() with the whole loop on the device (tcscf_scf_graph): from the zero density, every
        iteration builds, assembles, tests |dE| < tol and diagonalises (real-harmonic basis, canonical
        orthogonalisation, device Jacobi) on the device; with capture the iterations after the first two are
        one CUDA graph launch with a device-side WHILE loop (self.graphLaunches == 1)."""
        ctx = r1Grid.ctx
        S = np.ascontiguousarray(np.real(overlap), dtype=np.float64)
        hh = np.ascontiguousarray(oneElectronTerms, dtype=np.float64)
        nb = r1Grid.nBasis()
        if S.shape != (nb, nb) or hh.shape != (nb, nb) or nb != self.basisSize:
            raise ffi.TcscfError(ffi.ERR_INVALID_ARGUMENT, "overlap / oneElectronTerms do not match nBasis")
        e, it, gl = C.c_double(), C.c_int(), C.c_int()
        code = ffi.lib().tcscf_scf_graph(ctx.handle, r1Grid.id, r2Grid.id, self.nElectrons[0], self.nElectrons[1], ffi.dptr(S),
                                         ffi.dptr(hh), int(respectOneElectronSymmetry), precision, tol, max_iter or self.max_iter,
                                         int(capture), C.byref(e), C.byref(it), ffi.dptr(self.density[0]),
                                         ffi.dptr(self.eigenvalues[0]), C.byref(gl))
        self._iter = it.value
        self.graphLaunches = gl.value
        _raise(code, ctx.handle)
        return e.value


class UOSHartreeFock(_SCF):
    """UOSHartreeFock (HartreeFock.hpp:297-349): unrestricted open shell, at most 100 iterations."""

    nspin = 2
    max_iter = 100

    def highestOccupiedOrbitalEnergy(self) -> float:
        return float(max(self.eigenvalues[0, self.nElectrons[0] - 1], self.eigenvalues[1, self.nElectrons[1] - 1]))

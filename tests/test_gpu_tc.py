"""Transcorrelated Fock build and SCF on the GPU vs the oracle (TCHartreeFock, HartreeFock.cpp:1007-1362).

The F and V tensors are computed on the GPU (tcscf_compute_F / tcscf_compute_V, themselves checked
against the oracle in test_gpu_parity.py) and by the oracle, so each TC build compares the whole
chain.  FP64 throughout: G2, G3 and F agree to 1e-10 of their largest element, the energy to
1e-10 Eh; the SCF energies (different eigen-solvers: LAPACK zggev in the oracle, Cholesky +
cusolverDnXgeev here) to 1e-8 Eh at a 1e-10 convergence threshold.
"""
import numpy as np
import pytest

import oracle
from tcscf_b200 import api, ffi, grids
from tcscf_b200 import basis as wl

pytestmark = pytest.mark.gpu

U = dict(a=1.0, a12=1.0, terms=[((1, 0, 0), -0.5, -0.25)])   # HartreeFockTest.cpp:351-360 sign convention
BASIS = wl.expand(0, [0.6, 1.5, 3.6, 8.5]) + wl.expand(1, [1.2])   # 7 functions
Z, NUP, NDOWN = 4, 2, 2


@pytest.fixture(scope="module")
def tc_setup(ctx):
    g1 = grids.qmc_grid(3, 192, 51)
    g2 = grids.qmc_grid(3, 768, 52)
    G1 = api.QMCGrid(ctx, g1)
    G1.setBasisFunctions(BASIS, storeGradients=True)
    G2 = api.QMCGrid(ctx, g2)
    G2.setBasisFunctions(BASIS)
    u = ffi.ochi_struct(U["a"], U["a12"], U["terms"])
    uo = oracle.ochi(U["a"], U["a12"], U["terms"])
    t = {}
    t["Fs"] = api.computeF(G1, G2, ffi.K_TC_SCALAR_SAME, u, keep=True, copy=False)[1]
    t["Fo"] = api.computeF(G1, G2, ffi.K_TC_SCALAR_OPPO, u, keep=True, copy=False)[1]
    t["Vs"] = api.computeV(G1, G2, ffi.K_GRAD_U_SAME, u, keep=True, copy=False)[1]
    t["Vo"] = api.computeV(G1, G2, ffi.K_GRAD_U_OPPO, u, keep=True, copy=False)[1]
    vals2 = oracle.basis_values(g2.points, BASIS)
    vals1, grads1 = oracle.basis_values(g1.points, BASIS, gradients=True)
    nb = len(BASIS)
    o = dict(Fs=oracle.compute_F(g1.points, g2.points, g2.weights, vals2, nb, ffi.K_TC_SCALAR_SAME, uo),
             Fo=oracle.compute_F(g1.points, g2.points, g2.weights, vals2, nb, ffi.K_TC_SCALAR_OPPO, uo),
             Vs=oracle.compute_V(g1.points, g2.points, g2.weights, vals2, nb, ffi.K_GRAD_U_SAME, uo),
             Vo=oracle.compute_V(g1.points, g2.points, g2.weights, vals2, nb, ffi.K_GRAD_U_OPPO, uo),
             vals1=vals1, grads1=grads1, w1=g1.weights)
    S, h = api.overlap_core(BASIS, Z)
    yield G1, t, o, S, h
    for d in t.values():
        d.close()


def _random_orbitals(nb, n, rng):
    return (rng.normal(size=(n, nb)) + 1j * rng.normal(size=(n, nb))) * 0.3


def test_tc_fock_build_matches_oracle(ctx, tc_setup):
    G1, t, o, S, h = tc_setup
    nb = len(BASIS)
    rng = np.random.default_rng(7)
    occ = [_random_orbitals(nb, NUP, rng), _random_orbitals(nb, NDOWN, rng)]
    D = np.stack([c.T @ c.conj() for c in occ])        # D(u,v) = sum_a C(u,a) conj(C(v,a))
    for sym in (True, False):
        G2, G3, F, E = api.tc_fock_build(G1, t["Fs"], t["Fo"], t["Vs"], t["Vo"], NUP, NDOWN, D, occ[0], occ[1], h, sym)
        G2r, G3r, Fr, Er = oracle.tc_fock_build(o["Fs"], o["Fo"], o["Vs"], o["Vo"], o["vals1"], o["grads1"], o["w1"], D, NUP, NDOWN,
                                                occ[0], occ[1], h, sym)
        for a, b in ((G2, G2r), (G3, G3r), (F, Fr)):
            np.testing.assert_allclose(a, b, rtol=0, atol=1e-10 * max(1.0, np.abs(b).max()))
        assert abs(E - Er) < 1e-10 * max(1.0, abs(Er)), (E, Er)


def test_tc_scf_matches_oracle(ctx, tc_setup):
    G1, t, o, S, h = tc_setup
    scf = api.TCHartreeFock(NUP, NDOWN)
    E = scf.compute(S, h, G1, t["Fs"], t["Fo"], t["Vs"], t["Vo"], tol=1e-10, max_iter=200)
    st, Er, itr, Dr, per = oracle.tc_scf(o["Fs"], o["Fo"], o["Vs"], o["Vo"], o["vals1"], o["grads1"], o["w1"], S, h, NUP, NDOWN,
                                         tol=1e-10, max_iter=200)
    assert st == 0
    assert abs(E - Er) < 1e-8, (E, Er, scf.iterations, itr)
    np.testing.assert_allclose(scf.pseudo_energies[:, :NUP], per[:, :NUP], rtol=0, atol=1e-7)
    np.testing.assert_allclose(scf.density, Dr, rtol=0, atol=1e-6 * np.abs(Dr).max())


def test_tc_argument_checks(ctx, tc_setup):
    G1, t, o, S, h = tc_setup
    nb = len(BASIS)
    D = np.zeros((2, nb, nb), dtype=np.complex128)
    occ = np.zeros((NUP, nb), dtype=np.complex128)
    with pytest.raises(ffi.TcscfError) as e:      # V handle where an F handle belongs
        api.tc_fock_build(G1, t["Vs"], t["Fo"], t["Vs"], t["Vo"], NUP, NDOWN, D, occ, occ, h)
    assert e.value.code == ffi.ERR_INVALID_ARGUMENT


def test_compute_q_and_assemble_g_match_oracle(ctx, tc_setup):
    # the reference's verification route for the 3-body term (computeQ / assembleG,
    # HartreeFock.cpp:613-752): device ZGEMMs over r1 against the oracle's loops to 1e-10 of the
    # largest element; assembleG on the same Q to 1e-12
    G1, t, o, S, h = tc_setup
    Q = api.tc_compute_q(G1, t["Vs"], t["Vo"])
    Qr = oracle.compute_q(o["w1"], o["vals1"], o["Vs"], o["Vo"])
    for a, b in zip(Q, Qr):
        np.testing.assert_allclose(a, b, rtol=0, atol=1e-10 * np.abs(b).max())
    # c_same = c_opposite / 2 here, so Q_so = 2 Q_ss and Q_oo = 4 Q_ss (the reference's own checks)
    np.testing.assert_allclose(Q[1], 2 * Q[0], rtol=0, atol=1e-12 * np.abs(Q[1]).max())
    np.testing.assert_allclose(Q[2], 4 * Q[0], rtol=0, atol=1e-12 * np.abs(Q[2]).max())
    rng = np.random.default_rng(9)
    occ = [_random_orbitals(len(BASIS), n, rng) for n in (NUP, NDOWN)]
    D = np.stack([c.T @ c.conj() for c in occ])
    G3 = api.tc_assemble_g(ctx, *Qr, D)
    G3r = oracle.assemble_g(*Qr, D)
    np.testing.assert_allclose(G3, G3r, rtol=0, atol=1e-12 * np.abs(G3r).max())


# (basis, n_up, n_down, r2 grid dimension of the Fji tensors): the fused per-point build covers nb <= 32
# (when its shared-memory layout fits) with complex Fji (3-D r2) or real Fji (2-D r2, nb even); real
# Fji at odd nb and nb > 32 take the per-intermediate kernels.  Unequal spin counts leave the C columns of the smaller spin partly zero.
_SHAPES = {
    "nb7-2-1-complex": (BASIS, 2, 1, 3),
    "nb8-2-2-real": (wl.expand(0, [0.6, 1.5, 3.6, 8.5, 20.0]) + wl.expand(1, [1.2]), 2, 2, 2),
    "nb7-2-2-real-odd": (BASIS, 2, 2, 2),
    "nb32-2-1-complex": (wl.expand(0, [0.5 * 1.7 ** k for k in range(9)]) + wl.expand(1, [0.8 * 1.8 ** k for k in range(4)])
                         + wl.expand(2, [1.0, 2.6]) + wl.expand(0, [30.0]), 2, 1, 3),
    "nb33-3-2-complex": (wl.expand(0, [0.5 * 1.7 ** k for k in range(11)]) + wl.expand(1, [0.8 * 1.8 ** k for k in range(4)])
                         + wl.expand(2, [1.0, 2.6]), 3, 2, 3),
}


@pytest.mark.parametrize("case", sorted(_SHAPES))
def test_tc_fock_build_shapes(ctx, case):
    basis, nup, ndown, dim2 = _SHAPES[case]
    nb = len(basis)
    assert nb == int(case[2:].split("-")[0])
    g1 = grids.qmc_grid(3, 128, 61)
    g2 = grids.qmc_grid(dim2, 512, 62)
    g3 = grids.qmc_grid(3, 512, 63)
    G1 = api.QMCGrid(ctx, g1)
    G1.setBasisFunctions(basis, storeGradients=True)
    G2 = api.QMCGrid(ctx, g2)
    G2.setBasisFunctions(basis)
    G3 = api.QMCGrid(ctx, g3)
    G3.setBasisFunctions(basis)
    u = ffi.ochi_struct(U["a"], U["a12"], U["terms"])
    uo = oracle.ochi(U["a"], U["a12"], U["terms"])
    t = dict(Fs=api.computeF(G1, G2, ffi.K_TC_SCALAR_SAME, u, keep=True, copy=False)[1],
             Fo=api.computeF(G1, G2, ffi.K_TC_SCALAR_OPPO, u, keep=True, copy=False)[1],
             Vs=api.computeV(G1, G3, ffi.K_GRAD_U_SAME, u, keep=True, copy=False)[1],
             Vo=api.computeV(G1, G3, ffi.K_GRAD_U_OPPO, u, keep=True, copy=False)[1])
    vals2 = oracle.basis_values(g2.points, basis)
    vals3 = oracle.basis_values(g3.points, basis)
    vals1, grads1 = oracle.basis_values(g1.points, basis, gradients=True)
    o = dict(Fs=oracle.compute_F(g1.points, g2.points, g2.weights, vals2, nb, ffi.K_TC_SCALAR_SAME, uo),
             Fo=oracle.compute_F(g1.points, g2.points, g2.weights, vals2, nb, ffi.K_TC_SCALAR_OPPO, uo),
             Vs=oracle.compute_V(g1.points, g3.points, g3.weights, vals3, nb, ffi.K_GRAD_U_SAME, uo),
             Vo=oracle.compute_V(g1.points, g3.points, g3.weights, vals3, nb, ffi.K_GRAD_U_OPPO, uo))
    assert (o["Fs"].dtype == np.float64) == (dim2 == 2)
    _, h = api.overlap_core(basis, Z)
    rng = np.random.default_rng(nb)
    occ = [_random_orbitals(nb, nup, rng), _random_orbitals(nb, ndown, rng)]
    D = np.stack([c.T @ c.conj() for c in occ])
    try:
        G2g, G3g, Fg, Eg = api.tc_fock_build(G1, t["Fs"], t["Fo"], t["Vs"], t["Vo"], nup, ndown, D, occ[0], occ[1], h, False)
        G2r, G3r, Fr, Er = oracle.tc_fock_build(o["Fs"], o["Fo"], o["Vs"], o["Vo"], vals1, grads1, g1.weights, D, nup, ndown,
                                                occ[0], occ[1], h, False)
        for a, b in ((G2g, G2r), (G3g, G3r), (Fg, Fr)):
            np.testing.assert_allclose(a, b, rtol=0, atol=1e-10 * max(1.0, np.abs(b).max()))
        assert abs(Eg - Er) < 1e-10 * max(1.0, abs(Er)), (Eg, Er)
    finally:
        for d in t.values():
            d.close()


def test_compute_q_and_assemble_g_beyond_sixteen_functions(ctx):
    # the 6-index route is limited by device memory rather than a basis size: 18 functions (the old
    # fixed limit was 16; 3 x 18^6 complex = 1.6 GB per set of Q tensors), against the oracle
    basis = wl.expand(0, [0.5, 1.1, 2.4, 5.2, 11.0, 23.0]) + wl.expand(1, [0.9, 2.0, 4.4, 9.5])   # 6 + 12 = 18
    nb = len(basis)
    g1 = grids.qmc_grid(3, 16, 71)
    g2 = grids.qmc_grid(3, 256, 72)
    G1 = api.QMCGrid(ctx, g1)
    G1.setBasisFunctions(basis)
    G2 = api.QMCGrid(ctx, g2)
    G2.setBasisFunctions(basis)
    u = ffi.ochi_struct(U["a"], U["a12"], U["terms"])
    uo = oracle.ochi(U["a"], U["a12"], U["terms"])
    Vs = api.computeV(G1, G2, ffi.K_GRAD_U_SAME, u, keep=True, copy=False)[1]
    Vo = api.computeV(G1, G2, ffi.K_GRAD_U_OPPO, u, keep=True, copy=False)[1]
    try:
        Q = api.tc_compute_q(G1, Vs, Vo)
    finally:
        Vs.close()
        Vo.close()
    vals2 = oracle.basis_values(g2.points, basis)
    Vso = oracle.compute_V(g1.points, g2.points, g2.weights, vals2, nb, ffi.K_GRAD_U_SAME, uo)
    Voo = oracle.compute_V(g1.points, g2.points, g2.weights, vals2, nb, ffi.K_GRAD_U_OPPO, uo)
    Qr = oracle.compute_q(g1.weights, oracle.basis_values(g1.points, basis), Vso, Voo)
    for a, b in zip(Q, Qr):
        np.testing.assert_allclose(a, b, rtol=0, atol=1e-10 * np.abs(b).max())
    del Q
    rng = np.random.default_rng(11)
    occ = [_random_orbitals(nb, n, rng) for n in (NUP, NDOWN)]
    D = np.stack([c.T @ c.conj() for c in occ])
    G3 = api.tc_assemble_g(ctx, *Qr, D)
    G3r = oracle.assemble_g(*Qr, D)
    np.testing.assert_allclose(G3, G3r, rtol=0, atol=1e-12 * np.abs(G3r).max())

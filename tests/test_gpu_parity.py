"""FP64 GPU path vs the CPU oracle on identical point sets (parity tests proper, through the C ABI).

Bars: basis values and Fji to ~1e-13 relative; Fock matrices to 1e-11 absolute; energies to
1e-10 Eh (the FP64 target).
"""
import numpy as np
import pytest

import oracle
from tcscf_b200 import api, ffi, grids
from tcscf_b200 import basis as wl

pytestmark = pytest.mark.gpu

E_TOL = 1e-10


def rand_density(nb, nocc, rng, complex_=True, scale=0.3):
    C = rng.normal(size=(nb, nocc)) * scale
    if complex_:
        C = C + 1j * rng.normal(size=(nb, nocc)) * scale
    return C @ C.conj().T


def real_density(basis, nocc, rng):
    """A density that is real in the real-harmonic basis (the closed-shell SCF case): built from
    orbitals that are real combinations of cos/sin-type functions."""
    nb = len(basis)
    U = wl.real_harmonic_unitary(basis)
    CR = rng.normal(size=(nb, nocc)) * 0.3          # real-basis orbital coefficients
    C = U.T @ CR                                   # psi = sum_k CR_k phiR_k = sum_i (U^T CR)_i phi_i
    return C @ C.conj().T


@pytest.fixture(scope="module")
def he_setup(ctx):
    w = wl.he()
    g = grids.product_grid(w.nrad, w.order)
    G = api.QMCGrid(ctx, g)
    G.setBasisFunctions(w.basis)
    return w, g, G


def test_basis_values_and_gradients_match_oracle(ctx):
    basis = wl.ne().basis + [(1.1, 4, 3, m) for m in range(-3, 4)]
    g = grids.product_grid(6, 17)
    G = api.QMCGrid(ctx, g)
    G.setBasisFunctions(basis, storeGradients=True)
    ref = oracle.basis_values(g.points, basis)
    got = G.basisValues
    np.testing.assert_allclose(got, ref, rtol=0, atol=1e-12 * np.abs(ref).max())
    # gradients on a QMC grid (no pole points, which the reference formula divides by)
    q = grids.qmc_grid(3, 2048, 11)
    Q = api.QMCGrid(ctx, q)
    Q.setBasisFunctions(basis, storeGradients=True)
    rv, rg = oracle.basis_values(q.points, basis, gradients=True)
    np.testing.assert_allclose(Q.basisValues, rv, rtol=0, atol=1e-12 * np.abs(rv).max())
    gg = Q.basisGradients
    np.testing.assert_allclose(gg, rg, rtol=1e-9, atol=1e-11 * np.abs(rg).max())
    # 2-D grid: real values at phi = 0
    q2 = grids.qmc_grid(2, 1024, 5)
    Q2 = api.QMCGrid(ctx, q2)
    Q2.setBasisFunctions(basis)
    np.testing.assert_allclose(Q2.basisValues, oracle.basis_values(q2.points, basis), rtol=0, atol=1e-12 * np.abs(rv).max())


def test_quadrature_overlap_equals_analytic_on_gpu(ctx):
    # the SlaterTypeOrbitalTest.cpp:14-47 pin, run through the device basis evaluator and S/H sums
    r, wr = grids.radial_grid(1000, ffi.MAP_TREUTLER_AHLRICHS_M4, 1.0, 1.0)
    # Lebedev-11 rotated off the axes: the rule stays exact for the same polynomial space and no point
    # sits on a pole, where the reference's gradient formula (SlaterTypeOrbital.hpp:73-74) divides by 0
    from scipy.integrate import lebedev_rule
    from scipy.spatial.transform import Rotation

    x, wa = lebedev_rule(11)
    x = Rotation.from_euler("zyx", [0.3, 0.2, 0.1]).apply(x.T).T
    ang = np.ascontiguousarray(np.stack([np.arccos(np.clip(x[2], -1, 1)), np.arctan2(x[1], x[0]), wa], axis=1))
    pts = np.empty((3, 1000 * 50))
    w = np.empty(1000 * 50)
    ffi.check(ffi.lib().tcscf_grid_product(1000, ffi.dptr(r), ffi.dptr(wr), 50, ffi.dptr(ang), ffi.dptr(pts), ffi.dptr(w)))
    basis = []
    for n in range(1, 5):
        for l in range(0, n):
            for m in range(-l, l + 1):
                basis += [(1.524, n, l, m), (2.532, n, l, m)]
    G = api.QMCGrid(ctx, grids.QuadratureGrid(pts, w))
    G.setBasisFunctions(basis, storeGradients=True)
    S, H = api.overlap_core_quadrature(G, 3)
    S_an, H_an = api.overlap_core(basis, 3)
    assert np.abs(S - S_an).max() < 1e-13
    # kinetic + nuclear attraction by quadrature agrees with the analytic core Hamiltonian for the
    # m >= 0 functions; for m < 0 the reference's gradient formula (SlaterTypeOrbital.hpp:70) uses
    # Y_l^{m+1} with the wrong relative sign, a quirk the device evaluator reproduces for parity
    keep = np.array([b[3] >= 0 for b in basis])
    Hk, Hak = H[np.ix_(keep, keep)], H_an[np.ix_(keep, keep)]
    assert np.abs(Hk - Hak).max() < 1e-8 * np.abs(Hak).max()


@pytest.mark.parametrize("ndim2", [3, 2])
def test_computeF_matches_oracle(ctx, he_setup, ndim2):
    w, g, G = he_setup
    rng = np.random.default_rng(3)
    idx = rng.choice(g.n, 96, replace=False)
    g1 = grids.subset(g, idx)
    G1 = api.QMCGrid(ctx, g1)
    G1.setBasisFunctions(w.basis)
    if ndim2 == 3:
        g2, G2 = g, G
    else:
        g2 = grids.qmc_grid(2, 2000, 4)
        G2 = api.QMCGrid(ctx, g2)
        G2.setBasisFunctions(w.basis)
    F = api.computeF(G1, G2)
    vals2 = oracle.basis_values(g2.points, w.basis)
    Fr = oracle.compute_F(g1.points, g2.points, g2.weights, vals2, w.nb)
    assert F.dtype == Fr.dtype
    np.testing.assert_allclose(F, Fr, rtol=0, atol=1e-12 * np.abs(Fr).max())


def _oracle_fock(g1, g2, basis, D, h, nspin=1):
    vals1 = oracle.basis_values(g1.points, basis)
    vals2 = oracle.basis_values(g2.points, basis)
    F = oracle.compute_F(g1.points, g2.points, g2.weights, vals2, len(basis))
    return oracle.fock_build(F, vals1, g1.weights, D, h), F, vals1


@pytest.mark.parametrize("kind", ["real", "complex"])
def test_rcs_fock_build_direct_matches_oracle_he(ctx, he_setup, kind):
    w, g, G = he_setup
    rng = np.random.default_rng(7)
    D = real_density(w.basis, 1, rng) if kind == "real" else rand_density(w.nb, 1, rng)
    S, h = api.overlap_core(w.basis, w.Z)
    (Gr, Fr, Er), _, _ = _oracle_fock(g, g, w.basis, D, h)
    Gg, Fg, Eg = api.fock_build(G, G, D, h)
    assert abs(Eg - Er) < E_TOL, (Eg, Er)
    np.testing.assert_allclose(Gg, Gr, rtol=0, atol=1e-11)
    np.testing.assert_allclose(Fg, Fr, rtol=0, atol=1e-11)


def test_rcs_fock_build_direct_ne_subset(ctx):
    # Ne-sized r2 grid (59,000 points, nb = 40), 160 sampled r1 points, rank-5 density
    w = wl.ne()
    g = grids.product_grid(w.nrad, w.order)
    rng = np.random.default_rng(11)
    g1 = grids.subset(g, rng.choice(g.n, 160, replace=False))
    G1 = api.QMCGrid(ctx, g1)
    G1.setBasisFunctions(w.basis)
    G2 = api.QMCGrid(ctx, g)
    G2.setBasisFunctions(w.basis)
    D = real_density(w.basis, 5, rng)
    S, h = api.overlap_core(w.basis, w.Z)
    (Gr, Fr, Er), _, _ = _oracle_fock(g1, g, w.basis, D, h)
    Gg, Fg, Eg = api.fock_build(G1, G2, D, h)
    assert abs(Eg - Er) < E_TOL, (Eg, Er)
    np.testing.assert_allclose(Gg, Gr, rtol=0, atol=1e-11)


@pytest.mark.parametrize("n1", [96, 160])
def test_rcs_fock_build_direct_kr_basis_subset(ctx, n1):
    # nb = 120 takes the 128-column FP64 tile (the warp-specialised FP64 tensor-core contraction for
    # this rank): 18 occupied orbitals, one partial or two r1 tiles of sampled points against a
    # 12 x Lebedev-77 r2 grid (24,360 points), split over r2 into blocks of a few steps
    w = wl.kr()
    g = grids.product_grid(12, w.order)
    rng = np.random.default_rng(n1)
    g1 = grids.subset(g, rng.choice(g.n, n1, replace=False))
    G1 = api.QMCGrid(ctx, g1)
    G1.setBasisFunctions(w.basis)
    G2 = api.QMCGrid(ctx, g)
    G2.setBasisFunctions(w.basis)
    D = real_density(w.basis, 18, rng)
    S, h = api.overlap_core(w.basis, w.Z)
    (Gr, Fr, Er), _, _ = _oracle_fock(g1, g, w.basis, D, h)
    Gg, Fg, Eg = api.fock_build(G1, G2, D, h, precision=ffi.PREC_FP64)
    scale = np.abs(Gr).max()
    assert abs(Eg - Er) < E_TOL * max(1.0, abs(Er)), (Eg, Er)
    assert np.abs(Gg - Gr).max() <= 1e-12 * scale, np.abs(Gg - Gr).max() / scale
    G1.close()
    G2.close()


def test_uos_fock_build_and_2d_r2_grid(ctx, he_setup):
    w, g, G = he_setup
    rng = np.random.default_rng(5)
    D = np.stack([real_density(w.basis, 2, rng), rand_density(w.nb, 1, rng)])
    S, h = api.overlap_core(w.basis, w.Z)
    (Gr, Fr, Er), _, _ = _oracle_fock(g, g, w.basis, D, h)
    Gg, Fg, Eg = api.fock_build(G, G, D, h)
    assert abs(Eg - Er) < E_TOL
    np.testing.assert_allclose(Gg, Gr, rtol=0, atol=1e-11)
    # RCS with a 2-D r2 grid (QMCGrid<REAL,2>, real Fji x 2 pi, HartreeFock.hpp:88-131)
    g2 = grids.qmc_grid(2, 3000, 9)
    G2 = api.QMCGrid(ctx, g2)
    G2.setBasisFunctions(w.basis)
    D1 = real_density(w.basis, 1, rng)
    (Gr, Fr, Er), _, _ = _oracle_fock(g, g2, w.basis, D1, h)
    Gg, Fg, Eg = api.fock_build(G, G2, D1, h)
    assert abs(Eg - Er) < E_TOL
    np.testing.assert_allclose(Gg, Gr, rtol=0, atol=1e-11)


def test_precomputed_form_matches_oracle(ctx, he_setup):
    w, g, G = he_setup
    rng = np.random.default_rng(9)
    D = rand_density(w.nb, 1, rng)
    S, h = api.overlap_core(w.basis, w.Z)
    (Gr, Fr, Er), Fji, _ = _oracle_fock(g, g, w.basis, D, h)
    F, t = api.computeF(G, G, keep=True)
    np.testing.assert_allclose(F, Fji, rtol=0, atol=1e-12 * np.abs(Fji).max())
    Gg, Fg, Eg = api.fock_build_precomputed(G, t, D, h)
    t.close()
    assert abs(Eg - Er) < E_TOL
    np.testing.assert_allclose(Gg, Gr, rtol=0, atol=1e-11)


def test_rcs_scf_matches_oracle_he(ctx, he_setup):
    w, g, G = he_setup
    S, h = api.overlap_core(w.basis, w.Z)
    vals1 = oracle.basis_values(g.points, w.basis)
    F = oracle.compute_F(g.points, g.points, g.weights, vals1, w.nb)
    # converged to 1e-10 Eh so that the two energies agree to E_TOL wherever each loop stops: the GPU
    # build's rounding differs from the oracle's (it contracts each pair once when r1 = r2), which can
    # move the iteration that first meets the threshold by one
    st, Er, itr, Dr, eig = oracle.scf(1, 1, 1, F, vals1, g.weights, S, h, tol=1e-10, max_iter=50)
    assert st == 0
    hf = api.RCSHartreeFock(1, 1, w.nb)
    Eg = hf.compute(S, h, G, G, tol=1e-10)
    assert abs(Eg - Er) < E_TOL, (Eg, Er, itr, hf.numberOfConvergenceLoops())
    assert abs(hf.numberOfConvergenceLoops() - itr) <= 1
    # physically sensible: within the 50 x 50 product grid's quadrature error of the He Hartree-Fock
    # limit -2.8617 Eh (src/unitTests/HartreeFockTest.cpp:591-602)
    assert -2.95 < Eg < -2.75


def test_tc_kernels_match_oracle(ctx):
    w = wl.be_tc()
    u_params = dict(a=1.0, a12=1.0, terms=[((1, 0, 0), 0.5, 0.5)])
    u = ffi.ochi_struct(u_params["a"], u_params["a12"], u_params["terms"])
    uo = oracle.ochi(u_params["a"], u_params["a12"], u_params["terms"])
    g1 = grids.qmc_grid(3, 64, 21)
    g2 = grids.qmc_grid(3, 1024, 22)
    G1 = api.QMCGrid(ctx, g1)
    G1.setBasisFunctions(w.basis)
    G2 = api.QMCGrid(ctx, g2)
    G2.setBasisFunctions(w.basis)
    vals2 = oracle.basis_values(g2.points, w.basis)
    for k in (ffi.K_TC_SCALAR_SAME, ffi.K_TC_SCALAR_OPPO):
        F = api.computeF(G1, G2, kernel=k, jastrow=u)
        Fr = oracle.compute_F(g1.points, g2.points, g2.weights, vals2, w.nb, kernel=k, u=uo)
        np.testing.assert_allclose(F, Fr, rtol=0, atol=1e-11 * np.abs(Fr).max())
    for k in (ffi.K_GRAD_U_SAME, ffi.K_GRAD_U_OPPO):
        V = api.computeV(G1, G2, kernel=k, jastrow=u)
        Vr = oracle.compute_V(g1.points, g2.points, g2.weights, vals2, w.nb, kernel=k, u=uo)
        np.testing.assert_allclose(V, Vr, rtol=0, atol=1e-11 * np.abs(Vr).max())


def test_invalid_arguments_raise(ctx, he_setup):
    w, g, G = he_setup
    S, h = api.overlap_core(w.basis, w.Z)
    with pytest.raises(ffi.TcscfError) as e:
        api.fock_build(G, G, np.zeros((3, 3)), h)
    assert e.value.code == ffi.ERR_INVALID_ARGUMENT
    bad = api.QMCGrid(ctx, grids.product_grid(4, 11))
    with pytest.raises(ffi.TcscfError) as e:
        bad.setBasisFunctions([(1.0, 2, 1, 1)])  # missing the m = -1 partner
    assert e.value.code == ffi.ERR_UNSUPPORTED
    with pytest.raises(ffi.TcscfError) as e:
        bad.setBasisFunctions([(1.0, 1, 2, 0)])  # n < l
    assert e.value.code == ffi.ERR_INVALID_ARGUMENT
    hf = api.RCSHartreeFock(1, 1, w.nb)
    with pytest.raises(api.ConvergenceError):
        hf.compute(S, h, G, G, tol=1e-30, max_iter=2)


def test_rcs_scf_diis_reaches_the_same_energy(ctx):
    # optional Pulay DIIS (no reference counterpart): the converged energy of the plain Roothaan
    # iteration (closed-shell atoms converge in a similar number of steps either way); DIIS off
    # reproduces the plain iteration exactly
    w = wl.ne()
    g = grids.product_grid(24, 17)
    G = api.QMCGrid(ctx, g)
    G.setBasisFunctions(w.basis)
    S, h = api.overlap_core(w.basis, w.Z)
    plain = api.RCSHartreeFock(w.n_up, w.n_down, w.nb)
    Ep = plain.compute(S, h, G, G, tol=1e-10, max_iter=200)
    acc = api.RCSHartreeFock(w.n_up, w.n_down, w.nb)
    Ed = acc.compute(S, h, G, G, tol=1e-10, max_iter=200, diis=8)
    assert abs(Ed - Ep) < 1e-8, (Ed, Ep)
    assert acc.numberOfConvergenceLoops() <= plain.numberOfConvergenceLoops() + 5
    again = api.RCSHartreeFock(w.n_up, w.n_down, w.nb)
    assert again.compute(S, h, G, G, tol=1e-10, max_iter=200) == Ep
    with pytest.raises(ffi.TcscfError) as e:
        acc.compute(S, h, G, G, diis=17)
    assert e.value.code == ffi.ERR_INVALID_ARGUMENT

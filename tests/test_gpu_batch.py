"""Batched Fock builds (tcscf_fock_build_batch) vs one build at a time.

All instances' tensor contractions share one persistent launch per tile class; every work item is
computed exactly as in a single build (same splits, deterministic sums), so the batched energies and
Fock matrices equal the single-build ones bit for bit.  Against FP64 the bar is max(1e-9 Eh, 2e-7 |E|):
these are random, non-physical densities (energies up to ~4e5 Eh) on coarse 8-20-point radial grids,
where the fixed-point slicing error averages over few points (measured up to 6.7e-8 |E|); physical
densities on the workload grids stay near 1e-10 |E| (Ne, Kr).
"""
import numpy as np
import pytest

from tcscf_b200 import api, ffi, grids
from tcscf_b200 import basis as wl

from .test_gpu_parity import rand_density, real_density

pytestmark = pytest.mark.gpu


def _instances(ctx, count, seed):
    rng = np.random.default_rng(seed)
    out = []
    for w in wl.batch(seed=seed, count=count):
        w.nrad = int(rng.integers(8, 20))                   # small grids keep the test quick
        g = grids.product_grid(w.nrad, min(w.order, 29))
        G = api.QMCGrid(ctx, g)
        G.setBasisFunctions(w.basis)
        S, h = api.overlap_core(w.basis, w.Z)
        out.append((w, G, h))
    return out


def test_batch_matches_single_builds(ctx):
    inst = _instances(ctx, 6, 20261203)
    rng = np.random.default_rng(11)
    Ds = [real_density(w.basis, max(1, min(w.n_up, 8)), rng) for w, G, h in inst]
    # one instance with a density that is complex in the real-harmonic basis (built on its own)
    w0 = inst[0][0]
    Ds[0] = rand_density(w0.nb, 2, rng)
    Gs = [G for w, G, h in inst]
    hs = [h for w, G, h in inst]
    E, F = api.fock_build_batch(Gs, Gs, Ds, hs, precision=ffi.PREC_BF16X3, want_fock=True)
    for k, (w, G, h) in enumerate(inst):
        _, Fs, Es = api.fock_build(G, G, Ds[k], h, precision=ffi.PREC_BF16X3)
        assert E[k] == Es, (k, E[k], Es)
        np.testing.assert_array_equal(F[k], Fs[0])
        _, _, Ed = api.fock_build(G, G, Ds[k], h, precision=ffi.PREC_FP64)
        assert abs(E[k] - Ed) < max(1e-9, 2e-7 * abs(Ed)), (k, E[k], Ed)


def test_batch_fp64_and_arguments(ctx):
    inst = _instances(ctx, 3, 7)
    rng = np.random.default_rng(12)
    Ds = [real_density(w.basis, max(1, min(w.n_up, 4)), rng) for w, G, h in inst]
    Gs = [G for w, G, h in inst]
    hs = [h for w, G, h in inst]
    E = api.fock_build_batch(Gs, Gs, Ds, hs, precision=ffi.PREC_FP64)
    for k, (w, G, h) in enumerate(inst):
        _, _, Ed = api.fock_build(G, G, Ds[k], h, precision=ffi.PREC_FP64)
        assert abs(E[k] - Ed) < 1e-12 * max(1.0, abs(Ed))
    with pytest.raises(ffi.TcscfError) as e:
        api.fock_build_batch(Gs, Gs, Ds, hs, precision=7)
    assert e.value.code == ffi.ERR_INVALID_ARGUMENT


def test_batch_tf32_matches_single_builds(ctx):
    # the TF32 tile classes run in the same persistent launches: each instance's result is the one its
    # own build gives (same tiles, splits and summation order)
    inst = _instances(ctx, 3, 11)
    rng = np.random.default_rng(13)
    Ds = [real_density(w.basis, max(1, min(w.n_up, 4)), rng) for w, G, h in inst]
    Gs = [G for w, G, h in inst]
    hs = [h for w, G, h in inst]
    E = api.fock_build_batch(Gs, Gs, Ds, hs, precision=ffi.PREC_TF32)
    for k, (w, G, h) in enumerate(inst):
        _, _, Et = api.fock_build(G, G, Ds[k], h, precision=ffi.PREC_TF32)
        assert E[k] == Et, (k, E[k], Et)


def test_batch_graph_replays_give_identical_results(ctx):
    # the batch's persistent launches run as a CUDA graph: captured on the first call with a new launch
    # sequence, replayed on repeats (fresh device tables each time); results are bit-identical
    inst = _instances(ctx, 3, 17)
    rng = np.random.default_rng(19)
    Ds = [real_density(w.basis, max(1, min(w.n_up, 4)), rng) for w, G, h in inst]
    Gs = [G for w, G, h in inst]
    hs = [h for w, G, h in inst]
    c0, r0 = ctx.batch_graph_stats()
    E1 = api.fock_build_batch(Gs, Gs, Ds, hs, precision=ffi.PREC_BF16X3)
    c1, r1 = ctx.batch_graph_stats()
    E2 = api.fock_build_batch(Gs, Gs, Ds, hs, precision=ffi.PREC_BF16X3)
    c2, r2 = ctx.batch_graph_stats()
    assert r2 == r1 + 1 and c2 == c1, (c0, r0, c1, r1, c2, r2)
    assert np.array_equal(E1, E2)
    # a different density on the same instances replays the same graph and changes the result
    Ds2 = [real_density(w.basis, max(1, min(w.n_up, 4)), rng) for w, G, h in inst]
    E3 = api.fock_build_batch(Gs, Gs, Ds2, hs, precision=ffi.PREC_BF16X3)
    assert ctx.batch_graph_stats()[1] == r2 + 1
    for k, (w, G, h) in enumerate(inst):
        _, _, Es = api.fock_build(G, G, Ds2[k], h, precision=ffi.PREC_BF16X3)
        assert E3[k] == Es, (k, E3[k], Es)


def test_batch_graph_recaptured_for_a_new_launch_sequence(ctx):
    # another set of instances gives another launch sequence: a fresh capture, and its results still
    # equal the single builds
    inst = _instances(ctx, 2, 23)
    rng = np.random.default_rng(29)
    Ds = [real_density(w.basis, max(1, min(w.n_up, 4)), rng) for w, G, h in inst]
    Gs = [G for w, G, h in inst]
    hs = [h for w, G, h in inst]
    c0, _ = ctx.batch_graph_stats()
    E = api.fock_build_batch(Gs, Gs, Ds, hs, precision=ffi.PREC_BF16X3)
    assert ctx.batch_graph_stats()[0] == c0 + 1
    for k, (w, G, h) in enumerate(inst):
        _, _, Es = api.fock_build(G, G, Ds[k], h, precision=ffi.PREC_BF16X3)
        assert E[k] == Es, (k, E[k], Es)

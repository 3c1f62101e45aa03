"""Launch-schedule autotuner on the device (tcscf_set_autotune), each test on a context of its own.

With autotuning on, the first tensor-path build of a shape times the candidate tile classes (TMA
stages, T tile width; bit-identical results) and then every candidate r2 split of its persistent
launch, and the first batch of a signature times every split policy; later builds of the same
shape or signature reuse the choice without measuring again.  A split changes only the order of
the r2 block sums (each split's double-float partial sums are added in FP64 afterwards), so the bar
against the default schedule is 1e-10 relative in the energy and 1e-9 of the largest |Fock| element,
far below the mixed path's own error against FP64 (about 1e-8 relative).  A fixed schedule is
deterministic: the same split gives bit-identical results, and turning the tuner off returns the
default schedule's results exactly. 
"""
import numpy as np
import pytest
import torch

from tcscf_b200 import api, ffi, grids
from tcscf_b200 import basis as wl

from .test_gpu_parity import real_density

pytestmark = pytest.mark.gpu

E_REL = 1e-10
F_REL = 1e-9


def _sms():
    return torch.cuda.get_device_properties(0).multi_processor_count


@pytest.mark.parametrize("name, nocc", [("he", 1), ("ne", 5)])
def test_autotuned_single_build_matches_default_schedule(name, nocc):
    w = getattr(wl, name)()
    g = grids.product_grid(w.nrad, w.order)
    rng = np.random.default_rng(5)
    D = real_density(w.basis, nocc, rng)
    _, h = api.overlap_core(w.basis, w.Z)
    with api.Context(0) as c:
        G = api.QMCGrid(c, g)
        G.setBasisFunctions(w.basis)
        _, F0, E0 = api.fock_build(G, G, D, h, precision=ffi.PREC_BF16X3)
        c.set_autotune(True)
        _, F1, E1 = api.fock_build(G, G, D, h, precision=ffi.PREC_BF16X3)
        shapes, batches, meas = c.autotune_stats()
        assert (shapes, batches) == (1, 0)
        ncand = len(ffi.autotune_split_candidates(g.n, g.n, _sms()))
        # split-BF16 shapes with a 64-column tile (nb <= 64, rank padding 32) first time three tile
        # classes (the rule's, two TMA stages, the 128-column tile), then the splits
        nclass = 3 if w.nb <= 64 and nocc <= 32 else 0
        assert meas == nclass + (ncand if ncand > 1 else 0)
        assert abs(E1 - E0) <= E_REL * abs(E0), (E1, E0)
        assert np.abs(F1 - F0).max() <= F_REL * np.abs(F0).max()
        # the shape's choice is reused: no new measurements, the same bits
        _, F2, E2 = api.fock_build(G, G, D, h, precision=ffi.PREC_BF16X3)
        assert c.autotune_stats() == (1, 0, meas)
        assert E2 == E1
        np.testing.assert_array_equal(F2, F1)
        # off again: the default schedule, bit for bit
        c.set_autotune(False)
        _, F3, E3 = api.fock_build(G, G, D, h, precision=ffi.PREC_BF16X3)
        assert E3 == E0
        np.testing.assert_array_equal(F3, F0)


def test_autotuned_batch_matches_default_schedule():
    seed = 20261204
    rng = np.random.default_rng(seed)
    with api.Context(0) as c:
        Gs, Ds, hs = [], [], []
        for w in wl.batch(seed=seed, count=4):
            w.nrad = int(rng.integers(8, 20))               # small grids keep the test quick
            g = grids.product_grid(w.nrad, min(w.order, 29))
            G = api.QMCGrid(c, g)
            G.setBasisFunctions(w.basis)
            _, h = api.overlap_core(w.basis, w.Z)
            Gs.append(G)
            hs.append(h)
            Ds.append(real_density(w.basis, max(1, min(w.n_up, 8)), rng))
        E0, F0 = api.fock_build_batch(Gs, Gs, Ds, hs, precision=ffi.PREC_BF16X3, want_fock=True)
        c.set_autotune(True)
        E1, F1 = api.fock_build_batch(Gs, Gs, Ds, hs, precision=ffi.PREC_BF16X3, want_fock=True)
        _, batches, meas = c.autotune_stats()
        assert batches == 1 and meas == 4                     # four split policies, one measurement each
        np.testing.assert_allclose(E1, E0, rtol=E_REL, atol=0)
        for a, b in zip(F1, F0):
            assert np.abs(a - b).max() <= F_REL * np.abs(b).max()
        E2, F2 = api.fock_build_batch(Gs, Gs, Ds, hs, precision=ffi.PREC_BF16X3, want_fock=True)
        assert c.autotune_stats()[1:] == (1, 4)
        np.testing.assert_array_equal(E2, E1)
        c.set_autotune(False)
        E3, _ = api.fock_build_batch(Gs, Gs, Ds, hs, precision=ffi.PREC_BF16X3, want_fock=True)
        np.testing.assert_array_equal(E3, E0)

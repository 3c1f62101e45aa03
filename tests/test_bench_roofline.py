"""The benchmark line's roofline arithmetic (no device needed).

At the Kr configuration (406,000 points, 120 functions, 18 occupied orbitals) and the measured
458.2 ms split-BF16 contraction: F_alg = 2 N^2 (nb nocc + 1) = 7.124e14 flops gives 1,555 TFLOP/s
against the 1590 TFLOP/s fallback peak, the kernel's factored count 2 N^2 (nocc + nb + 1) 100 TFLOP/s,
and the issued slice products (12 x 32 + 12 x 128 per pair) 691 TFLOP/s.
"""
import pytest

import bench
from tcscf_b200 import ffi

KR = dict(n=406_000, nb=120, nocc=18)


def test_split_bf16_roofline_at_kr():
    r = bench.roofline(ffi.PREC_BF16X3, KR["n"], KR["nb"], KR["nocc"], 458.2, bench.PEAKS_FALLBACK, "fallback", 2.889e10)
    n2 = KR["n"] ** 2
    assert r["bound"] == "tensor" and r["unit"] == "TFLOP/s" and r["peak"] == 1590.0
    assert r["achieved"] == pytest.approx(2 * n2 * (120 * 18 + 1) / 0.4582 / 1e12)
    assert r["achieved"] == pytest.approx(1554.8, abs=0.1)
    assert r["frac"] == pytest.approx(r["achieved"] / 1590.0)
    assert r["kernel_algorithm_tflops"] == pytest.approx(2 * n2 * (18 + 120 + 1) / 0.4582 / 1e12)
    assert r["issued_tensor_tflops"] == pytest.approx(690.7, abs=0.1)
    assert r["issued_frac"] == pytest.approx(690.7 / 1590.0, abs=1e-4)
    assert r["traffic"] == 2.889e10 and "fallback" in r["peak_source"]


def test_tf32_and_fp64_rooflines():
    t = bench.roofline(ffi.PREC_TF32, KR["n"], KR["nb"], KR["nocc"], 312.0, bench.PEAKS_FALLBACK, "fallback", None)
    assert t["peak"] == 795.0 and t["frac"] == pytest.approx(t["achieved"] / 795.0)
    # one rank chunk of 32: GEMM1 2 x 32 and GEMM2 2 x 128 flops per pair
    assert t["issued_tensor_tflops"] == pytest.approx(KR["n"] ** 2 * (64 + 256) / 0.312 / 1e12)
    f = bench.roofline(ffi.PREC_FP64, KR["n"], KR["nb"], KR["nocc"], 3770.0, bench.PEAKS_FALLBACK, "fallback", None)
    assert f["bound"] == "fp64" and f["peak"] == 37.0 and "issued_tensor_tflops" not in f
    # the FP64 kernel's roofline counts the factored flops it performs; F_alg is its effective rate
    assert f["achieved"] == pytest.approx(2 * KR["n"] ** 2 * (18 + 120 + 1) / 3.77 / 1e12)
    assert f["effective_tflops"] == pytest.approx(2 * KR["n"] ** 2 * 2161 / 3.77 / 1e12)
    # measured matmul rates take precedence over the nominal FP64 figure and the half-BF16 TF32 rule
    m = dict(bench.PEAKS_FALLBACK, fp64_tflops=35.5, tf32_tflops=820.0)
    f = bench.roofline(ffi.PREC_FP64, KR["n"], KR["nb"], KR["nocc"], 3770.0, m, "fallback", None)
    assert f["peak"] == 35.5 and "measured" in f["peak_source"]
    t = bench.roofline(ffi.PREC_TF32, KR["n"], KR["nb"], KR["nocc"], 312.0, m, "fallback", None)
    assert t["peak"] == 820.0 and "measured" in t["peak_source"]


def test_measured_peaks_take_precedence(tmp_path, monkeypatch):
    monkeypatch.setattr(bench, "ROOT", tmp_path)
    assert bench.load_peaks() == (bench.PEAKS_FALLBACK, "fallback")
    (tmp_path / "MEASURED_PEAKS.json").write_text('{"hbm_gbs": 6555.8, "bf16_tflops": 1651.8, "bf16_tflops_sustained": 1395.3}')
    peaks, kind = bench.load_peaks()
    assert kind == "measured" and peaks["bf16_tflops"] == 1651.8


def test_symmetric_pair_counts_and_roofline():
    # one grid as r1 and r2: each 128-point r1 tile from its own diagonal on (the diagonal tile in full)
    n = KR["n"]
    tiles, blocks = -(-n // 128), -(-n // 64)
    assert bench.symmetric_pairs(n) == sum(128 * 64 * (blocks - 2 * p) for p in range(tiles)) == 82_450_481_152
    assert bench.symmetric_pairs(n, fp64=True) == sum(128 * (n - 128 * p) for p in range(tiles))
    assert abs(bench.symmetric_pairs(n) / n ** 2 - 0.5) < 1e-3
    r = bench.roofline(ffi.PREC_BF16X3, n, KR["nb"], KR["nocc"], 233.6, bench.PEAKS_FALLBACK, "fallback", 2.889e10, sym=True)
    assert r["symmetric"] and r["pairs"] == 82_450_481_152
    assert r["achieved"] == pytest.approx(2 * 82_450_481_152 * 2161 / 0.2336 / 1e12)
    assert r["full_pairs_tflops"] == pytest.approx(2 * n ** 2 * 2161 / 0.2336 / 1e12)
    # traffic given for a full launch scales with the units computed
    assert r["traffic"] == pytest.approx(2.889e10 * 82_450_481_152 / (tiles * 128 * blocks * 64))
    # ... and a per-pair figure measured on a symmetric launch takes precedence
    rs = bench.roofline(ffi.PREC_BF16X3, n, KR["nb"], KR["nocc"], 233.6, bench.PEAKS_FALLBACK, "fallback", 2.889e10, sym=True,
                        traffic_per_pair_sym=bench.TRAFFIC_BYTES_PER_PAIR_SYM["Kr"])
    assert rs["traffic"] == pytest.approx((2.4566e9 + 0.2366e9) / 3.4848e10 * 82_450_481_152)
    f = bench.roofline(ffi.PREC_FP64, n, KR["nb"], KR["nocc"], 1610.0, bench.PEAKS_FALLBACK, "fallback", None, sym=True)
    assert f["symmetric"] and f["achieved"] == pytest.approx(2 * bench.symmetric_pairs(n, fp64=True) * 139 / 1.61 / 1e12)
    # TF32 keeps the full contraction
    t = bench.roofline(ffi.PREC_TF32, n, KR["nb"], KR["nocc"], 312.0, bench.PEAKS_FALLBACK, "fallback", None, sym=True)
    assert not t["symmetric"] and t["pairs"] == float(n) ** 2

"""The fixed-point split-BF16 arithmetic of the tensor-core contraction, emulated on the CPU.

The kernel (tcscf_b200/csrc/flash_tc.cu) writes each operand row u with a power-of-two scale s so
that the largest |u s| lies in [2^23, 2^24), as u s = 65536 h + 256 m + l with integers |h| <= 256,
|m|, |l| <= 128.  Its accuracy rests on four facts checked here with numpy (BF16 rounding emulated
bit-exactly, round to nearest even):
  * every slice is exactly representable in BF16 and the slices reconstruct round(u s) exactly;
  * the hi x hi products of a block, summed over K <= 64, stay below 2^23, so an FP32 accumulator
    holds them exactly in any summation order (the tensor core's adder rounding cannot bias them);
  * the cross sum B = h m' + m h' + (h l' + l h' + m m') / 256 is 2^-8 below A, so its own FP32
    rounding enters the result at about 2^-32 relative;
  * rho = 2^24 (256 A + B) / (s1 s2) matches the FP64 product within 2^-24 of the bound
    max|u1| max|u2| K (measured 2^-26), and the 24-bit X times 24-bit Vt product of GEMM2 likewise.
"""
import numpy as np

RNG = np.random.default_rng(20261204)


def bf16(x):
    """Round float32 values to BF16 (8 significant bits), nearest even, returned as float32."""
    b = np.asarray(x, dtype=np.float32).view(np.uint32).astype(np.uint64)
    b = (b + 0x7FFF + ((b >> 16) & 1)) & 0xFFFF0000
    return b.astype(np.uint32).view(np.float32)


def slices24(u):
    """Row-wise scale and 24-bit slices (h, m, l) of a 2-D FP64 array, as the packing kernels do."""
    mx = np.abs(u).max(axis=1, keepdims=True)
    e = np.floor(np.log2(np.where(mx > 0, mx, 1.0)))
    s = 2.0 ** (23 - e)
    t = np.rint(u * s)
    h = np.rint(t / 65536)
    r = t - 65536 * h
    m = np.rint(r / 256)
    lo = r - 256 * m
    return s, h, m, lo, t


def fp32_sum(prod):
    """Sequential FP32 accumulation over the last axis (one order a tensor core may take)."""
    acc = np.zeros(prod.shape[:-1], dtype=np.float32)
    for k in range(prod.shape[-1]):
        acc = np.float32(acc + prod[..., k].astype(np.float32))
    return acc


def test_slices_are_exact_bf16_integers_and_reconstruct():
    u = RNG.normal(size=(128, 32)) * np.exp(RNG.normal(size=(128, 1)) * 3)
    s, h, m, lo, t = slices24(u)
    assert np.abs(h).max() <= 256 and np.abs(m).max() <= 128 and np.abs(lo).max() <= 128
    for part in (h, m, lo):
        assert np.array_equal(bf16(part).astype(np.float64), part)
    assert np.array_equal(65536 * h + 256 * m + lo, t)
    # 24 bits: the rounding is at most half a unit of 2^-23 of the row maximum
    assert (np.abs(t / s - u) <= 0.5 / s).all()


def test_block_hi_sums_are_exact_in_fp32_and_rho_is_accurate():
    K = 64                                   # the larger rank padding
    psi1 = RNG.normal(size=(128, K))
    psi2 = RNG.normal(size=(64, K))
    s1, h1, m1, l1, _ = slices24(psi1)
    s2, h2, m2, l2, _ = slices24(psi2)
    # A: integer products below 2^16, a K-sum below 2^22: exact in FP32 whatever the order
    prodA = h1[:, None, :] * h2[None, :, :]
    assert np.abs(prodA).sum(axis=-1).max() < 2 ** 23
    A32 = fp32_sum(prodA)
    assert np.array_equal(A32.astype(np.float64), prodA.sum(axis=-1))
    A32r = fp32_sum(prodA[..., ::-1])        # another order: identical
    assert np.array_equal(A32, A32r)
    # B: the level 2^-8 below A, accumulated in FP32 (its rounding is 2^-24 of B)
    prodB = (h1[:, None, :] * m2[None] + m1[:, None, :] * h2[None]
             + (h1[:, None, :] * l2[None] + l1[:, None, :] * h2[None] + m1[:, None, :] * m2[None]) / 256)
    B32 = fp32_sum(prodB)
    rho = (256.0 * A32.astype(np.float64) + B32.astype(np.float64)) * 2.0 ** 24 / (s1 * s2.T)
    exact = psi1 @ psi2.T
    scale = np.abs(psi1).max(axis=1, keepdims=True) * np.abs(psi2).max(axis=1)[None, :] * K
    assert (np.abs(rho - exact) / scale).max() < 2 ** -24          # measured 2^-26.1


def test_gemm2_with_24_bit_x_matches_fp64():
    # X (one r1 row block of 64 r2 points) times Vt (64 points x NB columns), both 24-bit
    X = RNG.normal(size=(128, 64)) / (1 + np.abs(RNG.normal(size=(128, 64))) * 10)
    V = RNG.normal(size=(64, 128))
    sx, hx, mx, lx, _ = slices24(X)
    sv, hv, mv, lv, _ = slices24(V.T)        # column scales of Vt
    A = fp32_sum(hx[:, None, :] * hv[None, :, :]).astype(np.float64)
    B = fp32_sum(mx[:, None, :] * hv[None] + hx[:, None, :] * mv[None]
                 + (hx[:, None, :] * lv[None] + lx[:, None, :] * hv[None] + mx[:, None, :] * mv[None]) / 256).astype(np.float64)
    T = (256 * A + B) * 2.0 ** 24 / (sx * sv.T)
    exact = X @ V
    scale = np.abs(X).max(axis=1, keepdims=True) * np.abs(V).max(axis=0)[None, :] * 64
    assert (np.abs(T - exact) / scale).max() < 2 ** -24            # measured 2^-26.2

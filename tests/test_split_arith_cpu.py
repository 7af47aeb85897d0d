"""CPU checks of the integer tricks of the split product's column kernels
(gpu-fft_b200/csrc/gf_split.cuh), restated with numpy float32 / int64
arithmetic:

* rounding by one addition: for float32 |v| < 2^22, v + 1.5 2^23 is exact to
  the nearest integer (ties to even, like rintf), subtracting 1.5 2^23 gives
  that integer back exactly, and the sum's encoding minus 0x4B400000 is it;
* add_shifted(acc, i, sh) = acc + i 2^sh modulo 2^64 for every shift, through
  its three forms (wide multiply-add below 2^31, a high-word add from 2^32, a
  64-bit shift at 31);
* digit_f: a w-bit digit u placed in the mantissa of 2^23 and reduced by
  2^23 + 2^(w-1) gives u - 2^(w-1) exactly;
* the 32-bit digit extraction equals the 64-bit one whenever every value fits
  an int32 and w (k - 1) <= 30."""
import numpy as np
import pytest

MAGIC = np.float32(12582912.0)
MAGIC_BITS = 0x4B400000


def test_rounding_by_one_addition():
    rng = np.random.default_rng(1)
    v = np.concatenate([
        rng.uniform(-(1 << 22) + 1, (1 << 22) - 1, 200000),
        np.arange(-40, 40) / 2.0,  # halves: ties to even
        rng.integers(-(1 << 21), 1 << 21, 1000) + 0.5,
        [-(1 << 22) + 0.5, (1 << 22) - 0.5, -0.0, 0.0],
    ]).astype(np.float32)
    t = (v + MAGIC).astype(np.float32)
    back = (t - MAGIC).astype(np.float32)
    assert np.array_equal(back, np.rint(v))
    ints = t.view(np.int32).astype(np.int64) - MAGIC_BITS
    assert np.array_equal(ints, np.rint(v).astype(np.int64))


def add_shifted(acc, i, sh):
    """The kernel's three forms, in unsigned 64-bit arithmetic."""
    if sh <= 30:
        return (acc + i * (1 << sh)) % (1 << 64)
    if sh >= 32:
        hi = ((i % (1 << 32)) << (sh - 32)) % (1 << 32)  # (unsigned)i << (sh - 32)
        return (acc + (hi << 32)) % (1 << 64)
    return (acc + (i % (1 << 64) << sh)) % (1 << 64)


@pytest.mark.parametrize("sh", list(range(0, 64)))
def test_add_shifted_is_a_shifted_add_mod_2_64(sh):
    rng = np.random.default_rng(sh)
    for _ in range(50):
        acc = int(rng.integers(0, 1 << 63)) * 2 + int(rng.integers(0, 2))
        i = int(rng.integers(-(1 << 22), 1 << 22))
        want = (acc + i * (1 << sh)) % (1 << 64)
        assert add_shifted(acc, i, sh) == want


def digit_f(u, w):
    bias = np.float32(8388608.0 + (1 << (w - 1)))
    return (np.array([u | 0x4B000000], np.uint32).view(np.float32) - bias).astype(np.float32)[0]


@pytest.mark.parametrize("w", [1, 3, 5, 8, 12, 20])
def test_digit_through_the_mantissa(w):
    for u in list(range(min(1 << w, 64))) + [(1 << w) - 1]:
        assert digit_f(u, w) == np.float32(u - (1 << (w - 1)))


@pytest.mark.parametrize("w,k,bits,nonneg", [(5, 5, 24, True), (6, 4, 24, False), (4, 7, 24, True), (8, 3, 20, False)])
def test_32_bit_digits_equal_64_bit_digits(w, k, bits, nonneg):
    K = (1 << (bits - 1)) if nonneg else 0
    hoff = sum(1 << (w * i + w - 1) for i in range(k - 1))
    voff = hoff - K
    lo = 0 if nonneg else -(1 << bits) + 1
    hi = (1 << bits) - 1
    assert lo + voff >= -(1 << 31) and hi + voff < (1 << 31) and w * (k - 1) <= 30
    rng = np.random.default_rng(w * 100 + k)
    x = np.concatenate([rng.integers(lo, hi + 1, 20000), [lo, hi]])
    V = x.astype(np.int64) + voff
    V32 = V.astype(np.int32)
    mask, half = (1 << w) - 1, 1 << (w - 1)
    for l in range(k):
        if l < k - 1:
            d64 = ((V >> (w * l)) & mask) - half
            d32 = ((V32.view(np.uint32) >> np.uint32(w * l)) & np.uint32(mask)).astype(np.int64) - half
        else:
            d64 = V >> (w * l)
            d32 = (V32 >> np.int32(w * l)).astype(np.int64)
        assert np.array_equal(d32, d64), l

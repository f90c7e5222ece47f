"""The numeric argument behind the tcgen05 M2L's FP16 operands, checked on the
CPU with numpy's IEEE FP16 (no GPU): a level's multipoles (or the operator
set) are scaled by 2^e so that the largest magnitude lands in [2^14, 2^15)
(below FP16's largest finite value, 65504), then split into hi = fp16(x)
and lo = fp16(x - hi).  The pair keeps x to 2^-22 relative plus an absolute
floor of 2^-25 in scaled units (2^-39 of the largest value), so
B_hi T_hi + B_hi T_lo + B_lo T_hi matches a TF32 hi/lo split's accuracy on
the products the kernel forms.  The exponent rule restates f16_exponent in
csrc/m2l_tc.cu (float bits of the largest magnitude)."""
import numpy as np


def f16_exponent(mx: float) -> int:
    """e with 2^e * mx in [2^14, 2^15), from the float32 bits of mx, clamped
    to [-126, 126] (the kernel's rule)."""
    bits = int(np.float32(mx).view(np.uint32))
    e = 14 - (((bits >> 23) & 255) - 127) if bits else 0
    return max(-126, min(126, e))


def split(x):
    hi = x.astype(np.float16)
    lo = (x - hi.astype(np.float32)).astype(np.float16)
    return hi, lo


def test_scale_lands_below_fp16_max():
    """The scaled largest magnitude lands in [2^14, 2^15); below 2^-112 the
    exponent stops at 126 (so that 2^-e, the outputs' scale, stays a normal
    float) and the value stays below 2^14, still finite in FP16."""
    rng = np.random.default_rng(3)
    for mx in np.concatenate([10.0 ** rng.uniform(-30, 38, 500), [1.0, 2.0 ** 14, 65504.0, 3.0e38]]):
        mx = np.float32(mx)
        e = f16_exponent(mx)
        y = np.float32(mx) * np.float32(2.0 ** e)
        assert 2.0 ** 14 <= y < 2.0 ** 15, (mx, e, y)
        assert np.isfinite(np.float16(y))
    for mx in (1.5e-38, 2.0 ** -113):
        e = f16_exponent(mx)
        y = np.float32(mx) * np.float32(2.0 ** e)
        assert e == 126 and 0 < y < 2.0 ** 14 and np.isfinite(np.float16(y))
    assert f16_exponent(0.0) == 0


def test_hi_lo_error_bound():
    """|hi + lo - x| <= 2^-22 |x| + 2^-25 for x across FP16's range once scaled."""
    rng = np.random.default_rng(4)
    x = (rng.choice([-1, 1], 200000) * 2.0 ** rng.uniform(-40, 15, 200000)).astype(np.float32)
    hi, lo = split(x)
    err = np.abs(hi.astype(np.float64) + lo.astype(np.float64) - x.astype(np.float64))
    assert np.all(err <= 2.0 ** -22 * np.abs(x) + 2.0 ** -25)


def test_three_products_match_fp32_level():
    """A dot product of scaled operands with a wide dynamic range (decaying by
    degree, as multipoles and translation operators do): the three FP16
    products land within a few 1e-7 of the exact result, relative to the sum
    of the magnitudes; hi x hi alone misses by ~1e-4."""
    rng = np.random.default_rng(5)
    K = 288
    decay = 0.7 ** (np.arange(K) // 16)
    worst3 = worst1 = 0.0
    for _ in range(200):
        b = (rng.standard_normal(K) * decay * 10.0 ** rng.uniform(-3, 3)).astype(np.float32)
        t = (rng.standard_normal(K) * decay).astype(np.float32)
        sb, st = 2.0 ** f16_exponent(np.abs(b).max()), 2.0 ** f16_exponent(np.abs(t).max())
        bh, bl = split((b * sb).astype(np.float32))
        th, tl = split((t * st).astype(np.float32))
        f = lambda u, v: np.dot(u.astype(np.float64), v.astype(np.float64))
        exact = f(b, t)
        scale = np.dot(np.abs(b).astype(np.float64), np.abs(t).astype(np.float64))
        three = (f(bh, th) + f(bh, tl) + f(bl, th)) / (sb * st)
        one = f(bh, th) / (sb * st)
        worst3 = max(worst3, abs(three - exact) / scale)
        worst1 = max(worst1, abs(one - exact) / scale)
    assert worst3 < 3e-7
    assert worst1 > 1e-5

"""The conversion-free fixed-point rounding used by the mixed form.

The resident kernel family sums rint(v * 2^32) per cell, formed as two
signed limbs, hi * 2^20 + lo, from FP32 adds and multiplies only (fx_limbs
in mpcd_mixed.cuh); streaming adds rint(dx * 2^22) to the 22-bit offsets of
the position words, from one multiply and one add (fx_rint22).  This file
restates those steps in numpy float32 arithmetic (IEEE round-to-nearest-even,
as the __fadd_rn/__fmul_rn intrinsics) and checks them against exact float64
rounding over random and adversarial inputs; the GPU test of the streaming
rounding is in test_gpu_fixed_point.py.
"""
import numpy as np

F = np.float32
MAGIC = F(12582912.0)  # 1.5 * 2^23


def _bits(x):
    return int(np.array(F(x), dtype=np.float32).view(np.int32))


def limbs(v):
    v = F(v)
    a = F(v * F(4096.0))
    if not abs(a) < F(4194304.0):
        return None
    s = F(a + MAGIC)
    r = F(s - MAGIC)
    g = F(F(a - r) * F(1048576.0))
    hi = _bits(s) - 0x4B400000
    lo = _bits(F(g + MAGIC)) - 0x4B400000
    return hi, lo


def exact(v):
    x = float(F(v)) * 2.0 ** 32
    return int(np.rint(x))  # ties to even, exact in float64 for |v| < 1024


def _check(vals):
    for v in vals:
        hl = limbs(v)
        assert hl is not None, v
        h, l = hl
        assert -(1 << 19) <= l <= (1 << 19), (v, h, l)
        assert h * (1 << 20) + l == exact(v), (float(v), h, l, exact(v))


def test_random_magnitudes():
    rng = np.random.default_rng(3)
    mant = rng.random(20000).astype(np.float32) + F(1.0)
    expo = rng.integers(-40, 10, size=20000)
    sign = np.where(rng.random(20000) < 0.5, -1.0, 1.0)
    _check((sign * mant * np.exp2(expo)).astype(np.float32))


def test_ties_and_edges():
    vals = []
    for k in range(1, 200, 2):  # exact halves of 2^-32: ties
        vals += [F(k * 2.0 ** -33), F(-k * 2.0 ** -33)]
    vals += [F(0.0), F(-0.0), F(2.0 ** -32), F(-(2.0 ** -32)), F(1023.9999), F(-1023.9999),
             F(0.5), F(-0.5), F(1.0), F(-1.0), np.nextafter(F(1.0), F(0.0)),
             -np.nextafter(F(1.0), F(0.0)), F(2.0 ** -12), F(-(2.0 ** -12)),
             F(3.0 * 2.0 ** -13), F(-3.0 * 2.0 ** -13)]
    _check(vals)


def test_out_of_range_is_refused():
    assert limbs(F(1024.0)) is None
    assert limbs(F(-5000.0)) is None
    assert limbs(F(np.inf)) is None
    assert limbs(F(np.nan)) is None


def rint22(dx):
    s = F(F(F(dx) * F(4194304.0)) + MAGIC)
    return _bits(s) - 0x4B400000


def test_stream_rounding_rint22():
    rng = np.random.default_rng(5)
    vals = (rng.random(20000) * 1.998 - 0.999).astype(np.float32)
    vals = np.concatenate([vals, np.array([k * 2.0 ** -23 for k in range(-41, 42, 2)],
                                          dtype=np.float32)])  # exact ties
    for dx in vals:
        assert rint22(dx) == int(np.rint(float(dx) * 2.0 ** 22)), float(dx)

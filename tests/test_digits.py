"""The base-128 digit form of the tensor-core slices, restated on the host.

Every slicer (density_tc.cuh digits_m / digit_field / pack_digits) rounds
x 2^42 once on the FP64 adder, t = 2^52 + B + x 2^42 with
B = 64 (128^6 - 1) / 127, and reads six 7-bit fields of t's mantissa less 64
as balanced digits. This checks, with numpy doing the same bit operations, the
claims the kernels rely on: the digits reconstruct rint(x 2^42) / 2^42 exactly
(so |x - sum| <= 2^-43), every |digit| <= 64 (the level accumulators' int32
bound assumes it), and the byte-wise packing gives the int8 value of each
digit, the top one (which can reach +64) included. The GPU parity tests check
the device code itself against the oracle.
"""
import numpy as np

B = 64 * (128**6 - 1) // 127
C = float(2**52 + B)  # the constant of digits_m


def _fields(x):
    """t's 32-bit halves and the low byte of each slice's field, as digit_field takes them."""
    t = x * 2.0**42 + C  # x 2^42 is exact (a power-of-two scale): one rounding, as the FMA
    bits = t.view(np.uint64)
    lo = bits & np.uint64(0xFFFFFFFF)
    hi = bits >> np.uint64(32)
    f = [hi >> np.uint64(3),                                              # slice 0: bits 35..42
         ((lo >> np.uint64(28)) | (hi << np.uint64(4))) & np.uint64(0xFFFFFFFF),  # slice 1 (funnel shift)
         lo >> np.uint64(21), lo >> np.uint64(14), lo >> np.uint64(7), lo]
    return [(v & np.uint64(0xFF)).astype(np.int64) for v in f], lo, hi


def _pack_byte(w, top):
    """pack_digits on one byte lane: (m - 64) as int8, without carries between bytes."""
    low = (w & 0x7F) + 0x40
    z = low ^ (((w ^ 0xC0) & 0x80) if top else 0x80)
    z &= 0xFF
    return np.where(z >= 128, z - 256, z)


def _cases():
    rng = np.random.default_rng(7)
    edge = np.array([0.0, 2.0**-43, -2.0**-43, 3 * 2.0**-44, -3 * 2.0**-44, 0.496, -0.496,
                     np.nextafter(0.5, 0.0), -np.nextafter(0.5, 0.0), 0.25, -0.25])
    ties = (rng.integers(-2**41, 2**41, 20000) + 0.5) / 2.0**42  # remainders that tie
    return np.concatenate([rng.uniform(-0.5, 0.5, 200000), edge, ties])


def test_constant_is_even_and_exact():
    assert B % 2 == 0 and C == 2**52 + B
    assert B < 2**42 and B - 2**41 > 0  # B + x 2^42 stays in [0, 2^52) for |x| < 1/2


def test_digits_reconstruct_the_rounded_value():
    x = _cases()
    fields, lo, hi = _fields(x)
    m = ((hi & np.uint64(0xFFFFF)) << np.uint64(32)) | lo
    assert np.all(m.astype(np.int64) - B == np.rint(x * 2.0**42).astype(np.int64))
    d = np.stack([_pack_byte(f, s == 0) for s, f in enumerate(fields)])
    assert np.all(np.abs(d) <= 64)
    rec = sum(d[s].astype(np.float64) * 128.0 ** (-(s + 1)) for s in range(6))
    assert np.all(rec == np.rint(x * 2.0**42) / 2.0**42)
    assert np.all(np.abs(rec - x) <= 2.0**-43)


def test_top_digit_reaches_64():
    x = np.array([np.nextafter(0.5, 0.0), 0.4999])
    fields, _, _ = _fields(x)
    assert np.all(_pack_byte(fields[0], True) == 64)

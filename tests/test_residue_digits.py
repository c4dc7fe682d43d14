"""A CPU model of the residue arithmetic of the split DGEMM's operand kernels
(write_residues8 in csrc/ozaki.cu): an integer operand v is written in
balanced digits b_t of 14 bits (four digits, |v| <= 2^50 or 2^52) or 16 bits
(three digits, |v| <= 2^47); per odd modulus m the digit sum
s = sum_t b_t c_t with c_t = 2^(bits t) mods m is formed in FP32, the quotient
q = rint(s / m) from one FMA of s with fl(1/m) against 1.5 2^23, and the
residue r = s - m q, whose low byte goes to the residue plane.

Checked at the edges and at random values of each form's range, for every
modulus: every partial sum is an integer below 2^24 (so FP32 holds it
exactly), |s| stays below the bound the quotient needs (|s| 2^-24 / m <
1/(2m), i.e. |s| < 2^23), and r is the symmetric residue of v.  The FP32
quotient is modelled exactly: the FMA's rounding of s * fl(1/m) + 1.5 2^23 to
the nearest FP32 value (spacing 1 there, ties to even) is the rounding of the
exact rational value.
"""
import random
from fractions import Fraction

import numpy as np
import pytest

MODULI = [255, 253, 251, 247, 241, 239, 233, 229, 227, 223, 217, 211, 199, 197, 193]
MAGIC = 3 << 22  # 1.5 * 2^23


def mods(x, m):
    r = x % m
    return r - m if r > (m - 1) // 2 else r


def digits(v, form):
    """Balanced digits of v and their bit widths (the kernels' bias trick)."""
    if form == "d16":
        width, n = 16, 3
    else:
        width, n = 14, 4
    half = 1 << (width - 1)
    bias = sum(half << (width * t) for t in range(n))
    w = v + bias
    assert w >= 0
    us = [(w >> (width * t)) & ((1 << width) - 1) for t in range(n - 1)]
    us.append(w >> (width * (n - 1)))  # the top digit keeps the rest
    bs = [u - half for u in us]
    assert sum(b << (width * t) for t, b in enumerate(bs)) == v
    return bs, width


def residue(v, m, form):
    bs, width = digits(v, form)
    cs = [mods(1 << (width * t), m) for t in range(len(bs))]
    s = bs[0]
    for b, c in zip(bs[1:], cs[1:]):
        prod = b * c
        assert abs(prod) < 1 << 24 and abs(s + prod) < 1 << 24, "FP32 partial sum not exact"
        s += prod
    assert abs(s) < 1 << 23, f"|s| = {abs(s)} breaks the quotient bound"
    inv = Fraction(float(np.float32(1.0 / m)))  # fl(1/m) in FP32
    q = round(Fraction(s) * inv + MAGIC) - MAGIC  # the FMA, rounded to nearest even
    r = s - m * q
    assert abs(r) <= m // 2, "quotient off by one"
    return r


def edge_values(limit):
    vals = [0, 1, -1, limit, -limit, limit - 1, -(limit - 1)]
    vals += [(1 << k) - 1 for k in range(1, limit.bit_length())]
    vals += [-(1 << k) for k in range(1, limit.bit_length())]
    return vals


@pytest.mark.parametrize("form,bits", [("d16", 47), ("d14", 50), ("d14", 52)])
def test_residues_of_every_modulus(form, bits):
    rng = random.Random(bits)
    limit = 1 << bits
    vals = edge_values(limit) + [rng.randint(-limit, limit) for _ in range(300)]
    for m in MODULI:
        for v in vals:
            assert residue(v, m, form) == mods(v, m), (form, m, v)


def test_low_byte_is_the_residue_of_256():
    """Modulus 256: both digit biases are multiples of 256, so the low byte of
    the biased word is v's two's complement byte."""
    for form, width, n in (("d16", 16, 3), ("d14", 14, 4)):
        bias = sum((1 << (width - 1)) << (width * t) for t in range(n))
        assert bias % 256 == 0, form
        for v in (-(1 << 47), -1, 0, 1, 12345, (1 << 47) - 3):
            assert ((v + bias) & 0xFF) == (v & 0xFF)


def test_sixteen_bit_digits_need_the_47_bit_bound():
    """The worst case of |s| over the digits of |v| <= 2^bits: the top digit
    reaches 2^(bits - 32).  Below 2^23 for every modulus at 47 bits; at 48
    bits some modulus exceeds it, so the three-digit form stops at 47."""
    def worst(bits, m):
        c16, c32 = abs(mods(1 << 16, m)), abs(mods(1 << 32, m))
        return (1 << 15) * (1 + c16) + (1 << (bits - 32)) * c32

    assert all(worst(47, m) < 1 << 23 for m in MODULI)
    assert any(worst(48, m) >= 1 << 23 for m in MODULI)

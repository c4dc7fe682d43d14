"""A CPU model of the split DGEMM's reconstruction (the `reconstruct` kernel
in csrc/ozaki.cu): from the residues r_l = C' mods m_l of an integer
|C'| <= M/8 it forms, in FP64,

  X = sum_l r_l w_hi[l]  (exact: every partial sum is below 2^53),
  Y = sum_l r_l w_lo[l]  (FMAs, rounded),

with the CRT weights w_l = w_hi[l] 2^T + w_lo[l], and the quotient estimate
t = X (2^T / M) + Y / M -- within ~1e-12 of sum_l r_l w_l / M, which lies
within 1/8 of the integer q -- so q = rint(t), and then
C' = (X - q M_hi) 2^T + (Y - q M_lo).

Checked with exact rational arithmetic for each FP64 operation (an FMA is
the exact value rounded once) on edge and random C' for the moduli counts the
DGEMM uses: q is the exact quotient, and C' comes back within one rounding
of itself plus 2^-60 of the range M/8 (the rounding of Y, absolute, which the
scheme's normwise bound covers).
"""
import math
import random
from fractions import Fraction

import pytest

MODULI = [256, 255, 253, 251, 247, 241, 239, 233, 229, 227, 223, 217, 211, 199, 197, 193]


def rnd(x):
    """The double nearest to the rational x (ties to even)."""
    return float(x)  # Fraction.__float__ rounds correctly


def fma(a, b, c):
    return rnd(Fraction(a) * Fraction(b) + Fraction(c))


def plan(nmod):
    M = math.prod(MODULI[:nmod])
    logM = M.bit_length() - 1
    T = max(0, logM + 1 + 7 + math.ceil(math.log2(nmod + 1)) + 1 - 52)
    mask = (1 << T) - 1
    ws = []
    for m in MODULI[:nmod]:
        Ml = M // m
        ws.append(Ml * pow(Ml % m, -1, m))
    return dict(M=M, T=T, w_hi=[float(w >> T) for w in ws], w_lo=[rnd(Fraction(w & mask)) for w in ws],
                M_hi=float(M >> T), M_lo=rnd(Fraction(M & mask)),
                # as the plan forms them: double(2^T) / double(M), 1 / double(M)
                t_x=float(2**T) / float(M), t_y=1.0 / float(M), w=ws)


def mods(x, m):
    r = x % m
    return r - m if r > (m - 1) // 2 else r


def reconstruct(c, p, nmod):
    rs = [mods(c, m) for m in MODULI[:nmod]]
    X, Y = 0.0, 0.0
    for r, wh, wl in zip(rs, p["w_hi"], p["w_lo"]):
        X = fma(r, wh, X)
        Y = fma(r, wl, Y)
    assert abs(sum(r * int(wh) for r, wh in zip(rs, p["w_hi"]))) < 2**53
    t = fma(X, p["t_x"], rnd(Fraction(Y) * Fraction(p["t_y"])))
    q = round(t)
    q_exact = (sum(r * w for r, w in zip(rs, p["w"])) - c) // p["M"]
    assert sum(r * w for r, w in zip(rs, p["w"])) - c == q_exact * p["M"]
    assert abs(t - q_exact) < 1 / 8 + 1e-9, "estimate outside the margin"
    assert q == q_exact, "quotient"
    hi = fma(-q, p["M_hi"], X)
    lo = fma(-q, p["M_lo"], Y)
    return fma(hi, 2.0**p["T"], lo)


@pytest.mark.parametrize("nmod", [9, 13, 14, 16])
def test_reconstruction_of_every_range(nmod):
    p = plan(nmod)
    bound = p["M"] // 8
    rng = random.Random(nmod)
    cs = [0, 1, -1, bound, -bound, bound - 1, -(bound - 1)]
    cs += [rng.randint(-bound, bound) for _ in range(400)]
    cs += [rng.randint(-(1 << 30), 1 << 30) for _ in range(100)]
    for c in cs:
        got = reconstruct(c, p, nmod)
        err = abs(Fraction(got) - c)
        assert err <= abs(Fraction(c, 2**52)) + Fraction(bound, 2**60), (nmod, c)

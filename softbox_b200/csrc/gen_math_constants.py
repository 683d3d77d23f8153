"""Derive the split constants used by sbx_math.h.

Computes pi/2 and ln 2 to 60 decimal digits with the standard library's
decimal module (Machin's formula for pi, 2*atanh(1/3) for ln 2) and splits
them Cody-Waite style into a head with a short significand (so that k*head
is exact for the small multipliers k used here) plus correction terms.

Run:  python softbox_b200/csrc/gen_math_constants.py
"""
from decimal import Decimal, getcontext
import struct

getcontext().prec = 80


def atan_inv(n):
    # atan(1/n) = sum (-1)^k / ((2k+1) n^(2k+1))
    x = Decimal(1) / n
    x2 = x * x
    term, k, s = x, 0, Decimal(0)
    while True:
        t = term / (2 * k + 1)
        if t < Decimal(10) ** -75:
            break
        s += t if k % 2 == 0 else -t
        term *= x2
        k += 1
    return s


def atanh_inv(n):
    x = Decimal(1) / n
    x2 = x * x
    term, k, s = x, 0, Decimal(0)
    while True:
        t = term / (2 * k + 1)
        if t < Decimal(10) ** -75:
            break
        s += t
        term *= x2
        k += 1
    return s


PI = 16 * atan_inv(5) - 4 * atan_inv(239)
LN2 = 2 * atanh_inv(3)


def trunc_bits(d, keep):
    """Round Decimal d to double, then clear all but `keep` significand bits."""
    f = float(d)
    bits = struct.unpack('<Q', struct.pack('<d', f))[0]
    drop = 52 - (keep - 1)
    bits &= ~((1 << drop) - 1)
    return struct.unpack('<d', struct.pack('<Q', bits))[0]


def split3(d, keep=33):
    hi = trunc_bits(d, keep)
    mid = trunc_bits(d - Decimal(hi), keep)
    lo = float(d - Decimal(hi) - Decimal(mid))
    return hi, mid, lo


def split2(d, keep=32):
    hi = trunc_bits(d, keep)
    lo = float(d - Decimal(hi))
    return hi, lo


if __name__ == "__main__":
    p1, p2, p3 = split3(PI / 2)
    l1, l2 = split2(LN2)
    print("PIO2_HI  =", p1.hex(), repr(p1))
    print("PIO2_MID =", p2.hex(), repr(p2))
    print("PIO2_LO  =", p3.hex(), repr(p3))
    print("TWO_OVER_PI =", float(2 / PI).hex())
    print("LN2_HI   =", l1.hex(), repr(l1))
    print("LN2_LO   =", l2.hex(), repr(l2))
    print("INV_LN2  =", float(1 / LN2).hex())
    print("PI       =", float(PI).hex(), repr(float(PI)))
    print("SQRT2    =", float(Decimal(2).sqrt()).hex())

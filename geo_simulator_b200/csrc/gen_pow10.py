"""Generates pow10_table.h (CUDA): the 126-bit over-approximations of 10^-k used by the
shortest-decimal conversion in decimal.cuh (Giulietti's Schubfach method):

    g(k) = floor(10^-k * 2^(125 - floor(-k * log2(10)))) + 1,   k = -324 .. 292,

split into 63-bit limbs g1 = g >> 63, g0 = g & (2^63 - 1). Exact integer
arithmetic; also checks the multiply-shift forms of floor(q log10 2),
floor(log10(3/4 * 2^q)) and floor(e log2 10) over the ranges they are used on.

    python gen_pow10.py > pow10_table.h
"""
from fractions import Fraction

K_MIN, K_MAX = -324, 292
C10_2, C10_34, C2_10 = 661971961083, -274743187321, 913124641741   # fixed-point logs (2^41, 2^41, 2^38)


def floor_log2_pow10(e):  # floor(e * log2 10), exact
    x = Fraction(10) ** e
    n = x.numerator.bit_length() - x.denominator.bit_length()
    while Fraction(2) ** n > x:
        n -= 1
    while Fraction(2) ** (n + 1) <= x:
        n += 1
    return n


def floor_log10(x):  # x a positive Fraction
    n = len(str(x.numerator)) - len(str(x.denominator))
    while Fraction(10) ** n > x:
        n -= 1
    while Fraction(10) ** (n + 1) <= x:
        n += 1
    return n


def check():
    for q in range(-1080, 980):
        assert (q * C10_2) >> 41 == floor_log10(Fraction(2) ** q), q
        assert (q * C10_2 + C10_34) >> 41 == floor_log10(Fraction(3, 4) * Fraction(2) ** q), q
    for e in range(-K_MAX - 2, -K_MIN + 2):
        assert (e * C2_10) >> 38 == floor_log2_pow10(e), e


def g(k):
    r = floor_log2_pow10(-k) - 125
    x = Fraction(10) ** (-k) / Fraction(2) ** r
    v = x.numerator // x.denominator + 1
    assert 2 ** 125 <= v < 2 ** 126
    return v


def main():
    check()
    mask = (1 << 63) - 1
    print("// Generated by gen_pow10.py: g(k) = floor(10^-k 2^(125 - floor(-k log2 10))) + 1 as")
    print("// 63-bit limbs {g >> 63, g & (2^63 - 1)}, for k = %d .. %d." % (K_MIN, K_MAX))
    print("#pragma once")
    print("#include <cstdint>")
    print("namespace geo {")
    print("constexpr int kPow10KMin = %d, kPow10KMax = %d;" % (K_MIN, K_MAX))
    print("constexpr int64_t kLog10Pow2 = %dLL, kLog10ThreeQuarters = %dLL, kLog2Pow10 = %dLL;" % (C10_2, C10_34, C2_10))
    print("// device constant memory: include from one CUDA translation unit only")
    print("__constant__ uint64_t kPow10G[%d][2] = {" % (K_MAX - K_MIN + 1))
    for k in range(K_MIN, K_MAX + 1):
        v = g(k)
        print("    {0x%016xULL, 0x%016xULL}," % (v >> 63, v & mask))
    print("};")
    print("}  // namespace geo")


if __name__ == "__main__":
    main()

// Rust's `{}` for f64 and integers, on the device: the number formatting of
// VtkWriter (mesh/vtk_writer.rs), which prints every coordinate, field value
// and index with Display.
//
// Rust's Display for f64 prints the shortest digit string that reads back as v,
// positionally ("0.0000001", "1000000000000000000000", "1", "-0", "NaN", "inf").
// Which string is "shortest" follows its decoder and Dragon4-style generation:
// the interval of reals that round to v = c * 2^q is
// [v - 2^(q-1), v + 2^(q-1)], or [v - 2^(q-2), v + 2^(q-1)] for a normal v with
// all fraction bits zero, the end points included iff c is even; the result is
// the multiple of the largest power of ten the interval holds that lies next to
// v, the nearer of the two when both are inside.
//
// The conversion follows R. Giulietti's Schubfach method ("The Schubfach way to
// render doubles", 2020): with k = floor(log10 of the interval width), 10^-k is
// over-approximated by a 126-bit g (pow10_table.h), and v and the interval end
// points are scaled to units of 10^k / 4 with round-to-odd products, which keeps
// every comparison below exact. In those units the interval is between 1 and 10
// units wide, so it holds at most one multiple of 10; if it holds one, that is
// the answer (Rust's coarser position), else the answer is floor(v) or
// floor(v) + 1 in units of 10^k. Java's two-digit minimum for tiny subnormals
// and its regular treatment of 2^-1022 are not applied: Rust has neither.
#pragma once

#include <cstdint>

#include "pow10_table.h"

namespace geo {

__device__ __forceinline__ int floor_log10_pow2(int q) { return (int)((q * kLog10Pow2) >> 41); }
__device__ __forceinline__ int floor_log10_three_quarters_pow2(int q) {
    return (int)((q * kLog10Pow2 + kLog10ThreeQuarters) >> 41);
}
__device__ __forceinline__ int floor_log2_pow10(int e) { return (int)((e * kLog2Pow10) >> 38); }

// floor(g * cp / 2^127) with the inexact flag ORed into bit 0 (round to odd);
// g = g1 * 2^63 + g0 with 63-bit limbs
__device__ __forceinline__ uint64_t round_to_odd(uint64_t g1, uint64_t g0, uint64_t cp) {
    const uint64_t x1 = __umul64hi(g0, cp);
    const uint64_t y0 = g1 * cp;
    const uint64_t y1 = __umul64hi(g1, cp);
    const uint64_t z = (y0 >> 1) + x1;
    const uint64_t vbp = y1 + (z >> 63);
    const uint64_t m63 = (uint64_t(1) << 63) - 1;
    return vbp | (((z & m63) + m63) >> 63);
}

// Shortest decimal of a positive finite double given by its bits: value = f * 10^e.
__device__ __forceinline__ void shortest_decimal(uint64_t bits, uint64_t& f, int& e) {
    const int bq = (int)((bits >> 52) & 0x7ff);
    const uint64_t bc = bits & ((uint64_t(1) << 52) - 1);
    const uint64_t c = bq ? (bc | (uint64_t(1) << 52)) : bc;
    const int q = bq ? bq - 1075 : -1074;
    const bool irregular = bq != 0 && bc == 0;
    const uint64_t out = c & 1;
    const uint64_t cb = c << 2;
    const uint64_t cbr = cb + 2;
    const uint64_t cbl = irregular ? cb - 1 : cb - 2;
    const int k = irregular ? floor_log10_three_quarters_pow2(q) : floor_log10_pow2(q);
    const int h = q + floor_log2_pow10(-k) + 2;
    const uint64_t g1 = kPow10G[k - kPow10KMin][0], g0 = kPow10G[k - kPow10KMin][1];
    const uint64_t vb = round_to_odd(g1, g0, cb << h);
    const uint64_t vbl = round_to_odd(g1, g0, cbl << h);
    const uint64_t vbr = round_to_odd(g1, g0, cbr << h);
    const uint64_t s = vb >> 2;
    const uint64_t sp10 = (s / 10) * 10, tp10 = sp10 + 10;
    const bool upin = vbl + out <= (sp10 << 2);
    const bool wpin = (tp10 << 2) + out <= vbr;
    uint64_t r;
    if (upin != wpin) {
        r = upin ? sp10 : tp10;
    } else {
        const uint64_t t = s + 1;
        const bool uin = vbl + out <= (s << 2);
        const bool win = (t << 2) + out <= vbr;
        if (uin != win) {
            r = uin ? s : t;
        } else {
            const int64_t d = (int64_t)(vb - ((s + t) << 1));
            r = (d < 0 || (d == 0 && (s & 1) == 0)) ? s : t;
        }
    }
    int ee = k;
    while (r % 10 == 0) {
        r /= 10;
        ++ee;
    }
    f = r;
    e = ee;
}

__device__ __forceinline__ int decimal_digits(uint64_t v) {
    int n = 1;
    uint64_t p = 10;
    while (n < 19 && v >= p) {
        ++n;
        p *= 10;
    }
    if (n == 19 && v >= p) ++n;
    return n;
}

// A formatted f64: kind 0 finite nonzero, 1 zero, 2 infinity, 3 NaN.
struct F64Text {
    uint64_t f;
    int n, x;  // value 0.d1..dn * 10^x
    int kind;
    bool neg;
    int len;
};

__device__ __forceinline__ F64Text f64_text(double v) {
    F64Text t;
    const uint64_t bits = (uint64_t)__double_as_longlong(v);
    const uint64_t mag = bits & ~(uint64_t(1) << 63);
    t.neg = (bits >> 63) != 0;
    t.f = 0;
    t.n = t.x = 0;
    if (mag > 0x7ff0000000000000ull) {
        t.kind = 3;
        t.neg = false;
        t.len = 3;
        return t;
    }
    if (mag == 0x7ff0000000000000ull) {
        t.kind = 2;
        t.len = 3 + t.neg;
        return t;
    }
    if (mag == 0) {
        t.kind = 1;
        t.len = 1 + t.neg;
        return t;
    }
    t.kind = 0;
    int e;
    shortest_decimal(mag, t.f, e);
    t.n = decimal_digits(t.f);
    t.x = e + t.n;
    t.len = t.neg + (t.x <= 0 ? 2 - t.x + t.n : (t.x < t.n ? t.n + 1 : t.x));
    return t;
}

// Writes t.len bytes at p.
__device__ __forceinline__ void f64_write(const F64Text& t, char* p) {
    if (t.neg) *p++ = '-';
    if (t.kind == 3) {
        p[0] = 'N';
        p[1] = 'a';
        p[2] = 'N';
        return;
    }
    if (t.kind == 2) {
        p[0] = 'i';
        p[1] = 'n';
        p[2] = 'f';
        return;
    }
    if (t.kind == 1) {
        p[0] = '0';
        return;
    }
    uint64_t f = t.f;
    if (t.x <= 0) {
        p[0] = '0';
        p[1] = '.';
        for (int j = 0; j < -t.x; ++j) p[2 + j] = '0';
        char* d = p + 2 - t.x;
        for (int j = t.n - 1; j >= 0; --j) {
            d[j] = (char)('0' + f % 10);
            f /= 10;
        }
    } else if (t.x < t.n) {
        for (int j = t.n - 1; j >= 0; --j) {
            p[j < t.x ? j : j + 1] = (char)('0' + f % 10);
            f /= 10;
        }
        p[t.x] = '.';
    } else {
        for (int j = t.n - 1; j >= 0; --j) {
            p[j] = (char)('0' + f % 10);
            f /= 10;
        }
        for (int j = t.n; j < t.x; ++j) p[j] = '0';
    }
}

// Rust `{}` of a non-negative integer.
__device__ __forceinline__ int uint_len(uint64_t v) { return decimal_digits(v); }

__device__ __forceinline__ void uint_write(uint64_t v, int n, char* p) {
    for (int j = n - 1; j >= 0; --j) {
        p[j] = (char)('0' + v % 10);
        v /= 10;
    }
}

}  // namespace geo

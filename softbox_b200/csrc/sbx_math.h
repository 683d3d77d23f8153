// sbx_math.h — scalar arithmetic shared by the CUDA kernels and by host code.
//
// Why this file exists: the reference evaluates Math.log / Math.sin / Math.cos /
// Math.exp in double and rounds the result to float (BrownianForceSystem.java:78-92,
// ChainBendingForceSystem.java:48-84, NucleotideCycleSystem.java:116). To make the
// device and a CPU checker produce the SAME bits, both sides must evaluate the SAME
// double-precision function. This header supplies one portable implementation of
// log, exp, sin and cos written from textbook mathematics:
//
//   * Cody & Waite argument reduction (W. J. Cody, W. Waite, "Software Manual for
//     the Elementary Functions", 1980): x = k*(pi/2) + r with pi/2 split into three
//     doubles, and x = k*ln2 + r with ln2 split into two doubles. The split constants
//     are derived by gen_math_constants.py (decimal arithmetic, 60 digits).
//   * minimax polynomials on the reduced range, evaluated by Horner's rule; their
//     coefficients come from the Remez exchange algorithm (gen_math_polys.py, 60-digit
//     arithmetic), which reaches double accuracy with 6 to 11 terms where the
//     truncated Taylor series of the same functions needs 10 to 14.
//   * log(m) = 2*atanh(f/(2+f)), f = m - 1, m in [sqrt(1/2), sqrt(2)).
//   * the Horner steps and the argument reductions are explicit fused multiply-adds
//     (fmad below: one rounding of a*b + c). CUDA's __fma_rn and C99's fma are both
//     correctly rounded, so they give the same bits; an FMA is one instruction where a
//     multiply and an add are two dependent ones.
//
// Accuracy (checked in tests/test_math.py against libm and, on the GPU, against
// CUDA's own functions): <= 2 ulp in double for |x| <= 2^20 (sin/cos), all positive
// normal x (log), |x| <= 700 (exp). Compiled with contraction disabled
// (-ffp-contract=off on the host, -fmad=false on the device) every other operation is
// a single IEEE-754 round-to-nearest step, so host and device agree bit for bit.
#pragma once
#include <stdint.h>
#include <string.h>

#if defined(__CUDACC__)
#define SBX_HD __host__ __device__ __forceinline__
#else
#define SBX_HD static inline
#endif
// The transcendentals themselves: inlined at every call site by default; a translation
// unit that defines SBX_SHARE_CALLS before including this header gets one out-of-line
// copy of each instead (a kernel with many call sites then runs the same instructions
// from every one of them and keeps them in the instruction cache)
#if defined(__CUDACC__) && defined(SBX_SHARE_CALLS)
#define SBX_HD_CALL static __host__ __device__ __noinline__
#else
#define SBX_HD_CALL SBX_HD
#endif

namespace sbxm {

// fused multiply-add, one rounding (CUDA's fma and C99 fma are both correctly rounded)
SBX_HD double fmad(double a, double b, double c) {
#ifdef __CUDA_ARCH__
    return __fma_rn(a, b, c);
#else
    return __builtin_fma(a, b, c);
#endif
}

// ---- split constants (gen_math_constants.py) ----
#define SBXM_PIO2_HI   0x1.921fb54400000p+0
#define SBXM_PIO2_MID  0x1.0b4611a600000p-34
#define SBXM_PIO2_LO   0x1.3198a2e037073p-69
#define SBXM_2_OVER_PI 0x1.45f306dc9c883p-1
#define SBXM_LN2_HI    0x1.62e42fee00000p-1
#define SBXM_LN2_LO    0x1.a39ef35793c76p-33
#define SBXM_INV_LN2   0x1.71547652b82fep+0
#define SBXM_SQRT2     0x1.6a09e667f3bcdp+0

// ---- minimax coefficients (gen_math_polys.py) ----
// SBXM_SIN: weighted minimax error 2^-58.0
#define SBXM_SIN0 -0x1.5555555555549p-3
#define SBXM_SIN1 0x1.111111110f87ap-7
#define SBXM_SIN2 -0x1.a01a019c1198fp-13
#define SBXM_SIN3 0x1.71de3577b6439p-19
#define SBXM_SIN4 -0x1.ae5e663a4e7efp-26
#define SBXM_SIN5 0x1.5d9300e9b8b15p-33
// SBXM_COS: weighted minimax error 2^-64.2
#define SBXM_COS0 0x1.555555555554cp-5
#define SBXM_COS1 -0x1.6c16c16c1517ep-10
#define SBXM_COS2 0x1.a01a019cb1bd6p-16
#define SBXM_COS3 -0x1.27e4f809f068ep-22
#define SBXM_COS4 0x1.1ee9ebe90849ap-29
#define SBXM_COS5 -0x1.8fae9c63fbf36p-37
// SBXM_LOG: weighted minimax error 2^-59.5
#define SBXM_LOG0 0x1.5555555555592p-2
#define SBXM_LOG1 0x1.999999997fd37p-3
#define SBXM_LOG2 0x1.24924941f8cffp-3
#define SBXM_LOG3 0x1.c71c5202b41b2p-4
#define SBXM_LOG4 0x1.7466405ba762dp-4
#define SBXM_LOG5 0x1.39a1933c05c0fp-4
#define SBXM_LOG6 0x1.2f070557504cdp-4
// SBXM_EXP: weighted minimax error 2^-59.3
#define SBXM_EXP0 0x1.0000000000000p-1
#define SBXM_EXP1 0x1.5555555555557p-3
#define SBXM_EXP2 0x1.5555555555558p-5
#define SBXM_EXP3 0x1.11111111100d8p-7
#define SBXM_EXP4 0x1.6c16c16c151f7p-10
#define SBXM_EXP5 0x1.a01a01abe9f2ap-13
#define SBXM_EXP6 0x1.a01a01acfce36p-16
#define SBXM_EXP7 0x1.71de022b7114ap-19
#define SBXM_EXP8 0x1.27e4ccc8e655ep-22
#define SBXM_EXP9 0x1.af4df62e8c93ep-26
#define SBXM_EXP10 0x1.1f8b54dcb8058p-29

SBX_HD uint64_t dbits(double x) { uint64_t u; memcpy(&u, &x, 8); return u; }
SBX_HD double bitsd(uint64_t u) { double x; memcpy(&x, &u, 8); return x; }

// nearest integer of a moderate-size double (ties away from zero)
SBX_HD int nearest_int(double x) {
    double t = (x >= 0.0) ? (x + 0.5) : (x - 0.5);
    return (int)t;
}

// sin and cos of a reduced argument |r| <= ~pi/4 (minimax in r^2, Horner)
SBX_HD double sin_poly(double r) {
    double r2 = r * r;
    double p = SBXM_SIN5;
    p = fmad(p, r2, SBXM_SIN4);
    p = fmad(p, r2, SBXM_SIN3);
    p = fmad(p, r2, SBXM_SIN2);
    p = fmad(p, r2, SBXM_SIN1);
    p = fmad(p, r2, SBXM_SIN0);                       // ~ -1/3!
    return fmad(r * r2, p, r);
}

SBX_HD double cos_poly(double r) {
    double r2 = r * r;
    double p = SBXM_COS5;
    p = fmad(p, r2, SBXM_COS4);
    p = fmad(p, r2, SBXM_COS3);
    p = fmad(p, r2, SBXM_COS2);
    p = fmad(p, r2, SBXM_COS1);
    p = fmad(p, r2, SBXM_COS0);                       // ~ 1/4!
    p = fmad(p, r2, -0.5);
    return fmad(r2, p, 1.0);
}

// x = k*(pi/2) + r, |r| <= pi/4 (+ tiny); returns r, writes the quadrant k & 3
SBX_HD double reduce_pio2(double x, int* quadrant) {
    int k = nearest_int(x * SBXM_2_OVER_PI);
    double kd = (double)k;
    double r = fmad(-kd, SBXM_PIO2_HI, x);
    r = fmad(-kd, SBXM_PIO2_MID, r);
    r = fmad(-kd, SBXM_PIO2_LO, r);
    *quadrant = k & 3;
    return r;
}

SBX_HD_CALL double sin(double x) {
    int q; double r = reduce_pio2(x, &q);
#ifdef __CUDA_ARCH__
    // both polynomials and a select: lanes in different quadrants do not diverge
    double sp = sin_poly(r), cp = cos_poly(r);
    double v = (q & 1) ? cp : sp;
    return (q & 2) ? -v : v;
#else
    switch (q) {
        case 0: return sin_poly(r);
        case 1: return cos_poly(r);
        case 2: return -sin_poly(r);
        default: return -cos_poly(r);
    }
#endif
}

SBX_HD_CALL double cos(double x) {
    int q; double r = reduce_pio2(x, &q);
#ifdef __CUDA_ARCH__
    double sp = sin_poly(r), cp = cos_poly(r);
    double v = (q & 1) ? sp : cp;
    return ((q + 1) & 2) ? -v : v;
#else
    switch (q) {
        case 0: return cos_poly(r);
        case 1: return -sin_poly(r);
        case 2: return -cos_poly(r);
        default: return sin_poly(r);
    }
#endif
}

// sin(x) and cos(x) together: one reduction and one evaluation of each polynomial, each
// result selected exactly as sin() and cos() above select it (the same bits)
SBX_HD_CALL void sincos(double x, double* sOut, double* cOut) {
    int q; double r = reduce_pio2(x, &q);
    double sp = sin_poly(r), cp = cos_poly(r);
    double vs = (q & 1) ? cp : sp;
    double vc = (q & 1) ? sp : cp;
    *sOut = (q & 2) ? -vs : vs;
    *cOut = ((q + 1) & 2) ? -vc : vc;
}

// natural log of a positive double (x <= 0 -> -inf / NaN like libm)
SBX_HD_CALL double log(double x) {
    if (!(x > 0.0)) return (x == 0.0) ? bitsd(0xfff0000000000000ULL) : bitsd(0x7ff8000000000000ULL);
    uint64_t u = dbits(x);
    int e = (int)((u >> 52) & 0x7ff);
    if (e == 0x7ff) return x;                          // +inf
    int adj = 0;
    if (e == 0) {                                      // subnormal: scale into the normal range
        x = x * 0x1p54; u = dbits(x); e = (int)((u >> 52) & 0x7ff); adj = -54;
    }
    e = e - 1023 + adj;
    double m = bitsd((u & 0x000fffffffffffffULL) | 0x3ff0000000000000ULL);   // [1,2)
    if (m > SBXM_SQRT2) { m = m * 0.5; e = e + 1; }
    double f = m - 1.0;
    double s = f / (2.0 + f);
    double s2 = s * s;
    double q = SBXM_LOG6;
    q = fmad(q, s2, SBXM_LOG5);
    q = fmad(q, s2, SBXM_LOG4);
    q = fmad(q, s2, SBXM_LOG3);
    q = fmad(q, s2, SBXM_LOG2);
    q = fmad(q, s2, SBXM_LOG1);
    q = fmad(q, s2, SBXM_LOG0);                       // ~ 1/3
    double two_s = 2.0 * s;
    double ed = (double)e;
    double lo = fmad(ed, SBXM_LN2_LO, two_s * (s2 * q));
    return ed * SBXM_LN2_HI + (two_s + lo);
}

// e^x
SBX_HD_CALL double exp(double x) {
    if (x != x) return x;
    if (x > 709.782712893384) return bitsd(0x7ff0000000000000ULL);
    if (x < -745.1332191019412) return 0.0;
    int k = nearest_int(x * SBXM_INV_LN2);
    double kd = (double)k;
    double r = fmad(-kd, SBXM_LN2_HI, x);
    r = fmad(-kd, SBXM_LN2_LO, r);
    double p = SBXM_EXP10;
    p = fmad(p, r, SBXM_EXP9);
    p = fmad(p, r, SBXM_EXP8);
    p = fmad(p, r, SBXM_EXP7);
    p = fmad(p, r, SBXM_EXP6);
    p = fmad(p, r, SBXM_EXP5);
    p = fmad(p, r, SBXM_EXP4);
    p = fmad(p, r, SBXM_EXP3);
    p = fmad(p, r, SBXM_EXP2);
    p = fmad(p, r, SBXM_EXP1);
    p = fmad(p, r, SBXM_EXP0);                        // ~ 1/2
    double er = 1.0 + fmad(r, r * p, r);
    // scale by 2^k in two halves so that k down to -1074 stays representable
    int k1 = k / 2, k2 = k - k1;
    double s1 = bitsd((uint64_t)(k1 + 1023) << 52);
    double s2 = bitsd((uint64_t)(k2 + 1023) << 52);
    return (er * s1) * s2;
}

// ---- integer hashing and counter-based generators ----

// 32-bit Wang hash (unsigned arithmetic == Java int wraparound with >>>)
SBX_HD uint32_t wang_hash(uint32_t s) {
    s = (s ^ 61u) ^ (s >> 16);
    s = s * 9u;
    s = s ^ (s >> 4);
    s = s * 0x27d4eb2du;
    s = s ^ (s >> 15);
    return s;
}

// per-(slot, step, seed) base key: (i*1000003) ^ (step*999983) ^ (seed*7919), int32 wrap
SBX_HD uint32_t rng_base(int32_t i, int32_t step, int32_t seed) {
    return ((uint32_t)i * 1000003u) ^ ((uint32_t)step * 999983u) ^ ((uint32_t)seed * 7919u);
}

// (h >>> 1) / 2147483647.0f : the float literal 2147483647.0f is exactly 2^31
SBX_HD float unit_from_hash(uint32_t h) {
    return (float)(int32_t)(h >> 1) / 2147483648.0f;
}

// Philox4x32-10 (Salmon, Moraes, Dror, Shaw, "Parallel random numbers: as easy as
// 1, 2, 3", SC'11): counter c[4], key k[2], 10 rounds.
SBX_HD void philox4x32_10(uint32_t c[4], uint32_t k0, uint32_t k1) {
    const uint32_t M0 = 0xD2511F53u, M1 = 0xCD9E8D57u;
    const uint32_t W0 = 0x9E3779B9u, W1 = 0xBB67AE85u;
    for (int r = 0; r < 10; r++) {
        uint64_t p0 = (uint64_t)M0 * c[0];
        uint64_t p1 = (uint64_t)M1 * c[2];
        uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
        uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
        uint32_t n0 = hi1 ^ c[1] ^ k0;
        uint32_t n1 = lo1;
        uint32_t n2 = hi0 ^ c[3] ^ k1;
        uint32_t n3 = lo0;
        c[0] = n0; c[1] = n1; c[2] = n2; c[3] = n3;
        k0 += W0; k1 += W1;
    }
}

}  // namespace sbxm

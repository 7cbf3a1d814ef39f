// noise.h — counter-based Gaussian inlet noise, bit-identical on host and device.
//
// The reference has no inlet noise (its oil inlet speed is the constant
// physics::u_oil, src/BoundaryConditions.cuh:127).  The jet configurations
// need u_in = u_oil (1 + a N(0,1)) per inlet cell and step, and the CPU
// oracle must see the same numbers, so this header is shared by both sides:
//
//   * Philox-4x32-10, the counter-based generator of Salmon, Moraes, Dror and
//     Shaw, "Parallel random numbers: as easy as 1, 2, 3" (SC'11): 10 rounds
//     of two 32x32->64 multiplies with the published multipliers and Weyl
//     key increments.
//   * Box-Muller, z = sqrt(-2 ln u1) cos(2 pi u2), evaluated in FP64 with this
//     file's own log and cos (range reduction + Taylor / atanh series written
//     from the series definitions), and every operation an explicit
//     round-to-nearest add/mul/div so no FMA contraction can change a bit
//     between nvcc and gcc.  sqrt is IEEE correctly rounded on both.
//
// Counter layout: (cell, step_lo, step_hi, stream), key = (seed_lo, seed_hi).
#pragma once

#include <stdint.h>

#if defined(__CUDACC__)
#define SSMD_HD __host__ __device__ __forceinline__
#else
#define SSMD_HD static inline
#endif

namespace ssmd_noise {

SSMD_HD uint32_t mulhi32(uint32_t a, uint32_t b) {
    return (uint32_t)(((uint64_t)a * (uint64_t)b) >> 32);
}

struct U4 {
    uint32_t v[4];
};

SSMD_HD U4 philox4x32_10(U4 c, uint32_t k0, uint32_t k1) {
    const uint32_t M0 = 0xD2511F53u, M1 = 0xCD9E8D57u;
    const uint32_t W0 = 0x9E3779B9u, W1 = 0xBB67AE85u;
    for (int r = 0; r < 10; ++r) {
        const uint32_t hi0 = mulhi32(M0, c.v[0]), lo0 = M0 * c.v[0];
        const uint32_t hi1 = mulhi32(M1, c.v[2]), lo1 = M1 * c.v[2];
        U4 n;
        n.v[0] = hi1 ^ c.v[1] ^ k0;
        n.v[1] = lo1;
        n.v[2] = hi0 ^ c.v[3] ^ k1;
        n.v[3] = lo0;
        c = n;
        k0 += W0;
        k1 += W1;
    }
    return c;
}

// Exact-rounding primitives (no contraction on either compiler).
#if defined(__CUDA_ARCH__)
SSMD_HD double dadd(double a, double b) { return __dadd_rn(a, b); }
SSMD_HD double dmul(double a, double b) { return __dmul_rn(a, b); }
SSMD_HD double ddiv(double a, double b) { return __ddiv_rn(a, b); }
SSMD_HD double dsqrt(double a) { return __dsqrt_rn(a); }
SSMD_HD int64_t dbits(double a) { return __double_as_longlong(a); }
SSMD_HD double dfrombits(int64_t b) { return __longlong_as_double(b); }
#else
SSMD_HD double dadd(double a, double b) {
    volatile double r = a + b;
    return r;
}
SSMD_HD double dmul(double a, double b) {
    volatile double r = a * b;
    return r;
}
SSMD_HD double ddiv(double a, double b) {
    volatile double r = a / b;
    return r;
}
SSMD_HD double dsqrt(double a) { return __builtin_sqrt(a); }
SSMD_HD int64_t dbits(double a) {
    int64_t b;
    __builtin_memcpy(&b, &a, 8);
    return b;
}
SSMD_HD double dfrombits(int64_t b) {
    double a;
    __builtin_memcpy(&a, &b, 8);
    return a;
}
#endif

// Natural log for normal positive x: x = m 2^e, m in [sqrt(1/2), sqrt(2)),
// ln m = 2 atanh(s), s = (m - 1)/(m + 1), |s| < 0.172, series to s^25.
SSMD_HD double ln(double x) {
    int64_t b = dbits(x);
    int e = (int)((b >> 52) & 0x7ff) - 1023;
    b = (b & 0x000fffffffffffffLL) | 0x3ff0000000000000LL; // m in [1, 2)
    double m = dfrombits(b);
    if (m > 1.4142135623730951) {
        m = dmul(m, 0.5);
        e += 1;
    }
    const double s = ddiv(dadd(m, -1.0), dadd(m, 1.0));
    const double s2 = dmul(s, s);
    double sum = 0.0;
    for (int k = 25; k >= 1; k -= 2) sum = dadd(dmul(sum, s2), ddiv(1.0, (double)k));
    const double lnm = dmul(2.0, dmul(s, sum));
    return dadd(dmul((double)e, 0.69314718055994530942), lnm);
}

// cos(2 pi t) for t in [0, 1): quarter-turn reduction, then Taylor series of
// sin / cos on |a| <= pi/4 (terms to a^22).
SSMD_HD double cos_turns(double t) {
    const double q = dmul(t, 4.0);           // exact
    const double k = (double)(int64_t)(dadd(q, 0.5)); // nearest quarter, q >= 0
    const double r = dadd(t, dmul(k, -0.25)); // exact, |r| <= 1/8
    const double a = dmul(r, 6.28318530717958647692);
    const double a2 = dmul(a, a);
    // cos a = sum (-1)^n a^(2n) / (2n)!, sin a = a sum (-1)^n a^(2n) / (2n+1)!
    double rc[12], rs[12]; // signed reciprocal factorials
    double fact = 1.0;     // (2n)!
    for (int n = 0; n < 12; ++n) {
        if (n > 0) fact = dmul(fact, dmul((double)(2 * n - 1), (double)(2 * n)));
        const double sign = (n & 1) ? -1.0 : 1.0;
        rc[n] = ddiv(sign, fact);
        rs[n] = ddiv(sign, dmul(fact, (double)(2 * n + 1)));
    }
    double c = 0.0, s = 0.0;
    for (int n = 11; n >= 0; --n) {
        c = dadd(dmul(c, a2), rc[n]);
        s = dadd(dmul(s, a2), rs[n]);
    }
    s = dmul(s, a);
    switch (((int64_t)k) & 3) {
    case 0: return c;
    case 1: return -s;
    case 2: return -c;
    default: return s;
    }
}

// Standard normal deviate for (seed, step, cell, stream).
SSMD_HD double gaussian(uint64_t seed, uint64_t step, uint32_t cell, uint32_t stream) {
    U4 c;
    c.v[0] = cell;
    c.v[1] = (uint32_t)step;
    c.v[2] = (uint32_t)(step >> 32);
    c.v[3] = stream;
    const U4 r = philox4x32_10(c, (uint32_t)seed, (uint32_t)(seed >> 32));
    const double inv32 = 2.3283064365386963e-10; // 2^-32
    const double u1 = dmul(dadd((double)r.v[0], 0.5), inv32); // (0, 1)
    const double u2 = dmul((double)r.v[1], inv32);            // [0, 1)
    const double rad = dsqrt(dmul(-2.0, ln(u1)));
    return dmul(rad, cos_turns(u2));
}

} // namespace ssmd_noise

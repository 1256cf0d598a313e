/*
 * hp_math.h -- single-precision elementary functions written for this
 * library, identical on the host and on the GPU.
 *
 * The MCC kernels need exp, log10, pow, sin/cos, tan and atan
 * (src/cuda_mcc.cu:139-201, src/cuda_mccAr.cu:57-58,110,707-776).  The CPU
 * checker must make the same integer decisions (collision channel, created
 * particle counts) as the GPU, so both sides evaluate these functions with
 * the very same sequence of IEEE-754 single-precision additions,
 * multiplications, divisions and square roots (all correctly rounded on both
 * sides; the GPU build uses --fmad=false and the host build
 * -ffp-contract=off so that no operation is fused).
 *
 * Methods (all from the mathematics, coefficients are exact reciprocals of
 * integers or constants of analysis):
 *   exp   Cody & Waite (1980) additive reduction x = n ln2 + r with a
 *         two-part ln2, Taylor series of e^r to degree 8, scaling by 2^n
 *         through the exponent field.
 *   log   x = m 2^e with m in [sqrt(1/2), sqrt(2)), ln m = 2 atanh(s),
 *         s = (m-1)/(m+1), odd series to s^13.
 *   sin/cos  of 2*pi*t ("turns"): reduction to the nearest quarter turn is
 *         exact (Sterbenz), then Taylor series on [-pi/4, pi/4].
 *   tan   sin/cos on [0, pi/4], cot of the complement with a two-part pi/2
 *         above it.
 *   atan  reflection for |x| > 1, the pi/6 addition formula for
 *         |x| > 2 - sqrt(3), then the odd Taylor series to x^17.
 * Accuracy (checked by tests/test_math.py against double-precision libm):
 * a few units in the last place over the ranges the kernels use.
 */
#ifndef HP_MATH_H
#define HP_MATH_H

#include <stdint.h>
#include <string.h>

#if defined(__CUDACC__)
#define HP_MHD __host__ __device__ __forceinline__
#else
#define HP_MHD static inline
#endif

#define HP_PI_F 3.14159265358979323846f
#define HP_TWO_PI_F 6.28318530717958647692f

HP_MHD uint32_t hp_f2u(float f) {
#if defined(__CUDA_ARCH__)
    return __float_as_uint(f);
#else
    uint32_t u; memcpy(&u, &f, 4); return u;
#endif
}
HP_MHD float hp_u2f(uint32_t u) {
#if defined(__CUDA_ARCH__)
    return __uint_as_float(u);
#else
    float f; memcpy(&f, &u, 4); return f;
#endif
}

/* round-to-nearest integer of a float in int range, ties away from zero */
HP_MHD int hp_nint(float x) { return (int)(x >= 0.0f ? x + 0.5f : x - 0.5f); }

HP_MHD float hp_expf(float x) {
    if (x != x) return x;
    if (x > 88.72f) return hp_u2f(0x7f800000u);
    if (x < -103.9f) return 0.0f;
    const float log2e = 1.44269504088896340736f;
    const float ln2_hi = 0.693145751953125f;       /* 2^-1 .. 13 bits of ln 2, exact */
    const float ln2_lo = 1.42860682030941723212e-6f; /* ln 2 - ln2_hi */
    int n = hp_nint(x * log2e);
    float fn = (float)n;
    float r = (x - fn * ln2_hi) - fn * ln2_lo;
    /* e^r, |r| <= 0.347: Taylor to r^8 (next term < 2e-10) */
    float p = 1.0f / 40320.0f;
    p = p * r + 1.0f / 5040.0f;
    p = p * r + 1.0f / 720.0f;
    p = p * r + 1.0f / 120.0f;
    p = p * r + 1.0f / 24.0f;
    p = p * r + 1.0f / 6.0f;
    p = p * r + 0.5f;
    p = p * r + 1.0f;
    p = p * r + 1.0f;
    /* scale by 2^n in two steps so that subnormal results stay exact-ish */
    int n1 = n / 2, n2 = n - n / 2;
    float s1 = hp_u2f((uint32_t)(n1 + 127) << 23);
    float s2 = hp_u2f((uint32_t)(n2 + 127) << 23);
    return p * s1 * s2;
}

HP_MHD float hp_logf(float x) {
    if (x != x) return x;
    if (x < 0.0f) return hp_u2f(0x7fc00000u);
    if (x == 0.0f) return hp_u2f(0xff800000u);
    uint32_t u = hp_f2u(x);
    if (u >= 0x7f800000u) return x; /* +inf */
    int e = 0;
    if (u < 0x00800000u) { /* subnormal: scale up by 2^25 */
        x = x * 33554432.0f;
        u = hp_f2u(x);
        e = -25;
    }
    e += (int)(u >> 23) - 127;
    float m = hp_u2f((u & 0x007fffffu) | 0x3f800000u); /* [1, 2) */
    if (m > 1.41421356237309504880f) { m = m * 0.5f; e += 1; }
    float s = (m - 1.0f) / (m + 1.0f);
    float s2 = s * s;
    float p = 2.0f / 13.0f;
    p = p * s2 + 2.0f / 11.0f;
    p = p * s2 + 2.0f / 9.0f;
    p = p * s2 + 2.0f / 7.0f;
    p = p * s2 + 2.0f / 5.0f;
    p = p * s2 + 2.0f / 3.0f;
    p = p * s2 + 2.0f;
    float lnm = p * s;
    const float ln2_hi = 0.693145751953125f;
    const float ln2_lo = 1.42860682030941723212e-6f;
    float fe = (float)e;
    return (fe * ln2_hi + lnm) + fe * ln2_lo;
}

HP_MHD float hp_log10f(float x) { return hp_logf(x) * 0.434294481903251827651f; }

/* b^e for b > 0 */
HP_MHD float hp_powf(float b, float e) {
    if (b == 1.0f || e == 0.0f) return 1.0f;
    return hp_expf(e * hp_logf(b));
}

/* sin and cos of a in [-pi/4, pi/4] */
HP_MHD void hp_sincos_small(float a, float *s, float *c) {
    float a2 = a * a;
    float ps = -1.0f / 39916800.0f;
    ps = ps * a2 + 1.0f / 362880.0f;
    ps = ps * a2 - 1.0f / 5040.0f;
    ps = ps * a2 + 1.0f / 120.0f;
    ps = ps * a2 - 1.0f / 6.0f;
    ps = ps * a2;
    *s = a + a * ps;
    float pc = 1.0f / 479001600.0f;
    pc = pc * a2 - 1.0f / 3628800.0f;
    pc = pc * a2 + 1.0f / 40320.0f;
    pc = pc * a2 - 1.0f / 720.0f;
    pc = pc * a2 + 1.0f / 24.0f;
    pc = pc * a2 - 0.5f;
    *c = 1.0f + a2 * pc;
}

/* sin(2 pi t) and cos(2 pi t) for |t| <= 2^20 */
HP_MHD void hp_sincos_turns(float t, float *s, float *c) {
    int q = hp_nint(t * 4.0f);
    float f = t - (float)q * 0.25f; /* exact, |f| <= 1/8 */
    float a = f * HP_TWO_PI_F;
    float ss, cc;
    hp_sincos_small(a, &ss, &cc);
    switch (q & 3) {
    case 0: *s = ss; *c = cc; break;
    case 1: *s = cc; *c = -ss; break;
    case 2: *s = -ss; *c = -cc; break;
    default: *s = -cc; *c = ss; break;
    }
}

/* tan(y) for y in [0, pi/2) */
HP_MHD float hp_tanf_q1(float y) {
    float s, c;
    if (y <= 0.785398163397448309616f) {
        hp_sincos_small(y, &s, &c);
        return s / c;
    }
    const float pio2_hi = 1.57079601287841796875f;  /* exact in float */
    const float pio2_lo = 3.13916473785604476e-7f;   /* pi/2 - pio2_hi */
    float z = (pio2_hi - y) + pio2_lo;
    hp_sincos_small(z, &s, &c);
    return c / s;
}

HP_MHD float hp_atanf(float x) {
    if (x != x) return x;
    float sgn = 1.0f;
    if (x < 0.0f) { sgn = -1.0f; x = -x; }
    const float pio2 = 1.57079632679489661923f;
    const float pio6 = 0.523598775598298873077f;
    const float sqrt3 = 1.73205080756887729353f;
    const float tan_pi12 = 0.267949192431122706473f;
    int inv = 0, shift = 0;
    if (x > 1.0f) { x = 1.0f / x; inv = 1; }
    if (x > tan_pi12) { x = (x * sqrt3 - 1.0f) / (sqrt3 + x); shift = 1; }
    float x2 = x * x;
    float p = 1.0f / 17.0f;
    p = p * x2 - 1.0f / 15.0f;
    p = p * x2 + 1.0f / 13.0f;
    p = p * x2 - 1.0f / 11.0f;
    p = p * x2 + 1.0f / 9.0f;
    p = p * x2 - 1.0f / 7.0f;
    p = p * x2 + 1.0f / 5.0f;
    p = p * x2 - 1.0f / 3.0f;
    float r = x + x * (x2 * p);
    if (shift) r = pio6 + r;
    if (inv) r = pio2 - r;
    return sgn * r;
}

#endif /* HP_MATH_H */

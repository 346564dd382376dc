/*
 * phiray_math.h — the transcendental functions the phiray-b200 kernels use,
 * written out in plain IEEE-754 single precision so that host code and
 * device code built from this header return the same bits for the same
 * argument.
 *
 * Why not libm / CUDA's sinf: the reference shades in WGSL, whose sin, cos,
 * pow, exp and log2 are whatever the platform driver provides (no precision
 * is pinned), and a CPU restatement calling glibc next to a kernel calling
 * CUDA's library would differ in the last bits and then, rarely, in a
 * sampling decision. Both sides include this header instead, so a CPU twin
 * of a kernel reproduces its image bit for bit.
 *
 * Methods (all published textbook ones, coefficients are 1/n! or 1/(2k+1)):
 *   - exp2: round-to-nearest split x = k + f, |f| <= 1/2; 2^f = e^(f ln 2)
 *     by its Taylor series to degree 7 (Horner); scale by 2^k built from
 *     the exponent bits.
 *   - log2: x = m 2^e with m in [sqrt(1/2), sqrt(2)); log(m) = 2 atanh(s),
 *     s = (m-1)/(m+1), by the odd series s + s^3/3 + ... + s^13/13.
 *   - sin/cos: Cody-Waite reduction by pi/2 in three parts, then the
 *     Taylor series on [-pi/4, pi/4] and a quadrant swap.
 *   - pow(x, y) = exp2(y log2 x) for x > 0; exp(x) = exp2(x log2 e).
 * Accuracy against float64, measured over 400,000 arguments a function
 * (tests/test_math_accuracy.py holds these bounds): exp2 <= 1.5 ulp on
 * [-126, 127]; log2 <= 3.5 ulp on [1e-30, 1e30]; sin and cos <= 1.5 x 2^-24
 * absolute on [-100, 100]; pow(x, y) <= 8 + 1.5 |y log2 x| ulp and exp(x)
 * <= 3 + 1.5 |x log2 e| ulp (the product's rounding is carried into the
 * exponent: ~10 ulp for the sRGB curve's pow(x, 1/2.4), more for large
 * results). More than a path tracer needs; the point is sameness, not the
 * last ulp: the device build returns the host build's bits.
 *
 * Build rule: every file that includes this must be compiled without
 * floating-point contraction (nvcc --fmad=false, gcc -ffp-contract=off),
 * or the two sides fuse different multiply-adds.
 */
#ifndef PHIRAY_MATH_H
#define PHIRAY_MATH_H

#include <stdint.h>
#include <string.h>
#include <math.h>

#if defined(__CUDACC__)
#define PM_HD __host__ __device__ __forceinline__
#else
#define PM_HD static inline
#endif

PM_HD uint32_t pm_bits(float f) {
#if defined(__CUDA_ARCH__)
    return __float_as_uint(f);
#else
    uint32_t u;
    memcpy(&u, &f, 4);
    return u;
#endif
}

PM_HD float pm_float(uint32_t u) {
#if defined(__CUDA_ARCH__)
    return __uint_as_float(u);
#else
    float f;
    memcpy(&f, &u, 4);
    return f;
#endif
}

/* 2^k for k in [-126, 127], exactly. */
PM_HD float pm_pow2i(int k) { return pm_float((uint32_t)(k + 127) << 23); }

PM_HD float pm_rint(float x) {
#if defined(__CUDA_ARCH__)
    return rintf(x);
#else
    return nearbyintf(x);
#endif
}

PM_HD float pm_exp2(float x) {
    if (x != x) return x;
    if (x >= 128.0f) return pm_float(0x7f800000u);
    if (x < -150.0f) return 0.0f;
    float k = pm_rint(x);
    float f = x - k;
    float t = f * 0.693147182f;
    float p = 1.98412701e-4f;
    p = p * t + 1.38888892e-3f;
    p = p * t + 8.33333377e-3f;
    p = p * t + 4.16666679e-2f;
    p = p * t + 1.66666672e-1f;
    p = p * t + 0.5f;
    p = p * t + 1.0f;
    p = p * t + 1.0f;
    int ki = (int)k;
    int k1 = ki / 2;
    int k2 = ki - k1;
    return p * pm_pow2i(k1) * pm_pow2i(k2);
}

PM_HD float pm_log2(float x) {
    if (x != x || x < 0.0f) return pm_float(0x7fc00000u);
    if (x == 0.0f) return pm_float(0xff800000u);
    uint32_t b = pm_bits(x);
    if (b == 0x7f800000u) return x;
    int e = 0;
    if (b < 0x00800000u) {
        x = x * 8388608.0f;
        b = pm_bits(x);
        e = -23;
    }
    e += (int)(b >> 23) - 127;
    float m = pm_float((b & 0x007fffffu) | 0x3f800000u);
    if (m > 1.41421354f) {
        m = m * 0.5f;
        e += 1;
    }
    float s = (m - 1.0f) / (m + 1.0f);
    float s2 = s * s;
    float p = 7.69230798e-2f;
    p = p * s2 + 9.09090936e-2f;
    p = p * s2 + 1.11111112e-1f;
    p = p * s2 + 1.42857149e-1f;
    p = p * s2 + 2.00000003e-1f;
    p = p * s2 + 3.33333343e-1f;
    p = p * s2 + 1.0f;
    float l = (2.0f * s * p) * 1.44269502f;
    return (float)e + l;
}

/* WGSL pow for the arguments the kernels give it (x >= 0). */
PM_HD float pm_pow(float x, float y) {
    if (y == 0.0f) return 1.0f;
    if (y == 1.0f) return x;
    if (x != x || y != y || x < 0.0f) return pm_float(0x7fc00000u);
    if (x == 0.0f) return y > 0.0f ? 0.0f : pm_float(0x7f800000u);
    return pm_exp2(y * pm_log2(x));
}

PM_HD float pm_exp(float x) { return pm_exp2(x * 1.44269502f); }

PM_HD void pm_sincos(float x, float* sn_out, float* cs_out) {
    float k = pm_rint(x * 0.636619747f);
    float r = x - k * 1.5703125f;
    r = r - k * 4.83751297e-4f;
    r = r - k * 7.54979013e-8f;
    int q = ((int)k) & 3;
    float r2 = r * r;
    float sp = -2.50521084e-8f;
    sp = sp * r2 + 2.75573192e-6f;
    sp = sp * r2 - 1.98412698e-4f;
    sp = sp * r2 + 8.33333377e-3f;
    sp = sp * r2 - 1.66666672e-1f;
    float sn = r + (r * r2) * sp;
    float cp = -2.75573192e-7f;
    cp = cp * r2 + 2.48015876e-5f;
    cp = cp * r2 - 1.38888892e-3f;
    cp = cp * r2 + 4.16666679e-2f;
    cp = cp * r2 - 0.5f;
    float cn = 1.0f + r2 * cp;
    float s, c;
    if (q == 0) {
        s = sn;
        c = cn;
    } else if (q == 1) {
        s = cn;
        c = -sn;
    } else if (q == 2) {
        s = -sn;
        c = -cn;
    } else {
        s = -cn;
        c = sn;
    }
    *sn_out = s;
    *cs_out = c;
}

PM_HD float pm_sin(float x) {
    float s, c;
    pm_sincos(x, &s, &c);
    return s;
}

PM_HD float pm_cos(float x) {
    float s, c;
    pm_sincos(x, &s, &c);
    return c;
}

#endif /* PHIRAY_MATH_H */

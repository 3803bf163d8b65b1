/*
 * rr_detmath.h — deterministic single-precision elementary functions.
 *
 * The reference shaders call sin/cos/exp/log through Slang, which lowers them
 * to SPIR-V GLSL.std.450 Sin/Cos/Exp/Log. Their precision is left to the
 * Vulkan driver (the spec allows an absolute error of 2^-11 for sin/cos), so
 * the reference defines no single correct answer for them. This header fixes
 * one: every sin, cos, exp and log on the light-transport path, on the GPU and
 * in the CPU checker alike, is the function below, evaluated with the same
 * IEEE-754 binary32 operations in the same order. Together with
 * `-fmad=false` (nvcc) / `-ffp-contract=off` (gcc), IEEE division and square
 * root, this makes the CUDA kernels and the CPU restatement produce
 * bit-identical results from the same seeds.
 *
 * Methods (all standard, no vendor code):
 *   sin/cos : Cody–Waite reduction by pi/2 split into three binary32 parts,
 *             then the Taylor series of sin (to x^9) and cos (to x^12) on
 *             [-pi/4, pi/4], evaluated by Horner's rule with fused multiply-add.
 *   exp     : x = k ln2 + r with a two-part ln2, Taylor series of e^r to r^8
 *             on |r| <= ln2/2, scaled by 2^k built from the exponent bits.
 *             Results below 2^-126 are returned as 0.
 *   log     : x = m 2^e with m in [sqrt(1/2), sqrt(2)), log m = 2 atanh(s),
 *             s = (m-1)/(m+1), odd series to s^11.
 * Measured accuracy against a binary64 libm is asserted by the CPU test suite
 * (<= 2 ulp for sin/cos on [0, 8 pi], exp on [-87, 88], log on (0, inf)).
 *
 * Header-only, C99/C++ and CUDA. Define nothing before including it.
 */
#ifndef RR_DETMATH_H
#define RR_DETMATH_H

#include <stdint.h>
#include <string.h>
#include <math.h>

#if defined(__CUDACC__)
#define RR_DM_FN static __host__ __device__ __forceinline__
#else
#define RR_DM_FN static inline
#endif

RR_DM_FN float rr_dm_fma(float a, float b, float c)
{
#if defined(__CUDA_ARCH__)
    return __fmaf_rn(a, b, c);
#else
    return fmaf(a, b, c);
#endif
}

RR_DM_FN uint32_t rr_dm_f2u(float f)
{
#if defined(__CUDA_ARCH__)
    return __float_as_uint(f);
#else
    uint32_t u; memcpy(&u, &f, 4); return u;
#endif
}

RR_DM_FN float rr_dm_u2f(uint32_t u)
{
#if defined(__CUDA_ARCH__)
    return __uint_as_float(u);
#else
    float f; memcpy(&f, &u, 4); return f;
#endif
}

/* round to nearest integer, ties to even (default rounding mode on both sides) */
RR_DM_FN float rr_dm_rint(float x)
{
#if defined(__CUDA_ARCH__)
    return rintf(x);
#else
    return rintf(x);
#endif
}

/* sin(r), cos(r) for |r| <= pi/4 (+ rounding slack) */
RR_DM_FN float rr_dm_sin_poly(float r)
{
    const float r2 = r * r;
    float p = 0x1.71de3ap-19f;              /*  1/9! */
    p = rr_dm_fma(p, r2, -0x1.a01a02p-13f); /* -1/7! */
    p = rr_dm_fma(p, r2, 0x1.111112p-7f);   /*  1/5! */
    p = rr_dm_fma(p, r2, -0x1.555556p-3f);  /* -1/3! */
    p = p * r2;
    return rr_dm_fma(p, r, r);
}

RR_DM_FN float rr_dm_cos_poly(float r)
{
    const float r2 = r * r;
    float p = 0x1.1eed8ep-29f;              /*  1/12! */
    p = rr_dm_fma(p, r2, -0x1.27e4fcp-22f); /* -1/10! */
    p = rr_dm_fma(p, r2, 0x1.a01a02p-16f);  /*  1/8!  */
    p = rr_dm_fma(p, r2, -0x1.6c16c2p-10f); /* -1/6!  */
    p = rr_dm_fma(p, r2, 0x1.555556p-5f);   /*  1/4!  */
    p = rr_dm_fma(p, r2, -0.5f);            /* -1/2!  */
    return rr_dm_fma(p, r2, 1.0f);
}

/* Cody–Waite reduction: x = k*(pi/2) + r. Accurate for |x| < 2^15. */
RR_DM_FN float rr_dm_reduce_pio2(float x, int* quadrant)
{
    const float k = rr_dm_rint(x * 0x1.45f306p-1f); /* x * 2/pi */
    float r = rr_dm_fma(-k, 0x1.921fb6p+0f, x);
    r = rr_dm_fma(-k, -0x1.777a5cp-25f, r);
    r = rr_dm_fma(-k, -0x1.ee59dap-50f, r);
    *quadrant = ((int)k) & 3;
    return r;
}

RR_DM_FN float rr_sinf(float x)
{
    int q;
    const float r = rr_dm_reduce_pio2(x, &q);
    switch (q) {
    case 0:  return rr_dm_sin_poly(r);
    case 1:  return rr_dm_cos_poly(r);
    case 2:  return -rr_dm_sin_poly(r);
    default: return -rr_dm_cos_poly(r);
    }
}

RR_DM_FN float rr_cosf(float x)
{
    int q;
    const float r = rr_dm_reduce_pio2(x, &q);
    switch (q) {
    case 0:  return rr_dm_cos_poly(r);
    case 1:  return -rr_dm_sin_poly(r);
    case 2:  return -rr_dm_cos_poly(r);
    default: return rr_dm_sin_poly(r);
    }
}

RR_DM_FN float rr_expf(float x)
{
    if (x != x) return x;                      /* NaN */
    if (x > 88.72283f) return rr_dm_u2f(0x7f800000u); /* +inf */
    if (x < -87.33654f) return 0.0f;           /* below 2^-126: flushed */
    const float k = rr_dm_rint(x * 0x1.715476p+0f); /* x * log2(e) */
    float r = rr_dm_fma(-k, 0x1.62e430p-1f, x);
    r = rr_dm_fma(-k, -0x1.05c610p-29f, r);
    float p = 0x1.a01a02p-16f;                 /* 1/8! */
    p = rr_dm_fma(p, r, 0x1.a01a02p-13f);      /* 1/7! */
    p = rr_dm_fma(p, r, 0x1.6c16c2p-10f);      /* 1/6! */
    p = rr_dm_fma(p, r, 0x1.111112p-7f);       /* 1/5! */
    p = rr_dm_fma(p, r, 0x1.555556p-5f);       /* 1/4! */
    p = rr_dm_fma(p, r, 0x1.555556p-3f);       /* 1/3! */
    p = rr_dm_fma(p, r, 0.5f);                 /* 1/2! */
    p = rr_dm_fma(p, r, 1.0f);
    p = rr_dm_fma(p, r, 1.0f);
    int ki = (int)k;
    if (ki > 127) { p = p * 2.0f; ki -= 1; }
    if (ki < -126) { p = p * 0.5f; ki += 1; }
    return p * rr_dm_u2f((uint32_t)(ki + 127) << 23);
}

RR_DM_FN float rr_logf(float x)
{
    if (x != x) return x;                              /* NaN */
    if (x < 0.0f) return rr_dm_u2f(0x7fc00000u);       /* NaN */
    if (x == 0.0f) return rr_dm_u2f(0xff800000u);      /* -inf */
    if (x == rr_dm_u2f(0x7f800000u)) return x;         /* +inf */
    int e_adj = 0;
    if (x < 0x1.0p-126f) { x = x * 0x1.0p+23f; e_adj = -23; }
    const uint32_t bits = rr_dm_f2u(x);
    int e = (int)((bits >> 23) & 0xffu) - 127 + e_adj;
    float m = rr_dm_u2f((bits & 0x007fffffu) | 0x3f800000u);
    if (m > 0x1.6a09e6p+0f) { m = m * 0.5f; e += 1; }  /* sqrt(2) */
    const float s = (m - 1.0f) / (m + 1.0f);
    const float s2 = s * s;
    float p = 0x1.745d18p-4f;                 /* 1/11 */
    p = rr_dm_fma(p, s2, 0x1.c71c72p-4f);     /* 1/9  */
    p = rr_dm_fma(p, s2, 0x1.24924ap-3f);     /* 1/7  */
    p = rr_dm_fma(p, s2, 0x1.99999ap-3f);     /* 1/5  */
    p = rr_dm_fma(p, s2, 0x1.555556p-2f);     /* 1/3  */
    p = p * s2;
    const float two_s = s + s;
    const float logm = rr_dm_fma(two_s, p, two_s);
    const float fe = (float)e;
    return rr_dm_fma(fe, 0x1.62e430p-1f, rr_dm_fma(fe, -0x1.05c610p-29f, logm));
}

#undef RR_DM_FN
#endif /* RR_DETMATH_H */

/*
 * st_pow.h -- x^0.687 for the Schiller-Naumann drag correction, written for this project.
 *
 * The drag correction 1 + 0.15 Re^0.687 decides how far a parcel moves, and therefore
 * which cell it ends up in.  Cell indices must agree bit for bit between the CUDA kernels
 * and the CPU oracle, so the power function cannot come from two different math libraries
 * (CUDA's pow and glibc's pow differ in the last ulp for some arguments).  This header is
 * compiled unchanged by nvcc (device) and gcc (host) and uses only IEEE-754 +, -, *, / and
 * explicit fma (correctly rounded on both), integer bit manipulation and comparisons.  Both
 * sides must be built without implicit contraction of a*b+c into fma: nvcc --fmad=false,
 * gcc -ffp-contract=off.
 *
 * Method (textbook, no library constants):
 *   pow(x, a) = exp(a ln x)
 *   ln x : x = 2^e m with m in [sqrt(1/2), sqrt(2));  ln m = 2 atanh(s), s = (m-1)/(m+1),
 *          atanh s = s (1 + z/3 + z^2/5 + ...), z = s^2 <= 0.0295  (series truncated after z^11,
 *          remainder < 1e-18 relative).  See Abramowitz & Stegun 4.1.28 (ln((1+s)/(1-s))).
 *   exp y: Cody & Waite (1980) reduction y = k ln2 + r, |r| <= ln2/2, e^r by its Taylor series
 *          to r^14/14! (remainder < 5e-18), result scaled by 2^k through the exponent field.
 * Accuracy: a few ulp in double (st_pow0687) and 2 ulp in single (st_pow0687f, a separate
 * polynomial method described at its definition), far below what the drag model needs; the
 * point is that host and device produce the same bits.
 * Checked against libm pow by the CPU tests and host vs device bit-equality by the GPU
 * tests.
 */
#ifndef ST_POW_H
#define ST_POW_H

#include <stdint.h>

#if defined(__CUDACC__)
#define ST_HD __host__ __device__ __forceinline__
#else
#define ST_HD static inline
#include <math.h>
#include <string.h>
#endif

ST_HD uint64_t st_bits_of(double x)
{
#if defined(__CUDA_ARCH__)
    return (uint64_t)__double_as_longlong(x);
#else
    uint64_t b;
    memcpy(&b, &x, sizeof b);
    return b;
#endif
}

ST_HD double st_double_of(uint64_t b)
{
#if defined(__CUDA_ARCH__)
    return __longlong_as_double((long long)b);
#else
    double x;
    memcpy(&x, &b, sizeof x);
    return x;
#endif
}

/* 2^k for -1022 <= k <= 1023, built from the exponent field (exact). */
ST_HD double st_pow2i(int k)
{
    return st_double_of((uint64_t)(k + 1023) << 52);
}

/* Natural logarithm for finite x > 0. */
ST_HD double st_log_pos(double x)
{
    const double LN2 = 0.69314718055994530942;
    const double SQRT2 = 1.41421356237309504880;
    int e = 0;
    if (x < 2.2250738585072014e-308) { /* subnormal: scale into the normal range first */
        x = x * 18014398509481984.0;    /* 2^54, exact */
        e = -54;
    }
    uint64_t b = st_bits_of(x);
    e += (int)((b >> 52) & 0x7ff) - 1023;
    double m = st_double_of((b & 0x000fffffffffffffULL) | 0x3ff0000000000000ULL); /* [1,2) */
    if (m > SQRT2) {
        m = m * 0.5;
        e += 1;
    }
    double s = (m - 1.0) / (m + 1.0);
    double z = s * s;
    double p = 1.0 / 23.0;
    p = p * z + 1.0 / 21.0;
    p = p * z + 1.0 / 19.0;
    p = p * z + 1.0 / 17.0;
    p = p * z + 1.0 / 15.0;
    p = p * z + 1.0 / 13.0;
    p = p * z + 1.0 / 11.0;
    p = p * z + 1.0 / 9.0;
    p = p * z + 1.0 / 7.0;
    p = p * z + 1.0 / 5.0;
    p = p * z + 1.0 / 3.0;
    p = p * z + 1.0;
    double lnm = (2.0 * s) * p;
    return (double)e * LN2 + lnm;
}

/* Exponential for |y| <= 700. */
ST_HD double st_exp_small(double y)
{
    const double LN2 = 0.69314718055994530942;
    const double INV_LN2 = 1.44269504088896340736;
    double t = y * INV_LN2;
    /* round to nearest integer without library calls: |t| < 1100 */
    int k = (int)(t >= 0.0 ? t + 0.5 : t - 0.5);
    double r = y - (double)k * LN2;
    double p = 1.0 / 87178291200.0;          /* 1/14! */
    p = p * r + 1.0 / 6227020800.0;          /* 1/13! */
    p = p * r + 1.0 / 479001600.0;           /* 1/12! */
    p = p * r + 1.0 / 39916800.0;            /* 1/11! */
    p = p * r + 1.0 / 3628800.0;             /* 1/10! */
    p = p * r + 1.0 / 362880.0;              /* 1/9!  */
    p = p * r + 1.0 / 40320.0;               /* 1/8!  */
    p = p * r + 1.0 / 5040.0;                /* 1/7!  */
    p = p * r + 1.0 / 720.0;                 /* 1/6!  */
    p = p * r + 1.0 / 120.0;                 /* 1/5!  */
    p = p * r + 1.0 / 24.0;                  /* 1/4!  */
    p = p * r + 1.0 / 6.0;                   /* 1/3!  */
    p = p * r + 0.5;                         /* 1/2!  */
    p = p * r + 1.0;
    p = p * r + 1.0;
    /* scale by 2^k in two halves so that k down to -1074 does not leave the exponent range */
    int k1 = k / 2;
    int k2 = k - k1;
    return (p * st_pow2i(k1)) * st_pow2i(k2);
}

/* x^0.687 for x >= 0 (0 for x <= 0, x itself for inf/nan). */
ST_HD double st_pow0687(double x)
{
    if (!(x > 0.0)) return x != x ? x : 0.0;
    if (x > 1.0e300) return x;
    return st_exp_small(0.687 * st_log_pos(x));
}

ST_HD uint32_t st_bits_of_f(float x)
{
#if defined(__CUDA_ARCH__)
    return (uint32_t)__float_as_uint(x);
#else
    uint32_t b;
    memcpy(&b, &x, sizeof b);
    return b;
#endif
}

ST_HD float st_float_of(uint32_t b)
{
#if defined(__CUDA_ARCH__)
    return __uint_as_float(b);
#else
    float x;
    memcpy(&x, &b, sizeof x);
    return x;
#endif
}

/* 2^k for -126 <= k <= 127 (exact) */
ST_HD float st_pow2if(int k)
{
    return st_float_of((uint32_t)(k + 127) << 23);
}

/* Fused multiply-add, correctly rounded on both sides (glibc's fmaf and the GPU's FFMA
 * round once), so explicit fma calls give the same bits on host and device even though
 * neither compiler may contract a*b+c on its own. */
ST_HD float st_fmaf(float a, float b, float c)
{
#if defined(__CUDA_ARCH__)
    return __fmaf_rn(a, b, c);
#else
    return fmaf(a, b, c);
#endif
}

/* x^0.687 for the FP32 and mixed drag (the drag is evaluated in FP32).
 *   x = 2^e m, m in [sqrt(1/2), sqrt(2)), t = m - 1 (exact);
 *   687 e = 1000 k + r with integer k and 0 <= r < 1000, so 0.687 e = k + r/1000 exactly;
 *   x^0.687 = (1 + t)^0.687 * 2^(r/1000) * 2^k,
 * the first two factors by polynomials (degree 8 in t, degree 6 in r; coefficients fitted by
 * least squares on Chebyshev nodes, pow_coeffs.py, approximation error below 0.05 ulp each)
 * evaluated by Horner's rule with fma, the last by the exponent field.  All arithmetic is
 * single precision or integer; nothing is converted to double.
 * Within 2 ulp of the correctly rounded value for every normal and subnormal x (the CPU
 * tests check this against a double-precision reference).
 *
 * st_pow0687f_mant: for finite x > 0, the first factor p and the exponent e. */
ST_HD float st_pow0687f_mant(float x, int* ep)
{
    uint32_t b = st_bits_of_f(x);
    int e = 0;
    if ((b >> 23) == 0) {                          /* subnormal */
        x = x * 16777216.0f;                       /* 2^24, exact */
        e = -24;
        b = st_bits_of_f(x);
    }
    e += (int)((b >> 23) & 0xff) - 127;
    float m = st_float_of((b & 0x007fffffu) | 0x3f800000u); /* [1,2) */
    if (m > 1.41421356f) {
        m = m * 0.5f;
        e += 1;
    }
    const float t = m - 1.0f;
    float p = -0x1.921f0ep-8f;
    p = st_fmaf(p, t, 0x1.68372ap-7f);
    p = st_fmaf(p, t, -0x1.b6bb7ep-7f);
    p = st_fmaf(p, t, 0x1.2657a8p-6f);
    p = st_fmaf(p, t, -0x1.bd5c3ap-6f);
    p = st_fmaf(p, t, 0x1.817e2ap-5f);
    p = st_fmaf(p, t, -0x1.b862bep-4f);
    p = st_fmaf(p, t, 0x1.5fbe76p-1f);
    p = st_fmaf(p, t, 1.0f);
    *ep = e;                                       /* -149 <= e <= 128 */
    return p;
}

/* The exponent factor of x^0.687 = p * q * 2^k for x = 2^e m: q = 2^(r/1000) and s2k = 2^k,
 * which depend on e alone (callers may tabulate them). */
ST_HD void st_pow0687f_efac(int e, float* q_out, float* s2k_out)
{
    const int y = 687 * e;                         /* |y| <= 103050 */
    const int k = y >= 0 ? y / 1000 : -((999 - y) / 1000);   /* floor(y / 1000) */
    const float r = (float)(y - 1000 * k);         /* exact integer in [0, 1000) */
    float q = 0x1.08638ep-72f;
    q = st_fmaf(q, r, 0x1.6dafdep-60f);
    q = st_fmaf(q, r, 0x1.5cea7ap-47f);
    q = st_fmaf(q, r, 0x1.e8030ap-35f);
    q = st_fmaf(q, r, 0x1.01f20ep-22f);
    q = st_fmaf(q, r, 0x1.6b689cp-11f);
    q = st_fmaf(q, r, 1.0f);
    *q_out = q;
    *s2k_out = st_pow2if(k);                       /* -104 <= k <= 88 */
}

ST_HD float st_pow0687f(float x)
{
    if (!(x > 0.0f)) return x != x ? x : 0.0f;
    if ((st_bits_of_f(x) >> 23) == 0xff) return x;   /* +inf */
    int e;
    const float p = st_pow0687f_mant(x, &e);
    float q, s2k;
    st_pow0687f_efac(e, &q, &s2k);
    return (p * q) * s2k;
}

#endif /* ST_POW_H */

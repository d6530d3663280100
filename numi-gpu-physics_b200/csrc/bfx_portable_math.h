/*
 * Portable, bit-reproducible sine and cosine for host (gcc) and device (nvcc).
 *
 * The geometry predicates of the moving-boundary step (cell occupancy, cut
 * links, wing frames) must evaluate to identical bits on the CPU and the GPU,
 * because cut-link sets and directions are compared bit-exactly.  Vendor math
 * libraries differ between host and device, so the few transcendental values
 * the geometry needs (flapping phase, stroke/pitch rotations, wing twist) are
 * computed here with plain IEEE-754 double additions and multiplications only:
 *
 *   1. Cody-Waite argument reduction by pi/2 with a three-part split of pi/2
 *      (33 + 33 + 53 significant bits; computed from pi to 80 digits by
 *      Machin's formula), so k * PIO2_HI and k * PIO2_MID are exact for
 *      |k| < 2^20.
 *   2. Truncated Taylor series of sin and cos on |r| <= pi/4 evaluated in
 *      Horner form (truncation error below 1e-20 there).
 *
 * Both compilers must be told not to contract a*b+c into FMA for this file's
 * callers (gcc -ffp-contract=off, nvcc --fmad=false), which the builds do.
 */
#ifndef BFX_PORTABLE_MATH_H
#define BFX_PORTABLE_MATH_H

#if defined(__CUDACC__)
#define BFX_HD __host__ __device__ __forceinline__
#else
#define BFX_HD static inline
#endif

#define BFX_PIO2_HI 1.5707963267341256
#define BFX_PIO2_MID 6.077100506303966e-11
#define BFX_PIO2_LO 2.0222662487959506e-21
#define BFX_TWO_OVER_PI 0.6366197723675814

/* sin(r) for |r| <= pi/4: r - r^3/3! + ... - r^19/19! */
BFX_HD double bfx_sin_kernel(double r) {
    double r2 = r * r;
    double p = -8.22063524662433e-18;
    p = p * r2 + 2.8114572543455206e-15;
    p = p * r2 - 7.647163731819816e-13;
    p = p * r2 + 1.6059043836821613e-10;
    p = p * r2 - 2.505210838544172e-08;
    p = p * r2 + 2.7557319223985893e-06;
    p = p * r2 - 0.0001984126984126984;
    p = p * r2 + 0.008333333333333333;
    p = p * r2 - 0.16666666666666666;
    return r + (r * r2) * p;
}

/* cos(r) for |r| <= pi/4: 1 - r^2/2! + ... + r^20/20! */
BFX_HD double bfx_cos_kernel(double r) {
    double r2 = r * r;
    double p = 4.110317623312165e-19;
    p = p * r2 - 1.5619206968586225e-16;
    p = p * r2 + 4.779477332387385e-14;
    p = p * r2 - 1.1470745597729725e-11;
    p = p * r2 + 2.08767569878681e-09;
    p = p * r2 - 2.755731922398589e-07;
    p = p * r2 + 2.48015873015873e-05;
    p = p * r2 - 0.001388888888888889;
    p = p * r2 + 0.041666666666666664;
    p = p * r2 - 0.5;
    return 1.0 + r2 * p;
}

/* Round to nearest integer (halves away from zero) with IEEE ops only. */
BFX_HD double bfx_round_d(double x) {
    double a = x < 0.0 ? -x : x;
    double t = a + 0.5;
    /* floor for non-negative values below 2^52 via the 2^52 trick */
    double f;
    if (t >= 4503599627370496.0) {
        f = t;
    } else {
        f = (t + 4503599627370496.0) - 4503599627370496.0;
        if (f > t) f = f - 1.0;
    }
    return x < 0.0 ? -f : f;
}

/* Reduces x to r in [-pi/4, pi/4] and returns the quadrant k mod 4. */
BFX_HD int bfx_reduce_pio2(double x, double* r) {
    double k = bfx_round_d(x * BFX_TWO_OVER_PI);
    *r = ((x - k * BFX_PIO2_HI) - k * BFX_PIO2_MID) - k * BFX_PIO2_LO;
    long long ki = (long long)k;
    return (int)(ki & 3LL);
}

BFX_HD double bfx_sin(double x) {
    double r;
    int q = bfx_reduce_pio2(x, &r);
    switch (q) {
    case 0: return bfx_sin_kernel(r);
    case 1: return bfx_cos_kernel(r);
    case 2: return -bfx_sin_kernel(r);
    default: return -bfx_cos_kernel(r);
    }
}

BFX_HD double bfx_cos(double x) {
    double r;
    int q = bfx_reduce_pio2(x, &r);
    switch (q) {
    case 0: return bfx_cos_kernel(r);
    case 1: return -bfx_sin_kernel(r);
    case 2: return -bfx_cos_kernel(r);
    default: return bfx_sin_kernel(r);
    }
}

/* Single-precision entry points: evaluate in double, round once. */
BFX_HD float bfx_sinf(float x) { return (float)bfx_sin((double)x); }
BFX_HD float bfx_cosf(float x) { return (float)bfx_cos((double)x); }

/*
 * Natural logarithm, exponential and power for the beta-planform chord law
 * (pow of a number in [0, 1/4]), with the same IEEE double operations on
 * host and device:
 *
 *   log x = e ln 2 + log m,  x = m 2^e with m in [sqrt(1/2), sqrt(2)),
 *           log m = 2 atanh s = 2 (s + s^3/3 + ... + s^25/25), s = (m-1)/(m+1),
 *           |s| <= 0.1716, so the first omitted term is below 1e-20;
 *   exp y = 2^k exp r,  k = round(y / ln 2), r = y - k ln 2 (two-part ln 2:
 *           a 29-bit head, exact times |k| < 2^24, and the double tail),
 *           |r| <= 0.35, exp r by its Taylor series to r^17/17!.
 *
 * ln 2 was evaluated to 60 digits with Python's decimal module; the series
 * coefficients are exact rational expressions folded by the compiler.
 */
#define BFX_LN2_HI 0.6931471806019545
#define BFX_LN2_LO -4.2009150726810846e-11
#define BFX_INV_LN2 1.4426950408889634

/* Bits of a double and back, by bit pattern (no arithmetic). */
BFX_HD unsigned long long bfx_dbits(double x) {
#if defined(__CUDA_ARCH__)
    return (unsigned long long)__double_as_longlong(x);
#else
    union { double d; unsigned long long u; } v;
    v.d = x;
    return v.u;
#endif
}
BFX_HD double bfx_dfrombits(unsigned long long u) {
#if defined(__CUDA_ARCH__)
    return __longlong_as_double((long long)u);
#else
    union { double d; unsigned long long u; } v;
    v.u = u;
    return v.d;
#endif
}

/* log x for a positive, finite, normal double x. */
BFX_HD double bfx_log(double x) {
    const unsigned long long b = bfx_dbits(x);
    int e = (int)((b >> 52) & 0x7FFull) - 1023;
    double m = bfx_dfrombits((b & 0x000FFFFFFFFFFFFFull) | 0x3FF0000000000000ull); /* [1, 2) */
    if (m > 1.4142135623730951) {
        m = m * 0.5;
        e += 1;
    }
    const double s = (m - 1.0) / (m + 1.0);
    const double s2 = s * s;
    double p = 1.0 / 25.0;
    p = p * s2 + 1.0 / 23.0;
    p = p * s2 + 1.0 / 21.0;
    p = p * s2 + 1.0 / 19.0;
    p = p * s2 + 1.0 / 17.0;
    p = p * s2 + 1.0 / 15.0;
    p = p * s2 + 1.0 / 13.0;
    p = p * s2 + 1.0 / 11.0;
    p = p * s2 + 1.0 / 9.0;
    p = p * s2 + 1.0 / 7.0;
    p = p * s2 + 1.0 / 5.0;
    p = p * s2 + 1.0 / 3.0;
    const double log_m = 2.0 * s + (2.0 * s) * (s2 * p);
    const double de = (double)e;
    return de * BFX_LN2_HI + (de * BFX_LN2_LO + log_m);
}

/* exp y for y in [-700, 700]. */
BFX_HD double bfx_exp(double y) {
    const double k = bfx_round_d(y * BFX_INV_LN2);
    const double r = (y - k * BFX_LN2_HI) - k * BFX_LN2_LO;
    double p = 1.0 / 355687428096000.0;    /* 1/17! */
    p = p * r + 1.0 / 20922789888000.0;    /* 1/16! */
    p = p * r + 1.0 / 1307674368000.0;
    p = p * r + 1.0 / 87178291200.0;
    p = p * r + 1.0 / 6227020800.0;
    p = p * r + 1.0 / 479001600.0;
    p = p * r + 1.0 / 39916800.0;
    p = p * r + 1.0 / 3628800.0;
    p = p * r + 1.0 / 362880.0;
    p = p * r + 1.0 / 40320.0;
    p = p * r + 1.0 / 5040.0;
    p = p * r + 1.0 / 720.0;
    p = p * r + 1.0 / 120.0;
    p = p * r + 1.0 / 24.0;
    p = p * r + 1.0 / 6.0;
    p = p * r + 0.5;
    p = p * r + 1.0;
    p = p * r + 1.0;
    const long long ki = (long long)k;
    return p * bfx_dfrombits((unsigned long long)(ki + 1023) << 52);
}

/* pow(b, e) for a finite float b >= 0 and |e * log b| <= 700: evaluated in
 * double, rounded once.  pow(0, e) is 0 for e > 0 and 1 for e == 0. */
BFX_HD float bfx_powf(float b, float e) {
    if (b == 0.0f) return e > 0.0f ? 0.0f : 1.0f;
    return (float)bfx_exp((double)e * bfx_log((double)b));
}

#endif /* BFX_PORTABLE_MATH_H */

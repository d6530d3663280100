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

#endif /* BFX_PORTABLE_MATH_H */

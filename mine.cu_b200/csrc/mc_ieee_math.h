/*
 * mc_ieee_math.h - the "ieee" numerics mode's transcendental functions.
 *
 * The reference compiles its kernels with `nvcc --use_fast_math`
 * (setup.py:19), so its sinf/cosf/tanf are hardware approximations whose
 * bits no CPU can reproduce.  The "ieee" numerics mode replaces them with
 * the functions below, which use only IEEE-754 single-precision +, -, *, /
 * (each rounded to nearest-even, no fused multiply-add) plus floorf.  The
 * same source is compiled by nvcc (device, -fmad=false, no fast math) and by
 * gcc (host, -ffp-contract=off, no -ffast-math), so both sides produce the
 * same bits for every input.
 *
 * Method (published): Cody & Waite argument reduction (W. J. Cody and
 * W. Waite, "Software Manual for the Elementary Functions", 1980) by
 * multiples of pi/2 split into three parts, P1 with 9 significant bits and
 * P2 with 12, so that k*P1 and k*P2 are exact for |k| < 2^12; followed by
 * the Taylor series of sin (degree 9) and cos (degree 10) on [-pi/4, pi/4],
 * whose truncation error there is below 3e-9 relative, under one float ulp.
 * tan is sin/cos with one correctly rounded division.
 *
 * Domain: |x| <= 1e7 gives a deterministic result (accurate to a few ulp
 * for |x| < 6000); NaN, +-inf and |x| > 1e7 return NaN (x - x) or a
 * deterministic value of the reduced argument, identically on host and
 * device.  The functions are not correctly rounded; they only need to be
 * identical on both sides.
 */
#ifndef MC_IEEE_MATH_H
#define MC_IEEE_MATH_H

#ifdef __CUDACC__
#define MC_HD static __host__ __device__ __forceinline__
#else
#define MC_HD static inline
#endif

#ifndef __CUDACC__
#include <math.h>
#endif

/* pi/2 = MC_PIO2_1 + MC_PIO2_2 + MC_PIO2_3 (to ~2^-48) */
#define MC_PIO2_1 1.5703125f                 /* 0x1.92p+0     (9 bits)  */
#define MC_PIO2_2 4.837512969970703125e-4f   /* 0x1.fb4p-12   (12 bits) */
#define MC_PIO2_3 7.549790126404332e-08f     /* 0x1.4442d2p-24          */
#define MC_2_OVER_PI 0.63661974668502807617f /* 0x1.45f306p-1           */

/* Reduce x to r in about [-pi/4, pi/4] and quadrant q in 0..3. */
MC_HD float mc_ieee_reduce(float x, int* q) {
    float k = floorf(x * MC_2_OVER_PI + 0.5f);
    /* |k| <= 6.4e6 here because callers pass |x| <= 1e7 */
    long long ki = (long long)k;
    *q = (int)(ki & 3);
    float r = x - k * MC_PIO2_1;
    r = r - k * MC_PIO2_2;
    r = r - k * MC_PIO2_3;
    return r;
}

/* Taylor series of sin on the reduced interval (Horner in r^2). */
MC_HD float mc_ieee_sin_poly(float r) {
    float r2 = r * r;
    float p = 2.7557318844628753e-06f;      /*  1/9!  */
    p = p * r2 - 1.9841270113829523e-04f;   /* -1/7!  */
    p = p * r2 + 8.3333337679505348e-03f;   /*  1/5!  */
    p = p * r2 - 1.6666667163372040e-01f;   /* -1/3!  */
    p = p * r2;
    return r + r * p;
}

/* Taylor series of cos on the reduced interval (Horner in r^2). */
MC_HD float mc_ieee_cos_poly(float r) {
    float r2 = r * r;
    float p = -2.7557319981497130e-07f;     /* -1/10! */
    p = p * r2 + 2.4801587642286904e-05f;   /*  1/8!  */
    p = p * r2 - 1.3888889225199819e-03f;   /* -1/6!  */
    p = p * r2 + 4.1666667908430100e-02f;   /*  1/4!  */
    p = p * r2 - 0.5f;                      /* -1/2!  */
    p = p * r2;
    return 1.0f + p;
}

MC_HD int mc_ieee_in_domain(float x) {
    /* false for NaN too */
    return (x >= -1.0e7f) && (x <= 1.0e7f);
}

MC_HD float mc_ieee_sinf(float x) {
    if (!mc_ieee_in_domain(x)) return x - x;
    int q;
    float r = mc_ieee_reduce(x, &q);
    float s = mc_ieee_sin_poly(r);
    float c = mc_ieee_cos_poly(r);
    switch (q) {
        case 0: return s;
        case 1: return c;
        case 2: return -s;
        default: return -c;
    }
}

MC_HD float mc_ieee_cosf(float x) {
    if (!mc_ieee_in_domain(x)) return x - x;
    int q;
    float r = mc_ieee_reduce(x, &q);
    float s = mc_ieee_sin_poly(r);
    float c = mc_ieee_cos_poly(r);
    switch (q) {
        case 0: return c;
        case 1: return -s;
        case 2: return -c;
        default: return s;
    }
}

MC_HD void mc_ieee_sincosf(float x, float* s_out, float* c_out) {
    *s_out = mc_ieee_sinf(x);
    *c_out = mc_ieee_cosf(x);
}

MC_HD float mc_ieee_tanf(float x) {
#ifdef __CUDA_ARCH__
    return __fdiv_rn(mc_ieee_sinf(x), mc_ieee_cosf(x));
#else
    return mc_ieee_sinf(x) / mc_ieee_cosf(x);
#endif
}

#endif /* MC_IEEE_MATH_H */

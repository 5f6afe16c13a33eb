/*
 * ORACLE / TEST INFRASTRUCTURE ONLY.  Deterministic FP64 exp, log, asin, acos
 * for the CPU oracle.
 *
 * The reference calls the libm routines exp (forcing.f90:261), log
 * (forcing.f90:222), acos (ridging.f90:57-58) and asin (ridging.f90:154).
 * Library transcendentals are not bit-identical between the host libm and the
 * CUDA device library, so the oracle and the GPU kernels both evaluate these
 * four functions with the same published methods, written here with only
 * IEEE-754 +, -, *, / and sqrt (all correctly rounded) so that both sides
 * round identically:
 *   - exp: Cody & Waite argument reduction x = k ln2 + r with ln2 split into a
 *     high part with 21 trailing zero bits and a low part, then the Taylor
 *     series of e^r to degree 14 (|r| <= ln2/2) in Horner form.
 *   - log: x = m 2^e with m in [sqrt(1/2), sqrt(2)), f = (m-1)/(m+1),
 *     log m = 2 atanh f = 2 (f + f^3/3 + f^5/5 + ...), 14 terms.
 *   - asin: |x| <= 1/2 by the Maclaurin series of asin to degree 57;
 *     |x| > 1/2 by asin x = pi/2 - 2 asin(sqrt((1-|x|)/2)).
 *   - acos from the same asin kernel (acos x = pi/2 - asin x, or
 *     2 asin(sqrt((1-x)/2)) / pi - 2 asin(sqrt((1+x)/2)) away from 0).
 * The coefficients are exact rationals (1/k!, 1/(2k+1), C(2k,k)/(4^k (2k+1)))
 * rounded to double; the split constants were computed from ln 2 and pi to 60
 * digits.  The product's copy of these routines lives in the CUDA sources and
 * is written independently; the tests check both against libm and against each
 * other bit for bit.
 *
 * Compile with -ffp-contract=off: no fused multiply-add may be formed.
 */
#ifndef GODAR_DETMATH_ORACLE_H
#define GODAR_DETMATH_ORACLE_H

#include <math.h>
#include <stdint.h>
#include <string.h>

static inline double odm_from_bits(uint64_t b) { double d; memcpy(&d, &b, 8); return d; }
static inline uint64_t odm_bits(double d) { uint64_t b; memcpy(&b, &d, 8); return b; }

/* 2^k for k in [-1022, 1023] */
static inline double odm_pow2(int k) { return odm_from_bits((uint64_t)(k + 1023) << 52); }

static inline double odm_exp(double x)
{
    const double INV_LN2 = 0x1.71547652b82fep+0;
    const double LN2_HI = 0x1.62e42fee00000p-1;
    const double LN2_LO = 0x1.a39ef35793c76p-33;
    if (x != x) return x;
    if (x > 709.782712893384) return odm_from_bits(0x7ff0000000000000ULL);
    if (x < -745.2) return 0.0;
    double kd = x * INV_LN2;
    /* round to nearest integer, ties away from zero */
    double kr = (kd >= 0.0) ? (double)(int64_t)(kd + 0.5) : -(double)(int64_t)(0.5 - kd);
    int k = (int)kr;
    double r = (x - kr * LN2_HI) - kr * LN2_LO;
    double p = 0x1.93974a8c07c9dp-37;          /* 1/14! */
    p = p * r + 0x1.6124613a86d09p-33;         /* 1/13! */
    p = p * r + 0x1.1eed8eff8d898p-29;
    p = p * r + 0x1.ae64567f544e4p-26;
    p = p * r + 0x1.27e4fb7789f5cp-22;
    p = p * r + 0x1.71de3a556c734p-19;
    p = p * r + 0x1.a01a01a01a01ap-16;
    p = p * r + 0x1.a01a01a01a01ap-13;
    p = p * r + 0x1.6c16c16c16c17p-10;
    p = p * r + 0x1.1111111111111p-7;
    p = p * r + 0x1.5555555555555p-5;
    p = p * r + 0x1.5555555555555p-3;
    p = p * r + 0x1.0000000000000p-1;
    p = p * r + 1.0;
    p = p * r + 1.0;
    if (k > 1023) return (p * 2.0) * odm_pow2(k - 1);
    if (k < -1021) return (p * odm_pow2(k + 1000)) * odm_pow2(-1000);
    return p * odm_pow2(k);
}

static inline double odm_log(double x)
{
    const double LN2_HI = 0x1.62e42fee00000p-1;
    const double LN2_LO = 0x1.a39ef35793c76p-33;
    const double SQRT2 = 0x1.6a09e667f3bcdp+0;
    if (x != x) return x;
    if (x < 0.0) return odm_from_bits(0x7ff8000000000000ULL);
    if (x == 0.0) return -odm_from_bits(0x7ff0000000000000ULL);
    if (x == odm_from_bits(0x7ff0000000000000ULL)) return x;
    int e = 0;
    uint64_t b = odm_bits(x);
    if ((b >> 52) == 0) {               /* subnormal: scale by 2^54 exactly */
        x = x * 0x1.0p54;
        b = odm_bits(x);
        e = -54;
    }
    e += (int)((b >> 52) & 0x7ff) - 1023;
    double m = odm_from_bits((b & 0x000fffffffffffffULL) | 0x3ff0000000000000ULL);
    if (m > SQRT2) { m = m * 0.5; e += 1; }
    double f = (m - 1.0) / (m + 1.0);
    double s = f * f;
    double p = 0x1.2f684bda12f68p-5;            /* 1/27 */
    p = p * s + 0x1.47ae147ae147bp-5;           /* 1/25 */
    p = p * s + 0x1.642c8590b2164p-5;
    p = p * s + 0x1.8618618618618p-5;
    p = p * s + 0x1.af286bca1af28p-5;
    p = p * s + 0x1.e1e1e1e1e1e1ep-5;
    p = p * s + 0x1.1111111111111p-4;
    p = p * s + 0x1.3b13b13b13b14p-4;
    p = p * s + 0x1.745d1745d1746p-4;
    p = p * s + 0x1.c71c71c71c71cp-4;
    p = p * s + 0x1.2492492492492p-3;
    p = p * s + 0x1.999999999999ap-3;
    p = p * s + 0x1.5555555555555p-2;           /* 1/3 */
    double f2 = f + f;
    double logm = f2 + (f2 * s) * p;
    double ed = (double)e;
    return ed * LN2_HI + (logm + ed * LN2_LO);
}

/* asin on [-1/2, 1/2] */
static inline double odm_asin_core(double x)
{
    double s = x * x;
    double p = 0x1.e82be60d9127ep-10;           /* k = 28 */
    p = p * s + 0x1.018f963c229bfp-9;
    p = p * s + 0x1.1052bc5fa960ap-9;
    p = p * s + 0x1.208d3570ae5a6p-9;
    p = p * s + 0x1.3275586c5f2f0p-9;
    p = p * s + 0x1.464c0950f7d47p-9;
    p = p * s + 0x1.5c5f56efaaaabp-9;
    p = p * s + 0x1.750de64d7d05fp-9;
    p = p * s + 0x1.90cb77f60c7cep-9;
    p = p * s + 0x1.b026f57b13b14p-9;
    p = p * s + 0x1.d3d2a8e0dd67dp-9;
    p = p * s + 0x1.fcaf8fb6db6dbp-9;
    p = p * s + 0x1.15ee9d45d1746p-8;
    p = p * s + 0x1.31683bdef7bdfp-8;
    p = p * s + 0x1.51ba308d3dcb1p-8;
    p = p * s + 0x1.782dda12f684cp-8;
    p = p * s + 0x1.a6863d70a3d71p-8;
    p = p * s + 0x1.df3bd37a6f4dfp-8;
    p = p * s + 0x1.12ef3cf3cf3cfp-7;
    p = p * s + 0x1.3fde50d79435ep-7;
    p = p * s + 0x1.7a87878787878p-7;
    p = p * s + 0x1.c99999999999ap-7;
    p = p * s + 0x1.1c4ec4ec4ec4fp-6;
    p = p * s + 0x1.6e8ba2e8ba2e9p-6;
    p = p * s + 0x1.f1c71c71c71c7p-6;
    p = p * s + 0x1.6db6db6db6db7p-5;
    p = p * s + 0x1.3333333333333p-4;
    p = p * s + 0x1.5555555555555p-3;           /* k = 1 */
    return x + (x * s) * p;
}

static inline double odm_asin(double x)
{
    const double PIO2_HI = 0x1.921fb54442d18p+0;
    const double PIO2_LO = 0x1.1a62633145c07p-54;
    double ax = x < 0.0 ? -x : x;
    if (!(ax <= 1.0)) return odm_from_bits(0x7ff8000000000000ULL);
    if (ax <= 0.5) return odm_asin_core(x);
    double z = sqrt((1.0 - ax) * 0.5);
    double a = odm_asin_core(z);
    double r = (PIO2_HI - 2.0 * a) + PIO2_LO;
    return x < 0.0 ? -r : r;
}

static inline double odm_acos(double x)
{
    const double PIO2_HI = 0x1.921fb54442d18p+0;
    const double PIO2_LO = 0x1.1a62633145c07p-54;
    const double PI_HI = 0x1.921fb54442d18p+1;
    const double PI_LO = 0x1.1a62633145c07p-53;
    double ax = x < 0.0 ? -x : x;
    if (!(ax <= 1.0)) return odm_from_bits(0x7ff8000000000000ULL);
    if (ax <= 0.5) return (PIO2_HI - odm_asin_core(x)) + PIO2_LO;
    if (x > 0.0) return 2.0 * odm_asin_core(sqrt((1.0 - x) * 0.5));
    return (PI_HI - 2.0 * odm_asin_core(sqrt((1.0 + x) * 0.5))) + PI_LO;
}

#endif

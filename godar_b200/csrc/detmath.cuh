// Deterministic FP64 transcendentals for the FP64 ("plain") step.
//
// The reference evaluates exp (forcing.f90:261), log (forcing.f90:222), acos
// (ridging.f90:57-58) and asin (ridging.f90:154) with the host libm.  The CUDA
// device library rounds differently in the last place, so the FP64 step uses
// these routines instead: only IEEE +, -, *, / and sqrt, no fused
// multiply-add (this file is compiled with --fmad=false), so the result is the
// same bit pattern on every device and on the host.
//
// Methods (published, textbook):
//   exp  - Cody & Waite reduction x = k ln2 + r (ln2 = hi + lo, hi with 21
//          trailing zero bits), Taylor polynomial of e^r of degree 14.
//   log  - x = m 2^e, m in [sqrt(1/2), sqrt(2)); log m = 2 atanh((m-1)/(m+1))
//          by its odd power series (13 terms after the first).
//   asin - Maclaurin series on |x| <= 1/2 (degree 57); beyond,
//          asin x = pi/2 - 2 asin(sqrt((1-|x|)/2)).
//   acos - pi/2 - asin x on |x| <= 1/2; 2 asin(sqrt((1-x)/2)) for x > 1/2;
//          pi - 2 asin(sqrt((1+x)/2)) for x < -1/2.
// Series coefficients are the exact rationals 1/k!, 1/(2k+1) and
// C(2k,k)/(4^k (2k+1)) rounded to double.  Accuracy: within 2 ulp of a
// correctly rounded result over the ranges the step uses (tested).
#pragma once
#include <cstdint>

#ifdef __CUDACC__
#define GD_HD __host__ __device__ __forceinline__
#else
#define GD_HD inline
#endif

namespace godar {
namespace dm {

GD_HD double from_bits(uint64_t b)
{
#ifdef __CUDA_ARCH__
    return __longlong_as_double((long long)b);
#else
    double d;
    __builtin_memcpy(&d, &b, 8);
    return d;
#endif
}

GD_HD uint64_t to_bits(double d)
{
#ifdef __CUDA_ARCH__
    return (uint64_t)__double_as_longlong(d);
#else
    uint64_t b;
    __builtin_memcpy(&b, &d, 8);
    return b;
#endif
}

GD_HD double two_to(int k) { return from_bits((uint64_t)(k + 1023) << 52); }

GD_HD double exp(double x)
{
    if (x != x) return x;
    if (x > 709.782712893384) return from_bits(0x7ff0000000000000ULL);
    if (x < -745.2) return 0.0;
    const double kd = x * 0x1.71547652b82fep+0;
    const double kr = (kd >= 0.0) ? (double)(long long)(kd + 0.5) : -(double)(long long)(0.5 - kd);
    const int k = (int)kr;
    const double r = (x - kr * 0x1.62e42fee00000p-1) - kr * 0x1.a39ef35793c76p-33;
    // Horner, highest degree first: 1/14!, 1/13!, ..., 1/2!, 1, 1
    double p = 0x1.93974a8c07c9dp-37;
    p = p * r + 0x1.6124613a86d09p-33;
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
    if (k > 1023) return (p * 2.0) * two_to(k - 1);
    if (k < -1021) return (p * two_to(k + 1000)) * two_to(-1000);
    return p * two_to(k);
}

GD_HD double log(double x)
{
    if (x != x) return x;
    if (x < 0.0) return from_bits(0x7ff8000000000000ULL);
    if (x == 0.0) return -from_bits(0x7ff0000000000000ULL);
    if (x == from_bits(0x7ff0000000000000ULL)) return x;
    int e = 0;
    uint64_t b = to_bits(x);
    if ((b >> 52) == 0) {
        x = x * 0x1.0p54;
        b = to_bits(x);
        e = -54;
    }
    e += (int)((b >> 52) & 0x7ff) - 1023;
    double m = from_bits((b & 0x000fffffffffffffULL) | 0x3ff0000000000000ULL);
    if (m > 0x1.6a09e667f3bcdp+0) {
        m = m * 0.5;
        e += 1;
    }
    const double f = (m - 1.0) / (m + 1.0);
    const double s = f * f;
    // 1/27, 1/25, ..., 1/5, 1/3
    double p = 0x1.2f684bda12f68p-5;
    p = p * s + 0x1.47ae147ae147bp-5;
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
    p = p * s + 0x1.5555555555555p-2;
    const double f2 = f + f;
    const double lm = f2 + (f2 * s) * p;
    const double ed = (double)e;
    return ed * 0x1.62e42fee00000p-1 + (lm + ed * 0x1.a39ef35793c76p-33);
}

// asin on [-1/2, 1/2]: coefficients C(2k,k)/(4^k (2k+1)), k = 28 .. 1
GD_HD double asin_core(double x)
{
    const double s = x * x;
    double p = 0x1.e82be60d9127ep-10;
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
    p = p * s + 0x1.5555555555555p-3;
    return x + (x * s) * p;
}

GD_HD double asin(double x)
{
    const double ax = x < 0.0 ? -x : x;
    if (!(ax <= 1.0)) return from_bits(0x7ff8000000000000ULL);
    if (ax <= 0.5) return asin_core(x);
    const double a = asin_core(::sqrt((1.0 - ax) * 0.5));
    const double r = (0x1.921fb54442d18p+0 - 2.0 * a) + 0x1.1a62633145c07p-54;
    return x < 0.0 ? -r : r;
}

GD_HD double acos(double x)
{
    const double ax = x < 0.0 ? -x : x;
    if (!(ax <= 1.0)) return from_bits(0x7ff8000000000000ULL);
    if (ax <= 0.5) return (0x1.921fb54442d18p+0 - asin_core(x)) + 0x1.1a62633145c07p-54;
    if (x > 0.0) return 2.0 * asin_core(::sqrt((1.0 - x) * 0.5));
    return (0x1.921fb54442d18p+1 - 2.0 * asin_core(::sqrt((1.0 + x) * 0.5))) + 0x1.1a62633145c07p-53;
}

}  // namespace dm
}  // namespace godar

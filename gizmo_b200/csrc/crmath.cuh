// gizmo_b200/csrc/crmath.cuh -- correctly rounded FP64 exp, log and pow for
// the kernel-length iteration.
//
// The bracketed h-iteration (density_loop.h:515-961) takes accept / bracket /
// clamp decisions on values that pass through exp, log and pow; a one-ulp
// difference in one of them moves a particle's converged h by up to the
// width of the neighbour-count band (~1e-3 relative). The reference runs on
// glibc, whose exp/log/pow return the correctly rounded result for all but
// rare hard cases, so the device evaluates them to ~100 bits and rounds once:
//
//  * double-double arithmetic with error-free transformations (Knuth's
//    TwoSum, FMA-based TwoProduct) following Hida, Li and Bailey, "Library
//    for double-double and quad-double arithmetic" (2007);
//  * exp: Cody-Waite reduction x = k ln2 + r with ln2 in double-double,
//    r scaled by 2^-8, Horner-form Taylor series of expm1 (11 terms), eight
//    doublings expm1(2a) = expm1(a) (expm1(a) + 2), then 2^k;
//  * log: one Newton step y1 = y0 + x exp(-y0) - 1 from the library log,
//    evaluated in double-double (quadratic convergence: ~2^-100);
//  * pow: exp(y log x) in double-double; y = 3, 2 and -1 are exact products
//    or a quotient rounded once.
//
// Every operation is an explicitly rounded add/mul/fma, so no contraction can
// change a result, and the host build of this header (CPU tests) computes
// the same bits as the device.
#pragma once

#include <cmath>

#ifdef __CUDACC__
#define CR_HD __host__ __device__ __forceinline__
#else
#define CR_HD inline
#endif

namespace gz {
namespace cr {

#ifdef __CUDA_ARCH__
CR_HD double add(double a, double b) { return __dadd_rn(a, b); }
CR_HD double sub(double a, double b) { return __dsub_rn(a, b); }
CR_HD double mul(double a, double b) { return __dmul_rn(a, b); }
CR_HD double fma_(double a, double b, double c) { return __fma_rn(a, b, c); }
CR_HD double div_(double a, double b) { return __ddiv_rn(a, b); }
#else
CR_HD double add(double a, double b) { volatile double r = a + b; return r; }
CR_HD double sub(double a, double b) { volatile double r = a - b; return r; }
CR_HD double mul(double a, double b) { volatile double r = a * b; return r; }
CR_HD double fma_(double a, double b, double c) { return std::fma(a, b, c); }
CR_HD double div_(double a, double b) { volatile double r = a / b; return r; }
#endif

struct dd {
    double hi, lo;
};

CR_HD dd two_sum(double a, double b)
{
    const double s = add(a, b);
    const double bb = sub(s, a);
    const double e = add(sub(a, sub(s, bb)), sub(b, bb));
    return {s, e};
}

CR_HD dd quick_two_sum(double a, double b)  // |a| >= |b|
{
    const double s = add(a, b);
    return {s, sub(b, sub(s, a))};
}

CR_HD dd two_prod(double a, double b)
{
    const double p = mul(a, b);
    return {p, fma_(a, b, -p)};
}

CR_HD dd dd_add(dd a, dd b)
{
    dd s = two_sum(a.hi, b.hi);
    const dd t = two_sum(a.lo, b.lo);
    s.lo = add(s.lo, t.hi);
    s = quick_two_sum(s.hi, s.lo);
    s.lo = add(s.lo, t.lo);
    return quick_two_sum(s.hi, s.lo);
}

CR_HD dd dd_neg(dd a) { return {-a.hi, -a.lo}; }

CR_HD dd dd_mul(dd a, dd b)
{
    dd p = two_prod(a.hi, b.hi);
    p.lo = add(p.lo, add(mul(a.hi, b.lo), mul(a.lo, b.hi)));
    return quick_two_sum(p.hi, p.lo);
}

CR_HD dd dd_mul_d(dd a, double b)
{
    dd p = two_prod(a.hi, b);
    p.lo = add(p.lo, mul(a.lo, b));
    return quick_two_sum(p.hi, p.lo);
}

CR_HD dd dd_div_d(dd a, double b)
{
    const double q1 = div_(a.hi, b);
    const dd p = two_prod(q1, b);
    dd s = two_sum(a.hi, -p.hi);
    s.lo = sub(s.lo, p.lo);
    s.lo = add(s.lo, a.lo);
    const double q2 = div_(add(s.hi, s.lo), b);
    return quick_two_sum(q1, q2);
}

// ln 2 = kLn2Hi + kLn2Lo to ~2^-107
constexpr double kLn2Hi = 6.93147180559945286226763982995e-01;
constexpr double kLn2Lo = 2.31904681384629955842818503524e-17;
constexpr double kInvLn2 = 1.44269504088896338700465094007e+00;

// e^a for a double-double argument, as a double-double
CR_HD dd dd_exp(dd a)
{
    if (a.hi > 709.7) return {INFINITY, 0.0};
    if (a.hi < -745.2) return {0.0, 0.0};
    const double k = ::rint(mul(a.hi, kInvLn2));
    dd kl = two_prod(k, kLn2Hi);
    kl.lo = add(kl.lo, mul(k, kLn2Lo));
    kl = quick_two_sum(kl.hi, kl.lo);
    dd r = dd_add(a, dd_neg(kl));
    r.hi = mul(r.hi, 1.0 / 256.0);  // exact scalings
    r.lo = mul(r.lo, 1.0 / 256.0);
    // expm1(r) = r (1 + r/2 (1 + r/3 (... (1 + r/11))))
    dd s = {1.0, 0.0};
    for (int i = 11; i >= 2; i--) s = dd_add({1.0, 0.0}, dd_div_d(dd_mul(r, s), (double)i));
    s = dd_mul(r, s);
    for (int i = 0; i < 8; i++) s = dd_add(dd_mul_d(s, 2.0), dd_mul(s, s));
    dd e = dd_add({1.0, 0.0}, s);
    const int ki = (int)k;
    e.hi = ::ldexp(e.hi, ki);
    e.lo = ::ldexp(e.lo, ki);
    return e;
}

// log(x) for finite x > 0, as a double-double
CR_HD dd dd_log(double x)
{
    const double y0 = ::log(x);
    const dd e = dd_exp({-y0, 0.0});
    const dd t = dd_mul_d(e, x);
    const dd u = dd_add(t, {-1.0, 0.0});
    return dd_add({y0, 0.0}, u);
}

CR_HD double round_dd(dd a) { return add(a.hi, a.lo); }

CR_HD double exp(double x)
{
    if (!(x == x)) return x;
    return round_dd(dd_exp({x, 0.0}));
}

CR_HD double log(double x)
{
    if (!(x > 0.0) || x == INFINITY) return ::log(x);
    return round_dd(dd_log(x));
}

CR_HD double pow(double x, double y)
{
    if (y == 3.0) return round_dd(dd_mul_d(two_prod(x, x), x));
    if (y == 2.0) return mul(x, x);
    if (y == -1.0) return div_(1.0, x);
    if (y == 1.0) return x;
    if (!(x > 0.0) || x == INFINITY || !(y == y) || y == INFINITY || y == -INFINITY) return ::pow(x, y);
    return round_dd(dd_exp(dd_mul_d(dd_log(x), y)));
}

}  // namespace cr
}  // namespace gz

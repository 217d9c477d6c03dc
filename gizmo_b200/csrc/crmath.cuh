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
//  * exp: table-driven reduction x = (64 m + j) ln2/64 + r (Tang 1989) with a
//    64-entry table of 2^(j/64) in double-double and a Taylor series of
//    expm1(r), then 2^m;
//  * log: one Newton step y1 = y0 + x exp(-y0) - 1 from the library log,
//    evaluated in double-double (quadratic convergence: ~2^-100);
//  * pow: exp(y log x) in double-double; y = 3, 2 and -1 are exact products
//    or a quotient rounded once.
//
// Each function first takes a shorter evaluation (Ziv's strategy: Ziv,
// "Fast evaluation of elementary mathematical functions with correctly
// rounded last bit", ACM TOMS 17(3), 1991): the same reduction with the
// series from its cubic term on in double, accurate to 2^-70 of the result,
// rounded once when that error bound proves the rounding (the value lies
// farther than the bound from the midpoint between two doubles); otherwise
// the ~2^-100 evaluation above decides. Both give the correctly rounded
// result, so the shorter one changes no output, only the time.
//
// Every operation is an explicitly rounded add/mul/fma, so no contraction can
// change a result, and the host build of this header (CPU tests) computes
// the same bits as the device.
#pragma once

#include <cmath>

#ifdef __CUDACC__
#define CR_HD __host__ __device__ __forceinline__
// the ~2^-100 evaluations, taken about once in 10^4-10^5 calls: one copy each,
// called, so the callers' code (and the instruction cache) holds only the
// shorter evaluation
#define CR_COLD inline __host__ __device__ __noinline__
#else
#define CR_HD inline
#define CR_COLD inline
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

// ln 2 = kLn2Hi + kLn2Lo to ~2^-107; ln 2 / 64 likewise (exact scalings)
constexpr double kLn2Hi = 6.93147180559945286226763982995e-01;
constexpr double kLn2Lo = 2.31904681384629955842818503524e-17;
constexpr double kLn2Hi64 = kLn2Hi / 64.0;
constexpr double kLn2Lo64 = kLn2Lo / 64.0;
constexpr double kInv64Ln2 = 92.33248261689366;

// 2^(j/64), j = 0..63, as double-doubles (hi, lo), from 70-digit arithmetic
#define GZ_CR_EXP2_TABLE \
    { \
    {1.0, 0.0}, \
    {1.0108892860517005, -1.5234778603368577e-17}, \
    {1.0218971486541166, 5.109225028973444e-17}, \
    {1.0330248790212284, 7.600838874027088e-18}, \
    {1.0442737824274138, 8.551889705537965e-17}, \
    {1.0556451783605572, 1.759325738772092e-18}, \
    {1.0671404006768237, -7.899853966841582e-17}, \
    {1.0787607977571199, -6.656660436056593e-17}, \
    {1.0905077326652577, -3.046782079812471e-17}, \
    {1.102382583307841, 5.2660368715706944e-17}, \
    {1.1143867425958924, 1.0410278456845571e-16}, \
    {1.1265216186082418, 5.165856758795457e-17}, \
    {1.1387886347566916, 8.912812676025408e-17}, \
    {1.1511892299529827, 3.250710218863827e-17}, \
    {1.1637248587775775, 3.8292048369240935e-17}, \
    {1.1763969916502812, 5.554203254218079e-17}, \
    {1.189207115002721, 3.982015231465646e-17}, \
    {1.202156731452703, 6.644981499252301e-17}, \
    {1.215247359980469, -7.712630692681488e-17}, \
    {1.22848053610687, -1.89878163130253e-17}, \
    {1.241857812073484, 4.658027591836937e-17}, \
    {1.255380757024691, -6.7113898212968784e-18}, \
    {1.2690509571917332, 2.667932131342186e-18}, \
    {1.2828700160787783, 1.713594918243561e-17}, \
    {1.2968395546510096, 2.5382502794888315e-17}, \
    {1.3109612115247644, -7.181536135519454e-17}, \
    {1.3252366431597413, -2.8587312100388614e-17}, \
    {1.339667524053303, 8.927282594831732e-17}, \
    {1.3542555469368927, 7.70094837980299e-17}, \
    {1.3690024229745905, 9.593797919118849e-17}, \
    {1.383909881963832, -6.770511658794786e-17}, \
    {1.3989796725383112, -9.614213209051323e-17}, \
    {1.4142135623730951, -9.667293313452913e-17}, \
    {1.42961333839197, -1.2031642489053655e-17}, \
    {1.4451808069770467, -3.0237581349939873e-17}, \
    {1.460917794180647, -5.600377186075216e-17}, \
    {1.4768261459394993, -3.483994556892796e-17}, \
    {1.4929077282912648, 1.4192920154284036e-17}, \
    {1.5091644275934228, -1.016455327754295e-16}, \
    {1.5255981507445384, -1.1024941712342561e-16}, \
    {1.5422108254079407, 7.949834809697621e-17}, \
    {1.559004400237837, 3.7812070533575275e-17}, \
    {1.5759808451078865, -1.0136916471278304e-17}, \
    {1.593142151342267, -1.0094406542311964e-16}, \
    {1.6104903319492543, 2.4707192569797888e-17}, \
    {1.6280274218573478, -6.712955084707084e-17}, \
    {1.645755478153965, -1.0125679913674773e-16}, \
    {1.6636765803267364, 5.8909926967131e-17}, \
    {1.681792830507429, 8.199010020581497e-17}, \
    {1.7001063537185235, -8.0237193703977e-18}, \
    {1.718619298122478, -1.851380418263111e-17}, \
    {1.7373338352737062, 3.164389299292957e-17}, \
    {1.7562521603732995, 2.960140695448873e-17}, \
    {1.7753764925265212, 6.429731796556572e-17}, \
    {1.7947090750031072, 1.8227458427912087e-17}, \
    {1.8142521755003989, -9.969531538920349e-17}, \
    {1.8340080864093424, 3.283107224245627e-17}, \
    {1.8539791250833855, 9.761887490727594e-17}, \
    {1.8741676341103, -6.122763413004143e-17}, \
    {1.8945759815869656, 3.4034035352165297e-17}, \
    {1.9152065613971474, -1.0619946056195963e-16}, \
    {1.9360617934922943, 1.0332385960676326e-16}, \
    {1.9571441241754002, 8.960767791036668e-17}, \
    {1.978456026387951, 4.0388753109278167e-17}, \
    }
#ifdef __CUDACC__
static __constant__ double kExp2TableDev[64][2] = GZ_CR_EXP2_TABLE;
#endif
static const double kExp2TableHost[64][2] = GZ_CR_EXP2_TABLE;

// e^a for a double-double argument, as a double-double, by table-driven
// reduction (Tang, "Table-driven implementation of the exponential function
// in IEEE floating-point arithmetic", 1989): a = (64 m + j) ln2 / 64 + r with
// |r| <= ln2 / 128, e^a = 2^m 2^(j/64) e^r. expm1(r) is a Taylor series whose
// first five terms are summed in double-double and whose terms from r^6 on
// (below 1e-15 relative) in double, Horner form throughout; accuracy ~2^-100.
CR_HD dd dd_exp_core(dd a, int &m)  // e^a = (result) 2^m, result in [0.98, 2.03]
{
    const double N = ::rint(mul(a.hi, kInv64Ln2));
    dd nl = two_prod(N, kLn2Hi64);
    nl.lo = add(nl.lo, mul(N, kLn2Lo64));
    nl = quick_two_sum(nl.hi, nl.lo);
    const dd r = dd_add(a, dd_neg(nl));
    const double x = r.hi;
    // sum_{k>=6} x^(k-6) / k!, to k = 12
    double q = 2.08767569878680989792e-09;                 // 1/12!
    q = add(mul(q, x), 2.50521083854417187751e-08);         // 1/11!
    q = add(mul(q, x), 2.75573192239858906526e-07);         // 1/10!
    q = add(mul(q, x), 2.75573192239858906526e-06);         // 1/9!
    q = add(mul(q, x), 2.48015873015873015873e-05);         // 1/8!
    q = add(mul(q, x), 1.98412698412698412698e-04);         // 1/7!
    q = add(mul(q, x), 1.38888888888888888889e-03);         // 1/6!
    dd s = dd_add({0.008333333333333333, 1.1564823173178714e-19}, {mul(q, x), 0.0});   // 1/5! + r q
    s = dd_add(dd_mul(s, r), {0.041666666666666664, 2.3129646346357427e-18});           // 1/4!
    s = dd_add(dd_mul(s, r), {0.16666666666666666, 9.25185853854297e-18});              // 1/3!
    s = dd_add(dd_mul(s, r), {0.5, 0.0});
    s = dd_add(dd_mul(s, r), {1.0, 0.0});
    const dd p = dd_mul(s, r);  // expm1(r)
    const int Ni = (int)N;
    const int j = Ni & 63;
    m = (Ni - j) >> 6;
#ifdef __CUDA_ARCH__
    const dd t = {kExp2TableDev[j][0], kExp2TableDev[j][1]};
#else
    const dd t = {kExp2TableHost[j][0], kExp2TableHost[j][1]};
#endif
    return dd_add(t, dd_mul(t, p));
}

CR_HD dd dd_exp(dd a)
{
    if (a.hi > 709.7) return {INFINITY, 0.0};
    if (a.hi < -745.2) return {0.0, 0.0};
    int m = 0;
    dd e = dd_exp_core(a, m);
    e.hi = ::ldexp(e.hi, m);
    e.lo = ::ldexp(e.lo, m);
    return e;
}

// e^a rounded once: the sum is rounded before the scaling by 2^m, which is
// exact for a normal result (scaling the low part first would drop its bits
// once it falls below the normal range, from results of ~2^-969 down)
CR_HD double exp_rounded(dd a)
{
    if (a.hi > 709.7) return INFINITY;
    if (a.hi < -745.2) return 0.0;
    int m = 0;
    const dd e = dd_exp_core(a, m);
    return ::ldexp(add(e.hi, e.lo), m);
}

// log(x) for finite x > 0, as a double-double
CR_HD dd dd_log(double x)
{
    const double y0 = ::log(x);
    int m = 0;
    const dd e = dd_exp_core({-y0, 0.0}, m);      // e^-y0 = e 2^m
    const dd t = dd_mul_d(e, ::ldexp(x, m));      // x 2^m ~ 1/e: exact
    const dd u = dd_add(t, {-1.0, 0.0});
    return dd_add({y0, 0.0}, u);
}

CR_HD double round_dd(dd a) { return add(a.hi, a.lo); }

CR_COLD double exp_long(double x) { return exp_rounded({x, 0.0}); }
CR_COLD double log_long(double x) { return round_dd(dd_log(x)); }
CR_COLD double pow_long(double x, double y) { return exp_rounded(dd_mul_d(dd_log(x), y)); }

// ------------------------------------------------------- the shorter evaluation
// Spacing of the doubles just below v (normal, v > 0): half the ulp of v when
// v is a power of two, its ulp otherwise. A value within half of it of v, on
// either side, rounds to v.
CR_HD double gap_below(double v)
{
    int e = 0;
    const double f = ::frexp(v, &e);  // v = f 2^e, f in [0.5, 1)
    return ::ldexp(f == 0.5 ? 0.5 : 1.0, e - 53);
}

// Whether hi + lo (|lo| <= half the spacing at hi, hi > 0 normal), known to
// within err of the exact value, rounds to hi.
CR_HD bool rounds_to_hi(double hi, double lo, double err) { return add(::fabs(lo), err) < mul(0.5, gap_below(hi)); }

// e^(a.hi + a.lo) = (hi + lo) 2^m for |a.hi| <= 708, |a.lo| <= 2^-40 |a.hi| + 2^-60,
// with |hi + lo - e^a 2^-m| <= 2^-72 hi and hi in [0.98, 2.03]:
//  * the reduction of dd_exp (r = a - N ln2/64 as rh + rl, |rh| <= 0.0055);
//  * expm1(r) = rh + rh^2/2 (rh^2 exact) + rh^3 P(rh) + rl (1 + rh + rh^2/2),
//    P the Taylor series of (e^r - 1 - r - r^2/2) / r^3 to r^5 / 8! (the
//    truncation is below 2^-85), in double: its rounding, below
//    5 x 2^-53 x rh^3/6 <= 2^-75.8, dominates;
//  * 2^(j/64) (1 + p) from the double-double table with one exact product and
//    sum, the small terms in double (their rounding below 2^-75).
CR_HD dd exp_short(dd a, int &m)
{
    const double N = ::rint(mul(a.hi, kInv64Ln2));
    dd nl = two_prod(N, kLn2Hi64);
    nl.lo = add(nl.lo, mul(N, kLn2Lo64));
    dd r = two_sum(a.hi, -nl.hi);
    r.lo = add(sub(r.lo, nl.lo), a.lo);
    r = two_sum(r.hi, r.lo);  // r.hi may be the smaller part when a lies near N ln2/64
    const double rh = r.hi, rl = r.lo;
    double q = 2.48015873015873015873e-05;           // 1/8!
    q = add(mul(q, rh), 1.98412698412698412698e-04);  // 1/7!
    q = add(mul(q, rh), 1.38888888888888888889e-03);  // 1/6!
    q = add(mul(q, rh), 8.33333333333333333333e-03);  // 1/5!
    q = add(mul(q, rh), 4.16666666666666666667e-02);  // 1/4!
    q = add(mul(q, rh), 1.66666666666666666667e-01);  // 1/3!
    const dd s2 = two_prod(rh, rh);
    const double cub = mul(mul(s2.hi, rh), q);
    const double tail = mul(rl, add(1.0, mul(rh, add(1.0, mul(0.5, rh)))));
    const dd p0 = two_sum(rh, mul(0.5, s2.hi));
    const double ph = p0.hi, pl = add(p0.lo, add(mul(0.5, s2.lo), add(cub, tail)));
    const int Ni = (int)N;
    const int j = Ni & 63;
    m = (Ni - j) >> 6;
#ifdef __CUDA_ARCH__
    const double th = kExp2TableDev[j][0], tl = kExp2TableDev[j][1];
#else
    const double th = kExp2TableHost[j][0], tl = kExp2TableHost[j][1];
#endif
    const dd tp = two_prod(th, ph);
    const dd sum = two_sum(th, tp.hi);
    const double lo = add(sum.lo, add(tp.lo, add(tl, add(mul(th, pl), mul(tl, ph)))));
    return quick_two_sum(sum.hi, lo);
}

constexpr double kShortErr = 0x1p-70;  // relative error bound of exp_short, with margin

// log(x) as Lh + Ll within 2^-71 absolute, for normal x with |log x| <= 708:
// one Newton step from the library log y0 (within a few ulp), L = y0 + u -
// u^2/2 with u = x e^-y0 - 1 (|u| < 2^-40), e^-y0 from exp_short.
CR_HD dd log_short(double x)
{
    const double y0 = ::log(x);
    int m = 0;
    const dd E = exp_short({-y0, 0.0}, m);
    const double xs = ::ldexp(x, m);  // x 2^m ~ 1 / E: exact (normal)
    const dd t = two_prod(xs, E.hi);
    const double u0 = sub(t.hi, 1.0);  // exact: t.hi lies within 2^-39 of 1
    const double u = add(u0, add(t.lo, mul(xs, E.lo)));
    return two_sum(y0, sub(u, mul(0.5, mul(u, u))));
}

CR_HD double exp(double x)
{
    if (!(x == x)) return x;
    if (::fabs(x) <= 708.0) {
        int m = 0;
        const dd e = exp_short({x, 0.0}, m);
        if (rounds_to_hi(e.hi, e.lo, mul(kShortErr, e.hi))) return ::ldexp(e.hi, m);
    }
    return exp_long(x);
}

CR_HD double log(double x)
{
    if (!(x > 0.0) || x == INFINITY) return ::log(x);
    if (x >= 0x1p-1020 && x <= 0x1p1020 && x != 1.0) {
        const dd L = log_short(x);
        if (L.hi != 0.0 && rounds_to_hi(::fabs(L.hi), ::fabs(L.hi) == L.hi ? L.lo : -L.lo, 0x1p-71))
            return L.hi;
    }
    return log_long(x);
}

CR_HD double pow(double x, double y)
{
    if (y == 3.0) return round_dd(dd_mul_d(two_prod(x, x), x));
    if (y == 2.0) return mul(x, x);
    if (y == -1.0) return div_(1.0, x);
    if (y == 1.0) return x;
    if (!(x > 0.0) || x == INFINITY || !(y == y) || y == INFINITY || y == -INFINITY) return ::pow(x, y);
    if (x >= 0x1p-1020 && x <= 0x1p1020 && ::fabs(y) <= 16.0) {
        // z = y log x within |y| 2^-71 + 2^-100 |z|; e^z within 2^-72 of itself
        const dd L = log_short(x);
        dd z = two_prod(y, L.hi);
        z.lo = add(z.lo, mul(y, L.lo));
        z = quick_two_sum(z.hi, z.lo);
        if (::fabs(z.hi) <= 708.0) {
            int m = 0;
            const dd e = exp_short(z, m);
            const double err = mul(e.hi, add(kShortErr, mul(add(::fabs(y), 1.0), 0x1p-70)));
            if (rounds_to_hi(e.hi, e.lo, err)) return ::ldexp(e.hi, m);
        }
    }
    return pow_long(x, y);
}

}  // namespace cr
}  // namespace gz

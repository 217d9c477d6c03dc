// gizmo_b200/csrc/physics.cuh -- per-pair and per-particle hydro math, device side.
//
// Templated on the pair arithmetic type T: T = double is the FP64 form
// (compiled without FMA contraction so it rounds like the reference's CPU
// build), T = float the mixed form. Per-particle steps that need FP64 for
// stability (the kernel-length iteration, the NV_T inversion and its
// conditioning loop, flux accumulation) are always double.
//
// Each function cites the reference lines it follows; the operation order
// is kept where it decides a branch.
#pragma once

#include "common.cuh"
#include "crmath.cuh"

namespace gz {

template <typename T> struct Real;
template <> struct Real<double> {
    static GZ_HD double min_real() { return 1e-56; }  // MIN_REAL_NUMBER
    static GZ_HD double sqrt_(double x) { return sqrt(x); }
    static GZ_HD double pow_(double x, double y) { return pow(x, y); }
    // x^y - 1 as the reference writes it (pow, then the subtraction)
    static GZ_HD double powm1_(double x, double y) { return pow(x, y) - 1.0; }
    static GZ_HD bool isnan_(double x) { return isnan(x); }
    // HLLC degenerate-wave tolerance 1e-12 (|S_L| + |S_R| + MIN_REAL), reimann.h:570
    static GZ_HD double hllc_tol(double s) { return 1.e-12 * (s + 1e-56); }
    // kernel support as the reference decides it: on r = sqrt(r2) < h
    static GZ_HD bool inside(double r, double /*r2d*/, double h, double /*hd*/) { return r < h; }
    static GZ_HD double support_r(double r, double /*r2d*/) { return r; }
    static GZ_HD double below_one(double u) { return u; }
    // 1 - u for the kernel polynomials, as the reference computes it
    static GZ_HD double one_minus_u(double u, double /*rd*/, double /*hd*/, double /*hinv*/) { return 1.0 - u; }
};
template <> struct Real<float> {
    // smallest value of the same role that FP32 represents (normal float)
    static GZ_HD float min_real() { return 1e-37f; }
    static GZ_HD float sqrt_(float x) { return sqrtf(x); }
    static GZ_HD float pow_(float x, float y) { return powf(x, y); }
    // x^y - 1 through expm1(y log x): for a near-isothermal gas y = (gamma - 1) / (2 gamma) is
    // tiny and x^y lies within a few FP32 ulps of 1, so pow(x, y) - 1 would keep no significant
    // bit (and the exact solver's Newton iteration would converge on the rounding of it)
    static GZ_HD float powm1_(float x, float y) { return expm1f(y * logf(x)); }
    static GZ_HD bool isnan_(float x) { return isnan(x); }
    // same tolerance, floored at the smallest normal so the all-zero vacuum
    // state (S_L = S_M = S_R = 0) is still trapped instead of dividing 0 by 0
    static GZ_HD float hllc_tol(float s) { return fmaxf(1.e-12f * s, 1e-37f); }
    // kernel support decided exactly as the FP64 form decides it, on the FP64
    // r = sqrt(r2) < h (support_r gives that r once per pair); FP32 rounding of
    // r may reach h there, so u is kept below 1 and a pair inside the support
    // never has both kernel weights zero
    static GZ_HD bool inside(double rd, double /*r2d*/, float, double hd) { return rd < hd; }
    static GZ_HD double support_r(float, double r2d) { return sqrt(r2d); }
    static GZ_HD float below_one(float u) { return u < 1.0f ? u : 0.99999994f; }
    // 1 - u from the FP64 separation and kernel length: near the kernel's edge
    // 1 - u computed in FP32 keeps only the few bits in which u and 1 differ,
    // and the weight (1 - u)^3 of an edge pair would lose as many
    static GZ_HD float one_minus_u(float, double rd, double hd, float hinv) { return float((hd - rd) * (double)hinv); }
};

template <typename T> GZ_HD T dmax(T a, T b) { return (a > b) ? a : b; }  // DMAX, macros.h:219
template <typename T> GZ_HD T dmin(T a, T b) { return (a < b) ? a : b; }  // DMIN, macros.h:220

// Branch guard of the pair arithmetic. The force pair takes discontinuous
// decisions on values it computes (wave-speed and vacuum tests, the pressure
// limits that trigger the Riemann retries, the face-area sign, the HLLC
// degenerate-wave test, the exact solver's sampling, the MFM entropic
// switch). In FP32 a decision whose two sides lie within kFragile of their
// common scale may go the other way than in FP64: Guard<float> records that
// (the pair is then evaluated again in FP64), Guard<double> records nothing
// and compiles away.
constexpr float kFragile = 1.0e-4f;
// Besides the branch decisions, Guard<float> checks precision: a value that
// cancels its own terms (a face state far below the terms it was formed from,
// a star pressure whose numerator cancels, a face area whose two sides
// cancel) carries an FP32 rounding error of 2^-24 x the terms, so it is
// evaluated in FP64 when that error could pass kPrecise relative.
constexpr float kPrecise = 2.0e-6f;

template <typename T> struct Guard;
template <> struct Guard<double> {
    GZ_HD void near(double, double, double, int = 0) {}
    GZ_HD void precise(double, double, int = 0) {}
    GZ_HD void flag(int = 0) {}
    GZ_HD void power(double, int = 0) {}
    GZ_HD int fragile() const { return 0; }
};
// The site numbers name the guarded decisions; built with GZ_GUARD_SITES the
// guard keeps one bit per site (for studying which decisions fire), otherwise
// a single flag.
template <> struct Guard<float> {
#ifdef GZ_GUARD_SITES
    unsigned long long f = 0;
    GZ_HD void set(bool c, int site) { if (c) f |= 1ull << site; }
#else
    int f = 0;
    GZ_HD void set(bool c, int) { f |= (int)c; }
#endif
    // a and b (about to be compared) closer than kFragile x scale; NaN operands count as close
    GZ_HD void near(float a, float b, float scale, int site = 0) { set(!(fabsf(a - b) > kFragile * scale), site); }
    // `value` computed from terms of total magnitude `terms`: too cancelled to hold kPrecise (2^-23 x terms)
    GZ_HD void precise(float value, float terms, int site = 0)
    {
        set(!(fabsf(value) * kPrecise > 1.1920929e-7f * terms), site);
    }
    GZ_HD void flag(int site = 0) { set(true, site); }
    // x^y about to be taken in FP32: its relative error is |y| times that of x (2^-24 from
    // the rounding of x, a few ulps more from the operations that formed it), beyond
    // kPrecise for the large exponents of a near-isothermal gas (2 gamma / (gamma - 1))
    GZ_HD void power(float y, int site = 0) { set(fabsf(y) * 4.0f * 5.9604645e-8f > kPrecise, site); }
    GZ_HD int fragile() const { return f != 0; }
};

// ---------------------------------------------------------------- kernel
// kernel_hinv + kernel_main (mesh/kernel.h:245-438): K=3 cubic, K=6 Wendland C2.
template <typename T> GZ_HD void k_hinv(T h, T &hinv, T &hinv3, T &hinv4)
{
    hinv = T(1.0) / h;
    hinv3 = hinv * hinv * hinv;
    hinv4 = hinv3 * hinv;
}

// k_main_t takes t1 = 1 - u from the caller (Real<T>::one_minus_u); k_main
// computes it as the reference does. u - 1 of the inner cubic branch is -t1
// exactly.
template <typename T> GZ_HD void k_main_t(int kf, T u, T t1, T hinv3, T hinv4, T &wk, T &dwk)
{
    if (u >= T(1)) { wk = T(0); dwk = T(0); return; }
    T w, dw;
    if (kf == 3) {
        if (u < T(0.5)) {
            dw = u * (T(18.0) * u - T(12.0));
            w = (T(1.0) + T(6.0) * (-t1) * u * u);
        } else {
            T t2 = t1 * t1;
            dw = T(-6.0) * t2;
            w = T(2.0) * t2 * t1;
        }
        dwk = dw * (T(8.0 / 3.14159265358979323846) * hinv4);
        wk = w * (T(8.0 / 3.14159265358979323846) * hinv3);
    } else {
        T t3 = t1 * t1 * t1;
        dw = T(-20.0) * u * t3;
        w = t3 * t1 * (T(1.0) + T(4.0) * u);
        dwk = dw * (T(21.0 / (2.0 * 3.14159265358979323846)) * hinv4);
        wk = w * (T(21.0 / (2.0 * 3.14159265358979323846)) * hinv3);
    }
}

template <typename T> GZ_HD void k_main(int kf, T u, T hinv3, T hinv4, T &wk, T &dwk)
{
    k_main_t(kf, u, T(1) - u, hinv3, hinv4, wk, dwk);
}

// ------------------------------------------------------------ 3x3 inverse
// Mat3::invert (math_types/mat3.h:50-63) + matrix_invert_ndims (core/proto.h:75-95).
GZ_HD double invert3(const double T[3][3], double Ti[3][3])
{
    double fro = (T[0][0] * T[0][0] + T[0][1] * T[0][1] + T[0][2] * T[0][2]) +
                 (T[1][0] * T[1][0] + T[1][1] * T[1][1] + T[1][2] * T[1][2]) +
                 (T[2][0] * T[2][0] + T[2][1] * T[2][1] + T[2][2] * T[2][2]);
    for (int a = 0; a < 3; a++)
        for (int b = 0; b < 3; b++) Ti[a][b] = 0;
    double d = T[0][0] * (T[1][1] * T[2][2] - T[1][2] * T[2][1]) - T[0][1] * (T[1][0] * T[2][2] - T[1][2] * T[2][0]) +
               T[0][2] * (T[1][0] * T[2][1] - T[1][1] * T[2][0]);
    if (!(d == 0 || d != d)) {
        double id = 1.0 / d;
        Ti[0][0] = (T[1][1] * T[2][2] - T[1][2] * T[2][1]) * id;
        Ti[0][1] = (T[0][2] * T[2][1] - T[0][1] * T[2][2]) * id;
        Ti[0][2] = (T[0][1] * T[1][2] - T[0][2] * T[1][1]) * id;
        Ti[1][0] = (T[1][2] * T[2][0] - T[1][0] * T[2][2]) * id;
        Ti[1][1] = (T[0][0] * T[2][2] - T[0][2] * T[2][0]) * id;
        Ti[1][2] = (T[0][2] * T[1][0] - T[0][0] * T[1][2]) * id;
        Ti[2][0] = (T[1][0] * T[2][1] - T[1][1] * T[2][0]) * id;
        Ti[2][1] = (T[0][1] * T[2][0] - T[0][0] * T[2][1]) * id;
        Ti[2][2] = (T[0][0] * T[1][1] - T[0][1] * T[1][0]) * id;
    }
    double froi = (Ti[0][0] * Ti[0][0] + Ti[0][1] * Ti[0][1] + Ti[0][2] * Ti[0][2]) +
                  (Ti[1][0] * Ti[1][0] + Ti[1][1] * Ti[1][1] + Ti[1][2] * Ti[1][2]) +
                  (Ti[2][0] * Ti[2][0] + Ti[2][1] * Ti[2][1] + Ti[2][2] * Ti[2][2]);
    return dmax(sqrt(fro * froi) / 3, 1.0);
}

// NV_T inversion with conditioning + face-closure error
// (density_loop.h:572-637; density_loop.cc:444-504). acc: raw sums.
GZ_HD void nvt_invert(double h, double NumNgb, const double *acc_nvt, const double *acc_face, double &CN,
                       double Tn[3][3], double &fce)
{
    const double V_i = kVolNorm * cr::pow(h, 3.0) / (NumNgb > 0 ? NumNgb : 1.0);
    const double norm = cr::pow(h, -1.0);
    double raw[3][3], T[3][3], Tinv[3][3];
    raw[0][0] = acc_nvt[0]; raw[1][1] = acc_nvt[1]; raw[2][2] = acc_nvt[2];
    raw[0][1] = raw[1][0] = acc_nvt[3];
    raw[1][2] = raw[2][1] = acc_nvt[4];
    raw[0][2] = raw[2][0] = acc_nvt[5];
    for (int a = 0; a < 3; a++)
        for (int b = 0; b < 3; b++) T[a][b] = raw[a][b] / norm;
    const double thr = 10.0 * kCnDanger;
    const double tr0 = T[0][0] + T[1][1] + T[2][2];
    double add = 1.05 * (tr0 / 3) / thr;
    for (int guard = 0; guard < 4096; guard++) {
        CN = invert3(T, Tinv);
        if (CN < thr) break;
        for (int k = 0; k < 3; k++) T[k][k] += add;
        add *= 1.2;
    }
    const double tr_raw = raw[0][0] + raw[1][1] + raw[2][2];
    const double dx_i = sqrt(V_i * tr_raw);
    for (int a = 0; a < 3; a++)
        for (int b = 0; b < 3; b++) Tn[a][b] = Tinv[a][b] / norm;
    double fo[3] = {0, 0, 0};
    for (int a = 0; a < 3; a++)
        for (int b = 0; b < 3; b++) fo[a] += 2.0 * V_i * Tn[a][b] * acc_face[b];
    double leak = 0;
    for (int a = 0; a < 3; a++) leak += fabs(fo[a]) / 3.0;
    fce = leak / (2.0 * 3.0 * cr::pow(dx_i, 2.0));
}

// ------------------------------------------------------- density after_iter
struct DensityScratch {
    double left, right, cn_cur;
    int cn_init;
    int pad;
};

struct PassParams {
    int kernel, method, first_step, selfgravity_off;
    double box, half, gamma, des_num_ngb, max_num_ngb_dev, min_kernel_radius, max_kernel_radius;
    int diag_flux_abs;  // the force pass also sums |pair flux| per row (a diagnostic)
};

// DensitySpec::after_iter_body for gas (density_loop.h:515-961). acc[14]:
// Ngb Rho DrkernNgb DivVel NVT(6) face(3) -. Returns 1 when converged.
GZ_HD int after_iter(const PassParams &p, int iter, double h, const double *acc, double cond_prev, DensityScratch &sc,
                      double &new_h_out, int &stop)
{
    double desnumngb = p.des_num_ngb;
    double desnumngbdev = p.max_num_ngb_dev;
    if (p.first_step) { if (p.max_num_ngb_dev > 0.05) desnumngbdev = 0.05; }
    const double desnumngbdev_0 = desnumngbdev;
    double NumNgb = acc[0], Drk = acc[2];
    if (NumNgb > 0) {
        Drk *= h / (3 * NumNgb);
        NumNgb *= kVolNorm * cr::pow(h, 3.0);
    } else { NumNgb = 0; Drk = 0; }
    if (Drk > -0.9) Drk = 1.0 / (1.0 + Drk); else Drk = 1.0;
    double CN, fce, Tn[3][3];
    nvt_invert(h, NumNgb, acc + 4, acc + 10, CN, Tn, fce);
    const double c0 = 0.1 * kCnDanger;
    if ((iter == 0) && (CN > cond_prev) && (cond_prev > 0)) {
        double ncorr_a = 1.0, cn_a = cond_prev;
        if (cn_a > c0) ncorr_a = sqrt(1.0 + (cn_a - c0) / kCnDanger);
        if (ncorr_a > 2.0) ncorr_a = 2.0;
        const double dn_ngb = fabs(NumNgb - p.des_num_ngb * ncorr_a) / (desnumngbdev_0 * ncorr_a);
        double ncorr_b = 1.0, cn_b = CN;
        if (cn_b > c0) ncorr_b = sqrt(1.0 + (cn_b - c0) / kCnDanger);
        if (ncorr_b > 2.0) ncorr_b = 2.0;
        const double dn_ngb_alt = fabs(NumNgb - p.des_num_ngb * ncorr_b) / (desnumngbdev_0 * ncorr_b);
        if (dmin(dn_ngb, dn_ngb_alt) < 10.0) { sc.cn_cur = CN; sc.cn_init = 1; }
    }
    if (!sc.cn_init) { sc.cn_cur = cond_prev; sc.cn_init = 1; }
    double ncorr = 1.0;
    {
        const double cn = sc.cn_cur;
        if (cn > c0) ncorr = sqrt(1.0 + (cn - c0) / kCnDanger);
        if (ncorr > 2.0) ncorr = 2.0;
        const double d00 = 0.35;
        if (fce > d00) ncorr = dmax(ncorr, dmin(fce / d00, 2.0));
    }
    desnumngb = p.des_num_ngb * ncorr;
    desnumngbdev = desnumngbdev_0 * ncorr;
    if (iter > 1)
        desnumngbdev = dmin(0.25 * desnumngb, desnumngbdev * cr::exp(0.1 * cr::log(desnumngb / (16.0 * desnumngbdev)) * (double)iter));
    const double minsoft = p.min_kernel_radius, maxsoft = p.max_kernel_radius;
    int redo = 0, setmin = 0, setmax = 0;
    double new_h = h;
    if ((NumNgb < (desnumngb - desnumngbdev) && new_h < 0.999 * maxsoft) ||
        (NumNgb > (desnumngb + desnumngbdev) && new_h > 1.001 * minsoft))
        redo = 1;
    if ((new_h >= 0.999 * maxsoft) && (NumNgb < (desnumngb - desnumngbdev))) {
        redo = 0;
        if (new_h == maxsoft) setmax = 0; else { redo = 1; new_h = maxsoft; setmax = 1; }
    }
    if ((new_h <= 1.001 * minsoft) && (NumNgb > (desnumngb + desnumngbdev))) {
        redo = 0;
        if (new_h == minsoft) setmin = 0; else { redo = 1; new_h = minsoft; setmin = 1; }
    }
    if (redo == 0) sc.cn_cur = CN;
    if (redo) {
        if (sc.left > 0 && sc.right > 0) {
            if ((sc.right - sc.left) < 1.0e-3 * sc.left) { sc.cn_cur = CN; new_h_out = new_h; return 1; }
        }
        if (setmax == 0 && setmin == 0) {
            if (NumNgb < (desnumngb - desnumngbdev)) {
                sc.left = dmax(new_h, sc.left);
            } else {
                if (sc.right != 0) { if (new_h < sc.right) sc.right = new_h; }
                else sc.right = new_h;
            }
            if (sc.right > 0 && sc.left > 0) {
                double maxjump = 0;
                if (iter > 1) maxjump = 0.2 * cr::log(sc.right / sc.left);
                if (NumNgb > 1) {
                    double jumpvar = Drk * cr::log(desnumngb / NumNgb) / 3;
                    if (iter > 1) { if (fabs(jumpvar) < maxjump) { if (jumpvar < 0) jumpvar = -maxjump; else jumpvar = maxjump; } }
                    new_h *= cr::exp(jumpvar);
                } else {
                    new_h *= 2.0;
                }
                if ((new_h < sc.right) && (new_h > sc.left)) {
                    if (iter > 1) {
                        const double hfac = cr::exp(maxjump);
                        if (new_h > sc.right / hfac) new_h = sc.right / hfac;
                        if (new_h < sc.left * hfac) new_h = sc.left * hfac;
                    }
                } else {
                    if (new_h > sc.right) new_h = sc.right;
                    if (new_h < sc.left) new_h = sc.left;
                    new_h = cr::pow(new_h * sc.left * sc.right, 1.0 / 3.0);
                }
            } else {
                if (sc.right == 0 && sc.left == 0) { stop = 90001009; new_h_out = new_h; return 1; }
                if (sc.right == 0 && sc.left > 0) {
                    double fac_lim = (NumNgb > 1) ? cr::log(desnumngb / NumNgb) / 3 : 1.4;
                    if ((NumNgb < 2.0 * desnumngb) && (NumNgb > 0.1 * desnumngb)) {
                        double slope = Drk;
                        if (iter > 2 && slope < 1.0) slope = 0.5 * (slope + 1.0);
                        double fac = fac_lim * slope;
                        if (iter >= 4) { if (Drk == 1.0) fac *= 10.0; }
                        if (fac < fac_lim + 0.231) new_h *= cr::exp(fac); else new_h *= cr::exp(fac_lim + 0.231);
                    } else {
                        new_h *= cr::exp(fac_lim);
                    }
                }
                if (sc.right > 0 && sc.left == 0) {
                    double fac_lim = (NumNgb > 1) ? cr::log(desnumngb / NumNgb) / 3 : 1.4;
                    if (fac_lim < -1.535) fac_lim = -1.535;
                    if ((NumNgb < 2.0 * desnumngb) && (NumNgb > 0.1 * desnumngb)) {
                        double slope = Drk;
                        if (iter > 2 && slope < 1.0) slope = 0.5 * (slope + 1.0);
                        double fac = fac_lim * slope;
                        if (iter >= 4) { if (Drk == 1.0) fac *= 10.0; }
                        if (fac > fac_lim - 0.231) new_h *= cr::exp(fac); else new_h *= cr::exp(fac_lim - 0.231);
                    } else {
                        new_h *= cr::exp(fac_lim);
                    }
                }
            }
        }
        if (new_h < minsoft) new_h = minsoft;
        if (setmin == 1) new_h = minsoft;
        if (new_h > maxsoft) new_h = maxsoft;
        if (setmax == 1) new_h = maxsoft;
        new_h_out = new_h;
        return 0;
    }
    sc.cn_cur = CN;
    new_h_out = new_h;
    return 1;
}

// ---------------------------------------------------------- gradients
// local_slopelimiter, Newtonian branch (gradients_loop.cc:76-104).
GZ_HD void slopelimiter(double *g, double valmax, double valmin, double alim, double h, double shoot_tol,
                         int pos_preserve, double d_max, double val_cen)
{
    double d_abs = g[0] * g[0] + g[1] * g[1] + g[2] * g[2];
    if (d_abs > 0) {
        d_abs = sqrt(d_abs);
        double cfac = 1 / (alim * h * d_abs);
        double fabs_max = fabs(valmax), fabs_min = fabs(valmin), abs_max = fabs_max, abs_min = fabs_min, f;
        if (abs_max < abs_min) { abs_max = fabs_min; abs_min = fabs_max; }
        f = dmin(abs_min + shoot_tol * abs_max, abs_max);
        cfac *= f;
        if (pos_preserve == 1) {
            double fmin_ = dmin(val_cen, dmax(0.0, dmax(kMinReal * val_cen, dmin(0.5 * (val_cen + valmin), val_cen - f))));
            cfac = dmin(((val_cen - fmin_) / d_max) / d_abs, cfac);
        }
        if (cfac < 1) { g[0] *= cfac; g[1] *= cfac; g[2] *= cfac; }
    }
}

template <typename T> GZ_HD void sym_matvec(const T *s, const T *v, T *o)
{  // SymmetricTensor2::matvec (symmetric_tensor2.h:80-84)
    const T a = s[0] * v[0] + s[3] * v[1] + s[5] * v[2];
    const T b = s[3] * v[0] + s[1] * v[1] + s[4] * v[2];
    const T c = s[5] * v[0] + s[4] * v[1] + s[2] * v[2];
    o[0] = a; o[1] = b; o[2] = c;
}

// ------------------------------------------------------------- Riemann
template <typename T> struct Crv { T rho, p, v[3], u, cs; };
template <typename T> struct RVec { Crv<T> L, R; };
template <typename T> struct ROut { T P_M, S_M; Crv<T> F; };
template <typename T> struct GConst { T G0, G1, G2, G3, G4, G5, G6, G7, G8, G9; int mfv; };

template <typename T> GZ_HD T dot3(const T *a, const T *b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }
template <typename T> GZ_HD T nsq3(const T *a) { return a[0] * a[0] + a[1] * a[1] + a[2] * a[2]; }

// get_wavespeeds_and_pressure_star (reimann.h:485-549)
template <typename T>
GZ_HD void wavespeeds(const RVec<T> &rv, ROut<T> &o, const T *n, T vL, T vR, T cL, T cR, T hL, T hR, T &SLo, T &SRo,
                       T ptl, const GConst<T> &gc, Guard<T> &g)
{
    const T MR = Real<T>::min_real();
    T S_L, S_R;
    g.near(vR - vL, dmax(cL, cR), fabs(vL) + fabs(vR) + dmax(cL, cR), 1);  // the vacuum test
    if ((vR - vL) > dmax(cL, cR)) {
        o.P_M = MR; o.S_M = S_L = S_R = T(0);
    } else {
        const T PT_L = rv.L.p, PT_R = rv.R.p;
        const T pscale = fabs(PT_L) + fabs(PT_R);
        S_L = dmin(vL, vR) - dmax(cL, cR);
        S_R = dmax(vL, vR) + dmax(cL, cR);
        T rho_wt_L = rv.L.rho * (S_L - vL);
        T rho_wt_R = rv.R.rho * (S_R - vR);
        o.S_M = ((PT_R - PT_L) + rho_wt_L * vL - rho_wt_R * vR) / (rho_wt_L - rho_wt_R);
        o.P_M = (PT_L * rho_wt_R - PT_R * rho_wt_L + rho_wt_L * rho_wt_R * (vR - vL)) / (rho_wt_R - rho_wt_L);
        // the star pressure's sign (the clamp at MIN_REAL zeroes the wave speeds), on the scale
        // of the terms its numerator cancels (rho_wt_L < 0 < rho_wt_R: the denominator cannot)
        g.precise(PT_L * rho_wt_R - PT_R * rho_wt_L + rho_wt_L * rho_wt_R * (vR - vL),
                  fabs(PT_L * rho_wt_R) + fabs(PT_R * rho_wt_L) + fabs(rho_wt_L * rho_wt_R * (vR - vL)), 3);
        g.near(o.P_M, ptl, ptl, 4);
        if (o.P_M <= MR) { o.P_M = MR; o.S_M = S_L = S_R = T(0); }
        if ((o.P_M <= T(0)) || Real<T>::isnan_(o.P_M) || (o.P_M > ptl)) {
            const T sL = Real<T>::sqrt_(rv.L.rho), sR = Real<T>::sqrt_(rv.R.rho);
            const T sinv = T(1) / (sL + sR);
            T v_roe[3];
            for (int k = 0; k < 3; k++) v_roe[k] = (rv.L.v[k] * sL + rv.R.v[k] * sR) * sinv;
            const T v_line_roe = dot3(v_roe, n);
            const T h_roe = (sL * hL + sR * hR) * sinv;
            const T cs_roe = Real<T>::sqrt_(dmax(T(1.e-30), gc.G9 * (h_roe - T(0.5) * nsq3(v_roe))));
            S_R = dmax(vR + cR, v_line_roe + cs_roe);
            S_L = dmin(vL - cL, v_line_roe - cs_roe);
            rho_wt_R = rv.R.rho * (S_R - vR);
            rho_wt_L = -rv.L.rho * (S_L - vL);
            o.S_M = ((rho_wt_R * vR + rho_wt_L * vL) + (PT_L - PT_R)) / (rho_wt_R + rho_wt_L);
            o.P_M = rv.L.rho * (vL - S_L) * (vL - o.S_M) + PT_L;
            g.near(o.P_M, T(0), pscale + fabs(rv.L.rho * (vL - S_L) * (vL - o.S_M)), 6);
            g.near(o.P_M, ptl, ptl, 7);
            if (o.P_M <= MR) { o.P_M = MR; o.S_M = S_L = S_R = T(0); }
            if ((o.P_M <= T(0)) || Real<T>::isnan_(o.P_M) || (o.P_M > ptl)) {
                o.P_M = T(0.5) * ((PT_L + PT_R) + (vL - vR) * T(0.25) * (rv.L.rho + rv.R.rho) * (cL + cR));
                o.S_M = T(0.5) * (vR + vL) + T(2.0) * (PT_L - PT_R) / ((rv.L.rho + rv.R.rho) * (cL + cR));
                const T S_plus = dmax(dmax(fabs(vL - cL), fabs(vR - cR)), dmax(fabs(vL + cL), fabs(vR + cR)));
                S_L = -S_plus; S_R = S_plus;
                if (o.S_M < S_L) o.S_M = S_L;
                if (o.S_M > S_R) o.S_M = S_R;
                g.near(o.P_M, T(0), pscale + fabs((vL - vR) * T(0.25) * (rv.L.rho + rv.R.rho) * (cL + cR)), 8);
                if (o.P_M <= MR) { o.P_M = MR; o.S_M = S_L = S_R = T(0); }
            }
        }
    }
    SLo = S_L;
    SRo = S_R;
}

// HLLC_fluxes, MFV, face frame (reimann.h:559-615)
template <typename T>
GZ_HD void hllc_fluxes(const RVec<T> &rv, ROut<T> &o, const T *n, T vL, T vR, T hL, T hR, T S_L, T S_R, Guard<T> &g)
{
    const T P_M = o.P_M, S_M = o.S_M;
    if ((P_M <= T(0)) || Real<T>::isnan_(P_M)) return;
    T nfac, eK, dv2, vf = T(0);
    {
        // the FP64 tolerance is 1e-12 of the wave speeds: in FP32 a contact this close to an outer
        // wave (where nfac divides by S_L - S_M or S_R - S_M) is decided in FP64; wave speeds all
        // zeroed by the vacuum or star-pressure clamps take the degenerate flux in both forms
        if (fabs(S_L) + fabs(S_R) > T(0)) {
            g.near(S_M, S_L, fabs(S_L) + fabs(S_R), 9);
            g.near(S_M, S_R, fabs(S_L) + fabs(S_R), 10);
        }
        const T tol_s = Real<T>::hllc_tol(fabs(S_L) + fabs(S_R));
        if ((fabs(S_M - S_L) < tol_s) || (fabs(S_M - S_R) < tol_s) || (fabs(S_M - vf) < tol_s)) {
            o.F.rho = T(0);
            o.F.p = o.P_M * o.S_M;
            for (int k = 0; k < 3; k++) o.F.v[k] = n[k] * o.P_M;
            return;
        }
    }
    if (vf < S_L) {
        o.F.rho = rv.L.rho * (vL - vf);
        o.F.p = rv.L.rho * hL * (vL - vf) + rv.L.p * vf;
        for (int k = 0; k < 3; k++) o.F.v[k] = rv.L.v[k] * o.F.rho + n[k] * rv.L.p;
    } else if ((S_L <= vf) && (vf <= S_M)) {
        nfac = rv.L.rho * (S_L - vL) / (S_L - S_M);
        if (nfac < T(0)) nfac = T(0);
        o.F.rho = rv.L.rho * (vL - S_L) + nfac * (S_L - vf);
        eK = rv.L.rho * hL - rv.L.p;
        o.F.p = (rv.L.rho * hL * vL - eK * S_L) +
                (S_L - vf) * nfac * (eK / rv.L.rho + (S_M - vL) * (S_M + rv.L.p / (rv.L.rho * (S_L - vL))));
        dv2 = nfac * (S_L - vf) * (S_M - vL) + rv.L.p;
        for (int k = 0; k < 3; k++) o.F.v[k] = rv.L.v[k] * o.F.rho + n[k] * dv2;
    } else if ((S_M <= vf) && (vf <= S_R)) {
        nfac = rv.R.rho * (S_R - vR) / (S_R - S_M);
        if (nfac < T(0)) nfac = T(0);
        o.F.rho = rv.R.rho * (vR - S_R) + nfac * (S_R - vf);
        eK = rv.R.rho * hR - rv.R.p;
        o.F.p = (rv.R.rho * hR * vR - eK * S_R) +
                (S_R - vf) * nfac * (eK / rv.R.rho + (S_M - vR) * (S_M + rv.R.p / (rv.R.rho * (S_R - vR))));
        dv2 = nfac * (S_R - vf) * (S_M - vR) + rv.R.p;
        for (int k = 0; k < 3; k++) o.F.v[k] = rv.R.v[k] * o.F.rho + n[k] * dv2;
    } else {
        o.F.rho = rv.R.rho * (vR - vf);
        o.F.p = rv.R.rho * hR * (vR - vf) + rv.R.p * vf;
        for (int k = 0; k < 3; k++) o.F.v[k] = rv.R.v[k] * o.F.rho + n[k] * rv.R.p;
    }
}

// Riemann_solver_KurganovTadmor_PWK (reimann.h:445-477), SLOPE_LIMITER_TOLERANCE 1
template <typename T>
GZ_HD void riemann_kt(const RVec<T> &rv, ROut<T> &o, const T *n, T vL, T vR, T cL, T cR, T hL, T hR,
                       const GConst<T> &gc)
{
    T S_L, S_R, S_M, alpha;
    const T delta_threshold = T(0.001) * T(0.5) * (rv.L.rho + rv.R.rho) * T(0.5) * (cL + cR);
    T dv[3];
    for (int k = 0; k < 3; k++) dv[k] = rv.R.v[k] * rv.R.rho - rv.L.v[k] * rv.L.rho;
    const T dv2 = nsq3(dv);
    const T dvL = fabs(rv.R.rho * vR - rv.L.rho * vL);
    alpha = dvL / Real<T>::sqrt_(delta_threshold * delta_threshold + dv2);
    S_L = alpha * cL; if (vL > T(0)) S_L += vL; else S_L -= vL;
    S_R = alpha * cR; if (vR > T(0)) S_R += vR; else S_R -= vR;
    S_M = dmax(S_L, S_R);
    o.S_M = dmax(cL + fabs(vL), cR + fabs(vR));
    const T f_rho_left = rv.L.rho * (vL + S_M);
    const T f_rho_right = rv.R.rho * (vR - S_M);
    if (gc.mfv) {
        o.P_M = T(0.5) * (rv.R.p + rv.L.p);
        o.F.rho = T(0.5) * (f_rho_left + f_rho_right);
        for (int k = 0; k < 3; k++) o.F.v[k] = T(0.5) * (rv.L.v[k] * f_rho_left + rv.R.v[k] * f_rho_right) + n[k] * o.P_M;
        o.F.p = T(0.5) * (f_rho_left * hL + f_rho_right * hR + S_M * (rv.R.p - rv.L.p));
    } else {
        const T denom = T(1) / (rv.L.rho * vL - rv.R.rho * vR + S_M * (rv.L.rho + rv.R.rho));
        o.P_M = (f_rho_left * rv.R.p - f_rho_right * rv.L.p) * denom;
        o.F.rho = T(0);
        for (int k = 0; k < 3; k++) o.F.v[k] = (rv.R.v[k] - rv.L.v[k]) * (f_rho_left * f_rho_right * denom) + n[k] * o.P_M;
        o.F.p = (S_M * (f_rho_left * rv.R.p + f_rho_right * rv.L.p) + (hR - hL) * f_rho_left * f_rho_right) * denom;
    }
}

// guess_for_pressure (reimann.h:1025-1062)
template <typename T>
GZ_HD T guess_pressure(const RVec<T> &rv, T vL, T vR, T cL, T cR, const GConst<T> &gc)
{
    const T pv = T(0.5) * (rv.L.p + rv.R.p) - T(0.125) * (vR - vL) * (rv.L.p + rv.R.p) * (cL + cR);
    const T pmin = dmin(rv.L.p, rv.R.p), pmax = dmax(rv.L.p, rv.R.p);
    if (pmin <= T(0)) return T(0.5) * (pmin + pmax);
    const T qrat = pmax / pmin;
    if (qrat <= T(2.0) && (pmin <= pv && pv <= pmax)) return pv;
    if (pv < pmin) {
        const T pnu = (cL + cR) - gc.G7 * (vR - vL);
        const T pde = cL / Real<T>::pow_(rv.L.p, gc.G1) + cR / Real<T>::pow_(rv.R.p, gc.G1);
        return Real<T>::pow_(pnu / pde, gc.G3);
    }
    const T gel = Real<T>::sqrt_((gc.G5 / rv.L.rho) / (gc.G6 * rv.L.p + pv));
    const T ger = Real<T>::sqrt_((gc.G5 / rv.R.rho) / (gc.G6 * rv.R.p + pv));
    T x = (gel * rv.L.p + ger * rv.R.p - (vR - vL)) / (gel + ger);
    if (x < pmin || x > pmax) x = pmin;
    return x;
}

// iterative_Riemann_solver (reimann.h:965-1020), NMAX_ITER 1000, TOL_ITER 1e-6
template <typename T>
GZ_HD int riemann_iterative(const RVec<T> &rv, ROut<T> &o, T vL, T vR, T cL, T cR, const GConst<T> &gc, Guard<T> &g)
{
    T Pg, Pg_prev, W_L = T(0), W_R = T(0), Z_L, Z_R, tol, pratio;
    int niter = 0;
    const T dvel = vR - vL;
    const T check_vel = gc.G4 * (cR + cL) - dvel;
    g.near(gc.G4 * (cR + cL), dvel, gc.G4 * (cR + cL) + fabs(vL) + fabs(vR), 11);  // vacuum generation
    if (check_vel < T(0)) return 0;
    tol = T(100.0);
    Pg = guess_pressure(rv, vL, vR, cL, cR, gc);
    while ((tol > T(1.e-6)) && (niter < 1000)) {
        Pg_prev = Pg;
        if (Pg > rv.L.p) {
            const T a0 = gc.G5 / rv.L.rho, a1 = gc.G6 * rv.L.p, a2 = Real<T>::sqrt_(a0 / (Pg + a1));
            W_L = (Pg - rv.L.p) * a2;
            Z_L = a2 * (T(1.0) - T(0.5) * (Pg - rv.L.p) / (a1 + Pg));
        } else {
            pratio = Pg / rv.L.p;
            W_L = gc.G4 * cL * Real<T>::powm1_(pratio, gc.G1);
            Z_L = T(1) / (rv.L.rho * cL) * Real<T>::pow_(Pg / rv.L.p, -gc.G2);
        }
        if (Pg > rv.R.p) {
            const T a0 = gc.G5 / rv.R.rho, a1 = gc.G6 * rv.R.p, a2 = Real<T>::sqrt_(a0 / (Pg + a1));
            W_R = (Pg - rv.R.p) * a2;
            Z_R = a2 * (T(1.0) - T(0.5) * (Pg - rv.R.p) / (a1 + Pg));
        } else {
            pratio = Pg / rv.R.p;
            W_R = gc.G4 * cR * Real<T>::powm1_(pratio, gc.G1);
            Z_R = T(1) / (rv.R.rho * cR) * Real<T>::pow_(pratio, -gc.G2);
        }
        if (niter < 1000 / 2) Pg -= (W_L + W_R + dvel) / (Z_L + Z_R);
        else Pg -= T(0.5) * (W_L + W_R + dvel) / (Z_L + Z_R);
        if (Pg < T(0.1) * Pg_prev) Pg = T(0.1) * Pg_prev;
        tol = T(2.0) * fabs((Pg - Pg_prev) / (Pg + Pg_prev));
        niter++;
    }
    if (niter < 1000) {
        o.P_M = Pg;
        o.S_M = T(0.5) * (vL + vR) + T(0.5) * (W_R - W_L);
        return 1;
    }
    g.flag(12);  // no convergence: the vacuum sampling follows; decided in FP64
    return 0;
}

// vacuum / fan sampling at S = 0 (reimann.h:672-840)
template <typename T>
GZ_HD void sample_vac_left(const RVec<T> &rv, ROut<T> &o, const T *n, T vR, T cR, const GConst<T> &gc)
{
    const T S = T(0), S_R = vR - gc.G4 * cR;
    if (!gc.mfv) { o.P_M = T(0); o.S_M = S_R; return; }
    if (S_R > S) { o.P_M = T(0); o.S_M = S_R; o.F.rho = T(0); }
    else {
        if (vR + cR > S) {
            const T C_eff = gc.G5 * (cR - gc.G7 * (vR - S));
            o.P_M = rv.R.p * Real<T>::pow_(C_eff / cR, gc.G3);
            o.S_M = gc.G5 * (-cR + gc.G7 * vR + S);
            o.F.rho = rv.R.rho * Real<T>::pow_(C_eff / cR, gc.G4);
        } else { o.P_M = rv.R.p; o.S_M = vR; o.F.rho = rv.R.rho; }
    }
    o.F.p = o.P_M;
    for (int k = 0; k < 3; k++) o.F.v[k] = rv.R.v[k] + n[k] * (o.S_M - vR);
}

template <typename T>
GZ_HD void sample_vac_right(const RVec<T> &rv, ROut<T> &o, const T *n, T vL, T cL, const GConst<T> &gc)
{
    const T S = T(0), S_L = vL + gc.G4 * cL;
    if (!gc.mfv) { o.P_M = T(0); o.S_M = S_L; return; }
    if (S_L < S) { o.P_M = T(0); o.S_M = S_L; o.F.rho = T(0); }
    else {
        if (vL - cL < S) {
            const T C_eff = gc.G5 * (cL + gc.G7 * (vL - S));
            o.P_M = rv.L.p * Real<T>::pow_(C_eff / cL, gc.G3);
            o.S_M = gc.G5 * (cL + gc.G7 * vL + S);
            o.F.rho = rv.L.rho * Real<T>::pow_(C_eff / cL, gc.G4);
        } else { o.P_M = rv.L.p; o.S_M = vL; o.F.rho = rv.L.rho; }
    }
    o.F.p = o.P_M;
    for (int k = 0; k < 3; k++) o.F.v[k] = rv.L.v[k] + n[k] * (o.S_M - vL);
}

template <typename T>
GZ_HD void sample_vac_internal(const RVec<T> &rv, ROut<T> &o, const T *n, T vL, T vR, T cL, T cR, const GConst<T> &gc)
{
    const T S = T(0), S_L = vL + gc.G4 * cL, S_R = vR - gc.G4 * cR;
    if (S <= S_L) sample_vac_right(rv, o, n, vL, cL, gc);
    else if (S >= S_R) sample_vac_left(rv, o, n, vR, cR, gc);
    else {
        o.P_M = T(0);
        o.S_M = S;
        if (gc.mfv) {
            o.F.rho = T(0);
            o.F.p = o.P_M;
            for (int k = 0; k < 3; k++)
                o.F.v[k] = (rv.L.v[k] + (rv.R.v[k] - rv.L.v[k]) * (S - S_L) / (S_R - S_L)) * (T(1) - n[k]) + S * n[k];
        }
    }
}

// The sampled face state jumps across the contact (S_M = 0) and across a shock
// (S_L or S_R = 0): those signs are guarded; at the edges of a rarefaction fan
// the state is continuous.
template <typename T>
GZ_HD void sample_standard(const RVec<T> &rv, ROut<T> &o, const T *n, T vL, T vR, T cL, T cR, const GConst<T> &gc,
                            Guard<T> &g)
{
    if (!gc.mfv) return;
    const T S = T(0);
    T C_eff, S_eff;
    const T sscale = fabs(vL) + fabs(vR) + cL + cR;
    g.near(o.S_M, S, sscale, 13);
    if (S <= o.S_M) {
        if (o.P_M <= rv.L.p) {
            if (S <= vL - cL) { o.F.p = rv.L.p; o.F.rho = rv.L.rho; for (int k = 0; k < 3; k++) o.F.v[k] = rv.L.v[k]; return; }
            const T C_eff_L = cL * Real<T>::pow_(o.P_M / rv.L.p, gc.G1);
            if (S > o.S_M - C_eff_L) {
                o.F.rho = rv.L.rho * Real<T>::pow_(o.P_M / rv.L.p, gc.G8);
                o.F.p = o.P_M;
                for (int k = 0; k < 3; k++) o.F.v[k] = rv.L.v[k] + n[k] * (o.S_M - vL);
                return;
            }
            S_eff = gc.G5 * (cL + gc.G7 * vL + S);
            C_eff = gc.G5 * (cL + gc.G7 * (vL - S));
            g.power(gc.G3, 17);  // inside the left fan
            o.F.rho = rv.L.rho * Real<T>::pow_(C_eff / cL, gc.G4);
            o.F.p = rv.L.p * Real<T>::pow_(C_eff / cL, gc.G3);
            for (int k = 0; k < 3; k++) o.F.v[k] = rv.L.v[k] + n[k] * (S_eff - vL);
            return;
        }
        if (rv.L.p > T(0)) {
            const T pml = o.P_M / rv.L.p;
            const T S_L = vL - cL * Real<T>::sqrt_(gc.G2 * pml + gc.G1);
            g.near(S_L, S, sscale, 14);
            if (S <= S_L) { o.F.p = rv.L.p; o.F.rho = rv.L.rho; for (int k = 0; k < 3; k++) o.F.v[k] = rv.L.v[k]; return; }
            o.F.rho = rv.L.rho * (pml + gc.G6) / (pml * gc.G6 + T(1.0));
            o.F.p = o.P_M;
            for (int k = 0; k < 3; k++) o.F.v[k] = rv.L.v[k] + n[k] * (o.S_M - vL);
            return;
        }
        o.F.rho = rv.L.rho / gc.G6;
        o.F.p = o.P_M;
        for (int k = 0; k < 3; k++) o.F.v[k] = rv.L.v[k] + n[k] * (o.S_M - vL);
        return;
    }
    if (o.P_M > rv.R.p) {
        if (rv.R.p > T(0)) {
            const T pmr = o.P_M / rv.R.p;
            const T S_R = vR + cR * Real<T>::sqrt_(gc.G2 * pmr + gc.G1);
            g.near(S_R, S, sscale, 15);
            if (S >= S_R) { o.F.p = rv.R.p; o.F.rho = rv.R.rho; for (int k = 0; k < 3; k++) o.F.v[k] = rv.R.v[k]; return; }
            o.F.rho = rv.R.rho * (pmr + gc.G6) / (pmr * gc.G6 + T(1.0));
            o.F.p = o.P_M;
            for (int k = 0; k < 3; k++) o.F.v[k] = rv.R.v[k] + n[k] * (o.S_M - vR);
            return;
        }
        o.F.rho = rv.R.rho / gc.G6;
        o.F.p = o.P_M;
        for (int k = 0; k < 3; k++) o.F.v[k] = rv.R.v[k] + n[k] * (o.S_M - vR);
        return;
    }
    if (S >= vR + cR) { o.F.p = rv.R.p; o.F.rho = rv.R.rho; for (int k = 0; k < 3; k++) o.F.v[k] = rv.R.v[k]; return; }
    const T C_eff_R = cR * Real<T>::pow_(o.P_M / rv.R.p, gc.G1);
    if (S <= o.S_M + C_eff_R) {
        o.F.rho = rv.R.rho * Real<T>::pow_(o.P_M / rv.R.p, gc.G8);
        o.F.p = o.P_M;
        for (int k = 0; k < 3; k++) o.F.v[k] = rv.R.v[k] + n[k] * (o.S_M - vR);
        return;
    }
    S_eff = gc.G5 * (-cR + gc.G7 * vR + S);
    C_eff = gc.G5 * (cR - gc.G7 * (vR - S));
    g.power(gc.G3, 17);  // inside the right fan
    o.F.rho = rv.R.rho * Real<T>::pow_(C_eff / cR, gc.G4);
    o.F.p = rv.R.p * Real<T>::pow_(C_eff / cR, gc.G3);
    for (int k = 0; k < 3; k++) o.F.v[k] = rv.R.v[k] + n[k] * (S_eff - vR);
}

// convert_face_to_flux (reimann.h:1070-1083)
template <typename T> GZ_HD void face_to_flux(ROut<T> &o, const T *n, const GConst<T> &gc)
{
    const T rho = o.F.rho, P = o.F.p;
    T v[3] = {o.F.v[0], o.F.v[1], o.F.v[2]};
    const T v_line = dot3(v, n) - T(0);
    T h = T(0.5) * rho * nsq3(v);
    h += (gc.G0 / gc.G9) * P;
    o.F.p = h * v_line;
    o.F.rho = rho * v_line;
    for (int k = 0; k < 3; k++) o.F.v[k] = v[k] * o.F.rho + n[k] * P;
}

// Riemann_solver_exact (reimann.h:625-664). Taken on a small fraction of
// faces only, but inlined: called out of line, the solver's inputs and
// outputs had to be addressable in local memory around the call, and the
// pair kernels ran 5% (FP32) and 4% (FP64) slower at 256^3.
template <typename T>
__host__ __device__ __forceinline__ void riemann_exact(const RVec<T> &rv, ROut<T> &o, const T *n, T vL, T vR, T cL, T cR,
                                                    const GConst<T> &gc, int &stop, Guard<T> &g)
{
    if ((rv.L.p == T(0) && rv.R.p == T(0)) || (rv.L.rho == T(0) && rv.R.rho == T(0))) {
        o.P_M = o.S_M = T(0);
        if (gc.mfv) { o.F.rho = o.F.p = o.F.v[0] = o.F.v[1] = o.F.v[2] = T(0); }
        return;
    }
    if ((rv.L.rho > T(0)) && (rv.R.rho > T(0))) {
        if (riemann_iterative(rv, o, vL, vR, cL, cR, gc, g)) sample_standard(rv, o, n, vL, vR, cL, cR, gc, g);
        else {
            if (gc.mfv) g.power(gc.G3, 16);  // the vacuum fans' states are powers of G3 and G4
            sample_vac_internal(rv, o, n, vL, vR, cL, cR, gc);
        }
    } else {
        if ((rv.L.rho < T(0)) || (rv.R.rho < T(0))) { stop = 1234545; return; }
        if (gc.mfv) g.power(gc.G3, 16);
        if (rv.L.rho > T(0)) sample_vac_right(rv, o, n, vL, cL, gc);
        if (rv.R.rho > T(0)) sample_vac_left(rv, o, n, vR, cR, gc);
    }
    if (gc.mfv) face_to_flux(o, n, gc);
}

// Riemann_solver, hydro branch (reimann.h:282-370); rv taken by value as in the reference
template <typename T>
GZ_HD void riemann_solver(RVec<T> rv, ROut<T> &o, const T *n, T ptl, const GConst<T> &gc, int &stop, Guard<T> &g)
{
    if ((rv.L.p < T(0) && rv.R.p < T(0)) || (rv.L.rho < T(0)) || (rv.R.rho < T(0))) { o.P_M = T(0); return; }
    rv.L.cs = Real<T>::sqrt_(gc.G0 * rv.L.p / rv.L.rho);
    rv.R.cs = Real<T>::sqrt_(gc.G0 * rv.R.p / rv.R.rho);
    rv.L.u = rv.L.p / (gc.G9 * rv.L.rho);
    rv.R.u = rv.R.p / (gc.G9 * rv.R.rho);
    const T cL = rv.L.cs, cR = rv.R.cs;
    const T hL = rv.L.p / rv.L.rho + rv.L.u + T(0.5) * nsq3(rv.L.v);
    const T hR = rv.R.p / rv.R.rho + rv.R.u + T(0.5) * nsq3(rv.R.v);
    const T vL = dot3(rv.L.v, n), vR = dot3(rv.R.v, n);
    T S_L, S_R;
    wavespeeds(rv, o, n, vL, vR, cL, cR, hL, hR, S_L, S_R, ptl, gc, g);  // HLLC_Riemann_solver, reimann.h:382-396
    if (gc.mfv) {
        if ((o.P_M >= T(0)) && (!Real<T>::isnan_(o.P_M))) hllc_fluxes(rv, o, n, vL, vR, hL, hR, S_L, S_R, g);
    } else {
        o.F.rho = T(0);
        for (int k = 0; k < 3; k++) o.F.v[k] = n[k] * o.P_M;
        o.F.p = o.P_M * o.S_M;
    }
    if ((o.P_M < T(0)) || Real<T>::isnan_(o.P_M)) {
        g.flag(20);  // only a NaN star pressure gets here: decided in FP64
        riemann_kt(rv, o, n, vL, vR, cL, cR, hL, hR, gc);
    }
    g.near(o.P_M, ptl, ptl, 21);
    if ((o.P_M < T(0)) || Real<T>::isnan_(o.P_M) || (o.P_M > ptl)) riemann_exact(rv, o, n, vL, vR, cL, cR, gc, stop, g);
}

// reconstruct_face_states, non-MHD (reimann.h:125-244).
// POS: density and pressure, positive and exact in sign, which enter the
// Riemann problem relatively, so their face states are checked for relative
// precision. Otherwise (velocities, differences v - v_frame) `scale` bounds
// the magnitudes Q_i and Q_j were computed from: the sign-preserving clamps
// jump where Qmax, Qmin or their extended bounds cross zero, so a crossing
// within the FP32 error of that scale is decided in FP64.
template <bool POS, typename T>
GZ_HD void reconstruct(T Q_i, const T *g_i, T Q_j, const T *g_j, const T *d_i, const T *d_j, T &Q_L, T &Q_R, int mode,
                        T scale, Guard<T> &g)
{
    if (mode == 0) { Q_R = Q_i; Q_L = Q_j; return; }
    if (Q_i == Q_j) { Q_L = Q_R = Q_i; return; }
    Q_R = Q_i + g_i[0] * d_i[0] + g_i[1] * d_i[1] + g_i[2] * d_i[2];
    Q_L = Q_j + g_j[0] * d_j[0] + g_j[1] * d_j[1] + g_j[2] * d_j[2];
    // the magnitude of the terms each candidate face value is a sum of (its
    // FP32 rounding error is 2^-24 of that), carried with the value it chooses
    T tR = fabs(Q_i) + fabs(g_i[0] * d_i[0]) + fabs(g_i[1] * d_i[1]) + fabs(g_i[2] * d_i[2]);
    T tL = fabs(Q_j) + fabs(g_j[0] * d_j[0]) + fabs(g_j[1] * d_j[1]) + fabs(g_j[2] * d_j[2]);
    T Qmin, Qmax, Qmed, Qmax_eff, Qmin_eff, fac, Qmed_max, Qmed_min;
    Qmed = T(0.5) * (Q_i + Q_j);
    if (Q_i < Q_j) { Qmax = Q_j; Qmin = Q_i; } else { Qmax = Q_i; Qmin = Q_j; }
    fac = T(0.5) * (Qmax - Qmin);
    Qmax_eff = Qmax + fac;
    Qmin_eff = Qmin - fac;
    T tmaxe = T(1.5) * fabs(Qmax) + T(0.5) * fabs(Qmin), tmine = T(1.5) * fabs(Qmin) + T(0.5) * fabs(Qmax);
    if (mode > 0) {
        // Qmax and Qmin carry the error of the values they were computed from
        // (none for rho and P, whose signs are exact); the extended bounds that
        // of their own terms
        if constexpr (!POS) {
            g.near(Qmax, T(0), scale, 22);
            g.near(Qmin, T(0), scale, 23);
        }
        const T sc = scale + fabs(Qmax) + fabs(Qmin);
        g.near(Qmax_eff, T(0), sc, 24);
        g.near(Qmin_eff, T(0), sc, 25);
        // the sign-preserving bounds divide by a sum of like-signed terms: well conditioned
        if (Qmax < T(0)) {
            if (Qmax_eff > T(0)) { Qmax_eff = Qmax * Qmax / (Qmax - (Qmax_eff - Qmax)); tmaxe = T(4) * fabs(Qmax_eff); }
        }
        if (Qmin > T(0)) {
            if (Qmin_eff < T(0)) { Qmin_eff = Qmin * Qmin / (Qmin + (Qmin - Qmin_eff)); tmine = T(4) * fabs(Qmin_eff); }
        }
    }
    fac = T(0.375) * (Qmax - Qmin);
    Qmed_max = Qmed + fac;
    Qmed_min = Qmed - fac;
    T tmedx = T(0.5) * (fabs(Q_i) + fabs(Q_j)) + T(0.375) * (fabs(Qmax) + fabs(Qmin)), tmedn = tmedx;
    if (Qmed_max > Qmax_eff) { Qmed_max = Qmax_eff; tmedx = tmaxe; }
    if (Qmed_min < Qmin_eff) { Qmed_min = Qmin_eff; tmedn = tmine; }
    if (Q_i < Q_j) {
        if (Q_R < Qmin_eff) { Q_R = Qmin_eff; tR = tmine; }
        if (Q_R > Qmed_max) { Q_R = Qmed_max; tR = tmedx; }
        if (Q_L > Qmax_eff) { Q_L = Qmax_eff; tL = tmaxe; }
        if (Q_L < Qmed_min) { Q_L = Qmed_min; tL = tmedn; }
    } else {
        if (Q_R > Qmax_eff) { Q_R = Qmax_eff; tR = tmaxe; }
        if (Q_R < Qmed_min) { Q_R = Qmed_min; tR = tmedn; }
        if (Q_L < Qmin_eff) { Q_L = Qmin_eff; tL = tmine; }
        if (Q_L > Qmed_max) { Q_L = Qmed_max; tL = tmedx; }
    }
    if constexpr (POS) {
        g.precise(Q_R, tR, 35);
        g.precise(Q_L, tL, 36);
    }
}

// One side of a force pair, in pair arithmetic T.
template <typename T> struct Side {
    T v[3], pv[3], nvt[6], grho[3], gp[3], gv[9];
    T m, rho, P, h, cs, cond, fce, drk;
    double dt;
    // FP64 per-particle values for the pair's discontinuous decisions (volume
    // contrast, condition-number fallback, reconstruction mode, entropic
    // switch): V = m / rho, ConditionNumber, FaceClosureError, P / rho. In the
    // FP64 form they equal what the pair would compute; in the mixed form they
    // make those decisions exactly the FP64 form's.
    double Vd, condd, fced, prd;
};

// Result of one canonical pair evaluation, i = the "local" (R) side.
// (16-byte aligned: 32 bytes in FP32, 64 in FP64, so that a stored flux
// fills whole sectors)
template <typename T> struct __align__(16) PairFlux {
    T rho, p, v[3];  // Fluxes.{rho,p,v} after face-area scaling and the MFM switch
    T vsig_ts;       // vsig + |c_i - c_j|, for MaxSignalVel
    int valid;       // inside support (r < max(h_i,h_j), r > 0, j has mass/density)
};

// hydro_accumulate_neighbor (hydro_functions.h:56-546) pair part: kernels at
// h_i and h_j, signal speed, then the meshless core
// (hydro_core_meshless_functions.h:48-616) with the face of
// compute_finitevol_faces_functions.h:46-168. dp = x_i - x_j (min image),
// r2 its exact FP64 square. The support test uses r2 in FP64 so both forms
// pick the same pairs.
// `g` collects the pair's fragile decisions (Guard<float>: a mixed-form pair
// whose branch may differ from the FP64 form's, or whose arithmetic cancels
// beyond FP32's reach; the caller evaluates it again in FP64).
template <typename T>
GZ_HD void force_pair(int kf, int mfv, int selfgravity_off, const GConst<T> &gc, const Side<T> &I, const Side<T> &J,
                       const T dp[3], double r2d, double hi_d, double hj_d, PairFlux<T> &out, int &stop, Guard<T> &g)
{
    out.valid = 0;
    out.rho = out.p = T(0);
    out.v[0] = out.v[1] = out.v[2] = T(0);
    out.vsig_ts = T(0);
    if (J.m <= T(0)) return;
    if (J.rho <= T(0)) return;
    if ((r2d >= hi_d * hi_d) && (r2d >= hj_d * hj_d)) return;
    if (r2d <= 0) return;
    out.valid = 1;
    const T r2 = T(r2d);
    const T r = Real<T>::sqrt_(r2);
    const T rinv = T(1.0) / r;
    T dv[3] = {I.v[0] - J.v[0], I.v[1] - J.v[1], I.v[2] - J.v[2]};
    T vsig = I.cs + J.cs;
    T hinv_i, hinv3_i, hinv4_i, hinv_j, hinv3_j, hinv4_j;
    T wk_i = T(0), dwk_i = T(0), wk_j = T(0), dwk_j = T(0);
    const double r_sup = Real<T>::support_r(r, r2d);
    k_hinv(I.h, hinv_i, hinv3_i, hinv4_i);
    if (Real<T>::inside(r_sup, r2d, I.h, hi_d)) {
        const T u = Real<T>::below_one(r * hinv_i);
        k_main_t(kf, u, Real<T>::one_minus_u(u, r_sup, hi_d, hinv_i), hinv3_i, hinv4_i, wk_i, dwk_i);
    }
    k_hinv(J.h, hinv_j, hinv3_j, hinv4_j);
    if (Real<T>::inside(r_sup, r2d, J.h, hj_d)) {
        const T u = Real<T>::below_one(r * hinv_j);
        k_main_t(kf, u, Real<T>::one_minus_u(u, r_sup, hj_d, hinv_j), hinv3_j, hinv4_j, wk_j, dwk_j);
    }
    // explicitly rounded FP64 (no contraction in either build)
    const double cnumcrit2 = cr::sub(cr::mul(kCnDanger, kCnDanger), cr::mul(I.condd, I.condd));
    const double cnum2 = cr::mul(J.condd, J.condd);
    T eps_big = T(0.5), eps_small = T(1.e-3);
    if (!mfv && !selfgravity_off) { eps_small = T(1.e-2); eps_big = T(0.6); }
    const T vdotr2 = dot3(dp, dv);
    if (vdotr2 < T(0)) {
        if (mfv) vsig -= T(3) * T(1.0) * vdotr2 * rinv;
        else vsig -= T(1.0) * vdotr2 * rinv;
    }
    const T V_i = I.m / I.rho;
    T V_j = J.m / J.rho;
    T FAN = T(0), FA[3] = {T(0), T(0), T(0)}, face_vel_i = T(0), face_vel_j = T(0);
    Crv<T> Fl = {};
    RVec<T> rv = {};
    ROut<T> ro = {};
    do {
        const double leak_vs_tol = cr::mul(0.5, cr::add(I.fced, J.fced));
        const T Pressure_i = I.P, Pressure_j = J.P;
        V_j = J.m / J.rho;
        {
            T wt_i = V_i, wt_j = V_j;
            if (cr::div_(cr::div_(fabs(cr::sub(I.Vd, J.Vd)), dmin(I.Vd, J.Vd)), 3.0) > 1.25)
                wt_i = wt_j = V_i * V_j * (wk_i + wk_j) / (V_i * wk_i + V_j * wk_j);
            T ai[3], aj[3];
            sym_matvec(I.nvt, dp, ai);
            sym_matvec(J.nvt, dp, aj);
            const T si = wk_i * wt_i, sj = wk_j * wt_j;
            for (int k = 0; k < 3; k++) FA[k] = (ai[k] * si + aj[k] * sj) * (T(1.0) * T(1.0));
            FAN = nsq3(FA);
            // the face area holds its relative precision where the two sides' terms cancel, and
            // its sign against dp is decided on the same scale (|dp_k| <= r)
            const T fterms = (fabs(ai[0]) + fabs(ai[1]) + fabs(ai[2])) * fabs(si) +
                             (fabs(aj[0]) + fabs(aj[1]) + fabs(aj[2])) * fabs(sj);
            g.precise(fabs(FA[0]) + fabs(FA[1]) + fabs(FA[2]), fterms, 37);
            const T fn_dot_dp = dot3(FA, dp);
            g.near(fn_dot_dp, T(0), fterms * r, 26);
            if ((cnum2 > cr::add(1.0e12, cnumcrit2)) || (fn_dot_dp < T(0))) {
                T fk = -(wt_i * V_i * dwk_i + wt_j * V_j * dwk_j) / r;
                fk *= T(1.0) * T(1.0);
                for (int k = 0; k < 3; k++) FA[k] = dp[k] * fk;
                FAN = fk * fk * r2;
            }
            FAN = Real<T>::sqrt_(FAN);
        }
        if (FAN == T(0)) { Fl = Crv<T>{}; break; }
        T n[3];
        {
            const T inv = T(1.0) / FAN;
            for (int k = 0; k < 3; k++) n[k] = FA[k] * inv;
        }
        T s_i = T(0.5) * r, s_j = T(-0.5) * r;
        s_i = T(0) - s_i;
        s_j = T(0) - s_j;
        T d_i[3], d_j[3];
        for (int k = 0; k < 3; k++) d_i[k] = dp[k] * rinv;
        for (int k = 0; k < 3; k++) { d_j[k] = d_i[k] * s_j; d_i[k] *= s_i; }
        T vframe[3];
        for (int k = 0; k < 3; k++) {
            const T wj = mfv ? J.pv[k] : J.v[k], wi = mfv ? I.pv[k] : I.v[k];  // values, not a pointer select
            vframe[k] = (wj * (-s_i) + wi * s_j) * rinv;
        }
        face_vel_i += dot3(I.v, n);
        face_vel_j += dot3(J.v, n);
        const T face_area_dot_vel = ((-s_i) * face_vel_j + s_j * face_vel_i) * rinv;
        T v2_approach = T(0);
        T vdotr2_phys = vdotr2;
        vdotr2_phys *= T(1.0) / (r * T(1.0));
        if (vdotr2_phys < T(0)) v2_approach = vdotr2_phys * vdotr2_phys;
        const T vdotf2_phys = face_vel_i - face_vel_j;
        if (vdotf2_phys < T(0)) v2_approach = dmax(v2_approach, vdotf2_phys * vdotf2_phys);
        int recon_mode = 1;
        if (leak_vs_tol > 1.0) recon_mode = 0;
        reconstruct<true>(I.rho, I.grho, J.rho, J.grho, d_i, d_j, rv.L.rho, rv.R.rho, recon_mode, T(0), g);
        reconstruct<true>(Pressure_i, I.gp, Pressure_j, J.gp, d_i, d_j, rv.L.p, rv.R.p, recon_mode, T(0), g);
        for (int k = 0; k < 3; k++)
            reconstruct<false>(I.v[k] - vframe[k], I.gv + 3 * k, J.v[k] - vframe[k], J.gv + 3 * k, d_i, d_j, rv.L.v[k],
                        rv.R.v[k], recon_mode, fabs(I.v[k]) + fabs(J.v[k]) + fabs(vframe[k]), g);
        const T press_i_tot = Pressure_i + I.rho * v2_approach;
        const T press_j_tot = Pressure_j + J.rho * v2_approach;
        T ptl = T(1.1) * T(1.0) * dmax(press_i_tot, press_j_tot);
        if (mfv) ptl *= T(2.0);
        if (recon_mode == 0) ptl = dmax(ptl, dmax(dmax(Pressure_i, Pressure_j), T(2.) * dmax(I.rho, J.rho) * v2_approach));
        // Up to three attempts (hydro_core_meshless_functions.h:350-427): the
        // reconstructed faces; then the cell-centred states at 1.4 x the
        // pressure limit; then the same at zero velocity at 2 x. The same calls
        // in the same order as the reference, through one call site: a single
        // inlined copy of the solver keeps the kernel's code (and its
        // instruction-cache misses) smaller.
        for (int attempt = 0; attempt < 3; attempt++) {
            T lim = ptl;
            if (attempt > 0) {
                rv.R.p = Pressure_i; rv.L.p = Pressure_j;
                rv.R.rho = I.rho; rv.L.rho = J.rho;
                for (int k = 0; k < 3; k++) {
                    rv.R.v[k] = attempt == 1 ? I.v[k] - vframe[k] : T(0);
                    rv.L.v[k] = attempt == 1 ? J.v[k] - vframe[k] : T(0);
                }
                lim = attempt == 1 ? T(1.4) * ptl : T(2.0) * ptl;
            }
            riemann_solver(rv, ro, n, lim, gc, stop, g);
            bool retry = (ro.P_M < T(0)) || Real<T>::isnan_(ro.P_M);
            if (attempt == 0) {
                g.near(ro.P_M, T(1.4) * ptl, ptl, 27);
                retry = retry || (ro.P_M > T(1.4) * ptl);
            }
            if (Real<T>::isnan_(ro.P_M)) g.flag(28);  // a NaN star pressure: decided in FP64
            if (!retry) break;
            if (attempt == 2) stop = 1234;
        }
        if (!((ro.P_M > T(0)) && (!Real<T>::isnan_(ro.P_M)))) { Fl = Crv<T>{}; break; }
        ro.F.p += dot3(vframe, ro.F.v);  // de-boost, hydro_core_meshless_functions.h:459-468
        if (mfv) {
            ro.F.p += T(0.5) * nsq3(vframe) * ro.F.rho;
            for (int k = 0; k < 3; k++) ro.F.v[k] += vframe[k] * ro.F.rho;
        }
        if (mfv) Fl.rho = FAN * ro.F.rho;
        Fl.p = FAN * ro.F.p;
        for (int k = 0; k < 3; k++) Fl.v[k] = ro.F.v[k] * FAN;
        if (!mfv) {  // MFM face entropic switch, hydro_core_meshless_functions.h:515-574
            const T SM_over_ceff = fabs(ro.S_M) / dmin(I.cs, J.cs);
            const T facenorm_pm = ro.P_M * FAN;
            const T PdV_fac = ro.P_M * vdotr2_phys / T(1.0);
            const T PdV_i = dwk_i * V_i * V_i * I.drk * PdV_fac;
            const T PdV_j = dwk_j * V_j * V_j * J.drk * PdV_fac;
            const T du_old = facenorm_pm * (ro.S_M + face_area_dot_vel);
            const T du_new = T(0.5) * (PdV_i - PdV_j + facenorm_pm * (face_vel_i + face_vel_j));
            // The switch's tests (SM/c against eps_big, which opens the switch, and eps_small, and
            // the signs and sizes of the energy changes each side would see) choose between du_old
            // and du_new: a flip moves the flux by |du_new - du_old|. Guarded only where that is
            // not negligible on the scale of the face's work terms; the opening test is guarded
            // whichever way FP32 takes it.
            const T es = fabs(du_old) + fabs(du_new) + fabs(facenorm_pm * face_vel_i) +
                         fabs(facenorm_pm * face_vel_j);
            const bool switch_matters = fabs(du_new - du_old) > T(1e-6) * es;
            if (switch_matters && !(leak_vs_tol > 1.0)) g.near(SM_over_ceff, eps_big, eps_big, 29);
            if ((SM_over_ceff < eps_big) || (leak_vs_tol > 1.0)) {
                int use = 1;
                const double ratio = 1.001;
                const double to_i = I.prd, to_j = J.prd;
                if (switch_matters) {
                    if (cnum2 < cnumcrit2) {
                        const T dtoj = -du_old + facenorm_pm * face_vel_j, dtoi = +du_old - facenorm_pm * face_vel_i;
                        g.near(SM_over_ceff, eps_small, T(0.1), 30);  // S_M to ~1e-6 c (the exact solver's tolerance)
                        g.near(dtoj, T(0), es, 31);
                        g.near(dtoi, T(0), es, 32);
                        g.near(dtoj, -du_new + facenorm_pm * face_vel_j, es, 33);
                        g.near(dtoi, +du_new - facenorm_pm * face_vel_i, es, 34);
                    }
                }
                if (use && SM_over_ceff > eps_small && cnum2 < cnumcrit2) {
                    if (to_i > cr::mul(ratio, to_j)) {
                        const T dtoj = -du_old + facenorm_pm * face_vel_j;
                        if (dtoj > T(0)) use = 0;
                        else { if (dtoj < T(0)) { if (dtoj > -du_new + facenorm_pm * face_vel_j) use = 0; } }
                    } else if (cr::mul(ratio, to_i) < to_j) {
                        const T dtoi = +du_old - facenorm_pm * face_vel_i;
                        if (dtoi > T(0)) use = 0;
                        else { if (dtoi < T(0)) { if (dtoi > +du_new - facenorm_pm * face_vel_i) use = 0; } }
                    } else {
                        const T dtoj = -du_old + facenorm_pm * face_vel_j;
                        const T dtoi = +du_old - facenorm_pm * face_vel_i;
                        if (dtoj < T(0)) { if (dtoj > -du_new + facenorm_pm * face_vel_j) use = 0; }
                        if (dtoi < T(0)) { if (dtoi > +du_new - facenorm_pm * face_vel_i) use = 0; }
                    }
                }
                if (cnum2 >= cnumcrit2) use = 1;
                if (use) Fl.p += du_new - du_old;
            }
        }
    } while (0);
    out.rho = Fl.rho;
    out.p = Fl.p;
    out.v[0] = Fl.v[0]; out.v[1] = Fl.v[1]; out.v[2] = Fl.v[2];
    out.vsig_ts = vsig + fabs(I.cs - J.cs);
}

// MFV mass-exchange bookkeeping of one side (hydro_functions.h:419-441, 511-532):
// with this side's flux f_rho, its own dt and the other's, returns this side's
// dMass increment, the accepted flux for its GravWorkTerm, and the write it
// makes on the other side's dMass.
GZ_HD void mfv_mass_side(double f_rho, double dt_self, double dt_other, double m_self, double m_other,
                          double &dmass_self, double &accepted, double &dmass_other)
{
    double dmass_holder = f_rho * dt_self, lim;
    if (dmass_holder > 0) lim = m_other; else lim = m_self;
    lim *= 0.1;
    accepted = f_rho;
    double jw = dmass_holder;
    if (fabs(dmass_holder) > lim) {
        accepted *= lim / fabs(dmass_holder);
        jw *= lim / fabs(dmass_holder);
    }
    dmass_holder = jw;
    dmass_self = 0;
    dmass_other = 0;
    if (dt_self < dt_other) { dmass_self = dmass_holder; dmass_other = -dmass_holder; }
    else if (dt_self == dt_other) { dmass_self = 0.5 * dmass_holder; accepted *= 0.5; dmass_other = -0.5 * dmass_holder; }
    else { accepted = 0; }
}

}  // namespace gz

/* oracle/gizmo_oracle.c -- CPU restatement of GIZMO's meshless hydro pass.
 *
 * TEST INFRASTRUCTURE ONLY (see gizmo_oracle.h for scope and citations).
 * Compiled with -ffp-contract=off so every expression rounds as written;
 * operation order follows the reference line by line (cited per function),
 * including its Vec3 conventions: v / s is v * (1/s) (math_types/vec3.h:29)
 * and scalar * Vec3 multiplies each component (vec3.h:38-40).
 * Reference configuration restated: 3-D, BOX_PERIODIC, ideal gas, no MHD,
 * no cooling, non-comoving (cf_atime = 1), SLOPE_LIMITER_TOLERANCE = 1,
 * HYDRO_FIX_MESH_MOTION = 5 for MFV, CONDITION_NUMBER_DANGER = 1e3.
 */
#define _DEFAULT_SOURCE 1 /* M_PI */
#include "gizmo_oracle.h"
#include "orc_grid.h"

#include <math.h>
#include <omp.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

#define NDIM 3
#define MIN_REAL 1e-56                 /* constants.h:220 */
#define CN_DANGER 1.0e3                /* constants.h:225 */
#define MAXITER 150                    /* constants.h:340 */
#define VOLNORM 4.188790204786         /* constants.h:445 */
#define DMAX(a, b) ((a) > (b) ? (a) : (b)) /* macros.h:219 */
#define DMIN(a, b) ((a) < (b) ? (a) : (b)) /* macros.h:220 */

/* ------------------------------------------------------------------ kernel */
/* kernel_hinv, kernel_main: mesh/kernel.h:245-260, 268-438 (K=3 cubic,
 * K=6 Wendland C2; norms kernel.h:69 8/pi and kernel.h:123 21/(2 pi)). */
static inline void k_hinv(double h, double *hinv, double *hinv3, double *hinv4)
{
    *hinv = 1.0 / h;
    *hinv3 = *hinv * *hinv * *hinv;
    *hinv4 = *hinv3 * *hinv;
}

static inline void k_main(int kf, double u, double hinv3, double hinv4, double *wk, double *dwk)
{
    if (u >= 1) { *wk = 0; *dwk = 0; return; }
    double w, dw;
    if (kf == GZ_KERNEL_CUBIC) {
        if (u < 0.5) {
            dw = u * (18.0 * u - 12.0);
            w = (1.0 + 6.0 * (u - 1.0) * u * u);
        } else {
            double t1 = (1.0 - u);
            double t2 = t1 * t1;
            dw = -6.0 * t2;
            w = 2.0 * t2 * t1;
        }
        *dwk = dw * ((8.0 / M_PI) * hinv4);
        *wk = w * ((8.0 / M_PI) * hinv3);
    } else {
        double t1 = (1 - u);
        double t3 = t1 * t1 * t1;
        dw = -20.0 * u * t3;
        w = t3 * t1 * (1.0 + 4.0 * u);
        *dwk = dw * ((21.0 / (2.0 * M_PI)) * hinv4);
        *wk = w * ((21.0 / (2.0 * M_PI)) * hinv3);
    }
}

/* NEAREST_XYZ for a periodic box (macros.h:58-109): y, x, z order. */
static inline void wrap3(double *dp, double box)
{
    const double half = 0.5 * box;
    dp[1] = orc_wrap(dp[1], box, half);
    dp[0] = orc_wrap(dp[0], box, half);
    dp[2] = orc_wrap(dp[2], box, half);
}

/* ------------------------------------------------------------ 3x3 inverse */
/* Mat3::invert (math_types/mat3.h:50-63) + matrix_invert_ndims (core/proto.h:75-95). */
static double invert3(const double T[3][3], double Ti[3][3])
{
    double fro = (T[0][0] * T[0][0] + T[0][1] * T[0][1] + T[0][2] * T[0][2]) +
                 (T[1][0] * T[1][0] + T[1][1] * T[1][1] + T[1][2] * T[1][2]) +
                 (T[2][0] * T[2][0] + T[2][1] * T[2][1] + T[2][2] * T[2][2]);
    memset(Ti, 0, sizeof(double) * 9);
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
    return DMAX(sqrt(fro * froi) / NDIM, 1);
}

/* symmetric {xx,yy,zz,xy,yz,xz} -> full (symmetric_tensor2.h:14-27) */
static inline void sym_full(const double *s, double T[3][3])
{
    T[0][0] = s[0]; T[1][1] = s[1]; T[2][2] = s[2];
    T[0][1] = T[1][0] = s[3];
    T[1][2] = T[2][1] = s[4];
    T[0][2] = T[2][0] = s[5];
}

/* NV_T inversion with conditioning + face-closure error, shared by
 * after_iter_body (density_loop.h:572-637) and the finalize
 * (density_loop.cc:444-504). acc_nvt/acc_face are the raw sums. */
static void nvt_invert(double h, double NumNgb, const double *acc_nvt, const double *acc_face, double *CN_out,
                       double Tinv_norm[3][3], double *fce_out)
{
    const double V_i = VOLNORM * pow(h, (double)NDIM) / (NumNgb > 0 ? NumNgb : 1.0);
    const double norm = pow(h, (double)(2 - NDIM));
    double raw[3][3], T[3][3], Tinv[3][3];
    sym_full(acc_nvt, raw);
    for (int a = 0; a < 3; a++)
        for (int b = 0; b < 3; b++) T[a][b] = raw[a][b] / norm;
    const double thr = 10.0 * CN_DANGER;
    const double tr0 = T[0][0] + T[1][1] + T[2][2];
    double add = 1.05 * (tr0 / NDIM) / thr;
    double CN;
    while (1) {
        CN = invert3(T, Tinv);
        if (CN < thr) break;
        for (int k = 0; k < NDIM; k++) T[k][k] += add;
        add *= 1.2;
    }
    const double tr_raw = raw[0][0] + raw[1][1] + raw[2][2];
    const double dx_i = sqrt(V_i * tr_raw);
    for (int a = 0; a < 3; a++)
        for (int b = 0; b < 3; b++) Tinv_norm[a][b] = Tinv[a][b] / norm;
    double fo[3] = {0, 0, 0};
    for (int a = 0; a < 3; a++)
        for (int b = 0; b < 3; b++) fo[a] += 2.0 * V_i * Tinv_norm[a][b] * acc_face[b];
    double leak = 0;
    for (int a = 0; a < 3; a++) leak += fabs(fo[a]) / (double)NDIM;
    *fce_out = leak / (2.0 * (double)NDIM * pow(dx_i, (double)(NDIM - 1)));
    *CN_out = CN;
}

/* ------------------------------------------------------------ density pair */
/* DensitySpec::pair_kernel, gas i and j (density_loop.h:1140-1385). */
static inline void density_pair(int kf, int mfv, double box, const double *xi, const double *vi, double h,
                                const double *xj, double mj, const double *vj, double *acc, double *pv)
{
    if (mj <= 0) return;
    double dp[3] = {xi[0] - xj[0], xi[1] - xj[1], xi[2] - xj[2]};
    wrap3(dp, box);
    const double r2 = dp[0] * dp[0] + dp[1] * dp[1] + dp[2] * dp[2];
    const double h2 = h * h;
    if (r2 >= h2) return;
    const double r = sqrt(r2);
    double hinv, hinv3, hinv4, wk, dwk;
    k_hinv(h, &hinv, &hinv3, &hinv4);
    const double u = r * hinv;
    k_main(kf, u, hinv3, hinv4, &wk, &dwk);
    const double mj_wk = mj * wk;
    acc[0] += wk;
    acc[1] += mj_wk;
    if (mfv && r == 0) { pv[0] += mj_wk * vj[0]; pv[1] += mj_wk * vj[1]; pv[2] += mj_wk * vj[2]; }
    acc[2] += -(NDIM * hinv * wk + u * dwk);
    if (r > 0) {
        acc[4] += dp[0] * dp[0] * wk;
        acc[5] += dp[1] * dp[1] * wk;
        acc[6] += dp[2] * dp[2] * wk;
        acc[7] += dp[0] * dp[1] * wk;
        acc[8] += dp[1] * dp[2] * wk;
        acc[9] += dp[0] * dp[2] * wk;
        acc[10] += wk * dp[0];
        acc[11] += wk * dp[1];
        acc[12] += wk * dp[2];
        const double dv[3] = {vi[0] - vj[0], vi[1] - vj[1], vi[2] - vj[2]};
        if (mfv) {
            pv[0] += mj_wk * (vi[0] - dv[0]);
            pv[1] += mj_wk * (vi[1] - dv[1]);
            pv[2] += mj_wk * (vi[2] - dv[2]);
        }
        acc[3] -= dwk * (dp[0] * dv[0] + dp[1] * dv[1] + dp[2] * dv[2]) / r;
    }
}

typedef struct {
    double left, right, cn_cur;
    int cn_init;
} dscratch;

/* DensitySpec::after_iter_body for a gas particle (density_loop.h:515-961).
 * Returns 1 when converged; *new_h is the next (or final) radius. */
static int after_iter(const gz_params *p, int iter, double h, const double *acc, double cond_prev, dscratch *sc,
                      double *new_h_out, int *stop)
{
    double desnumngb = p->des_num_ngb;
    double desnumngbdev = p->max_num_ngb_dev;
    if (p->first_step) { if (p->max_num_ngb_dev > 0.05) desnumngbdev = 0.05; }
    const double desnumngbdev_0 = desnumngbdev;
    double NumNgb = acc[0], Drk = acc[2], DivV = acc[3];
    if (NumNgb > 0) {
        Drk *= h / (NDIM * NumNgb);
        DivV /= NumNgb;
        NumNgb *= VOLNORM * pow(h, (double)NDIM);
    } else { NumNgb = 0; Drk = 0; DivV = 0; }
    if (Drk > -0.9) Drk = 1.0 / (1.0 + Drk); else Drk = 1.0;
    (void)DivV;
    double CN, fce, Tn[3][3];
    nvt_invert(h, NumNgb, acc + 4, acc + 10, &CN, Tn, &fce);
    const double c0 = 0.1 * (double)CN_DANGER;
    if ((iter == 0) && (CN > cond_prev) && (cond_prev > 0)) {
        double ncorr_a = 1.0, cn_a = cond_prev;
        if (cn_a > c0) ncorr_a = sqrt(1.0 + (cn_a - c0) / (double)CN_DANGER);
        if (ncorr_a > 2.0) ncorr_a = 2.0;
        const double dn_ngb = fabs(NumNgb - p->des_num_ngb * ncorr_a) / (desnumngbdev_0 * ncorr_a);
        double ncorr_b = 1.0, cn_b = CN;
        if (cn_b > c0) ncorr_b = sqrt(1.0 + (cn_b - c0) / (double)CN_DANGER);
        if (ncorr_b > 2.0) ncorr_b = 2.0;
        const double dn_ngb_alt = fabs(NumNgb - p->des_num_ngb * ncorr_b) / (desnumngbdev_0 * ncorr_b);
        if (DMIN(dn_ngb, dn_ngb_alt) < 10.0) { sc->cn_cur = CN; sc->cn_init = 1; }
    }
    if (!sc->cn_init) { sc->cn_cur = cond_prev; sc->cn_init = 1; }
    double ncorr = 1.0;
    {
        const double cn = sc->cn_cur;
        if (cn > c0) ncorr = sqrt(1.0 + (cn - c0) / (double)CN_DANGER);
        if (ncorr > 2.0) ncorr = 2.0;
        const double d00 = 0.35;
        if (fce > d00) ncorr = DMAX(ncorr, DMIN(fce / d00, 2.0));
    }
    desnumngb = p->des_num_ngb * ncorr;
    desnumngbdev = desnumngbdev_0 * ncorr;
    if (iter > 1)
        desnumngbdev = DMIN(0.25 * desnumngb, desnumngbdev * exp(0.1 * log(desnumngb / (16.0 * desnumngbdev)) * (double)iter));
    const double minsoft = p->min_kernel_radius, maxsoft = p->max_kernel_radius;
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
    if (redo == 0) sc->cn_cur = CN;
    if (redo) {
        if (sc->left > 0 && sc->right > 0) {
            if ((sc->right - sc->left) < 1.0e-3 * sc->left) { sc->cn_cur = CN; *new_h_out = new_h; return 1; }
        }
        if (setmax == 0 && setmin == 0) {
            if (NumNgb < (desnumngb - desnumngbdev)) {
                sc->left = DMAX(new_h, sc->left);
            } else {
                if (sc->right != 0) { if (new_h < sc->right) sc->right = new_h; }
                else sc->right = new_h;
            }
            if (sc->right > 0 && sc->left > 0) {
                double maxjump = 0;
                if (iter > 1) maxjump = 0.2 * log(sc->right / sc->left);
                if (NumNgb > 1) {
                    double jumpvar = Drk * log(desnumngb / NumNgb) / NDIM;
                    if (iter > 1) { if (fabs(jumpvar) < maxjump) { if (jumpvar < 0) jumpvar = -maxjump; else jumpvar = maxjump; } }
                    new_h *= exp(jumpvar);
                } else {
                    new_h *= 2.0;
                }
                if ((new_h < sc->right) && (new_h > sc->left)) {
                    if (iter > 1) {
                        const double hfac = exp(maxjump);
                        if (new_h > sc->right / hfac) new_h = sc->right / hfac;
                        if (new_h < sc->left * hfac) new_h = sc->left * hfac;
                    }
                } else {
                    if (new_h > sc->right) new_h = sc->right;
                    if (new_h < sc->left) new_h = sc->left;
                    new_h = pow(new_h * sc->left * sc->right, 1.0 / 3.0);
                }
            } else {
                if (sc->right == 0 && sc->left == 0) { *stop = GZ_ERR_EMPTY_BRACKET; *new_h_out = new_h; return 1; }
                if (sc->right == 0 && sc->left > 0) {
                    double fac_lim = (NumNgb > 1) ? log(desnumngb / NumNgb) / NDIM : 1.4;
                    if ((NumNgb < 2.0 * desnumngb) && (NumNgb > 0.1 * desnumngb)) {
                        double slope = Drk;
                        if (iter > 2 && slope < 1.0) slope = 0.5 * (slope + 1.0);
                        double fac = fac_lim * slope;
                        if (iter >= 4) { if (Drk == 1.0) fac *= 10.0; }
                        if (fac < fac_lim + 0.231) new_h *= exp(fac); else new_h *= exp(fac_lim + 0.231);
                    } else {
                        new_h *= exp(fac_lim);
                    }
                }
                if (sc->right > 0 && sc->left == 0) {
                    double fac_lim = (NumNgb > 1) ? log(desnumngb / NumNgb) / NDIM : 1.4;
                    if (fac_lim < -1.535) fac_lim = -1.535;
                    if ((NumNgb < 2.0 * desnumngb) && (NumNgb > 0.1 * desnumngb)) {
                        double slope = Drk;
                        if (iter > 2 && slope < 1.0) slope = 0.5 * (slope + 1.0);
                        double fac = fac_lim * slope;
                        if (iter >= 4) { if (Drk == 1.0) fac *= 10.0; }
                        if (fac > fac_lim - 0.231) new_h *= exp(fac); else new_h *= exp(fac_lim - 0.231);
                    } else {
                        new_h *= exp(fac_lim);
                    }
                }
            }
        }
        if (new_h < minsoft) new_h = minsoft;
        if (setmin == 1) new_h = minsoft;
        if (new_h > maxsoft) new_h = maxsoft;
        if (setmax == 1) new_h = maxsoft;
        *new_h_out = new_h;
        return 0;
    }
    sc->cn_cur = CN;
    *new_h_out = new_h;
    return 1;
}

/* density_finalize_post_runner for a gas particle (density_loop.cc:303-733:
 * normalisation, scatter, persistent NV_T inverse, MFV ParticleVel
 * smoothing, non-SPH density, EOS pressure, NumNgb^(1/3)). */
static void density_finalize(const gz_params *p, orc_state *s, int i, double h, const double *acc, const double *pv)
{
    s->h[i] = h;
    double NumNgb = acc[0], Drk = acc[2], DivV = acc[3];
    if (NumNgb > 0) {
        Drk *= h / (NDIM * NumNgb);
        DivV /= NumNgb;
        NumNgb *= VOLNORM * pow(h, (double)NDIM);
    } else { NumNgb = Drk = DivV = 0; }
    if (Drk > -0.9) Drk = 1.0 / (1.0 + Drk); else Drk = 1.0;
    DivV *= Drk;
    s->num_ngb[i] = NumNgb;
    s->drkern[i] = Drk;
    s->divvel[i] = DivV;
    double rho = acc[1];
    double pvl[3] = {pv[0], pv[1], pv[2]};
    double CN, fce, Tn[3][3];
    nvt_invert(h, NumNgb, acc + 4, acc + 10, &CN, Tn, &fce);
    double *nv = s->nvt + 6 * (size_t)i;
    nv[0] = Tn[0][0]; nv[1] = Tn[1][1]; nv[2] = Tn[2][2];
    nv[3] = Tn[0][1]; nv[4] = Tn[1][2]; nv[5] = Tn[0][2];
    s->cond[i] = CN;
    s->fce[i] = fce;
    const double m = s->mass[i];
    if (m > 0) {
        if (rho > 0 && p->method == GZ_METHOD_MFV) {
            const double eps = 0.3;
            for (int k = 0; k < 3; k++) pvl[k] = s->vel[3 * i + k] * (1.0 - eps) + pvl[k] * (eps / rho);
        }
        if ((h > 0) && (NumNgb > 0)) rho = m * NumNgb / (VOLNORM * pow(h, (double)NDIM));
        else if (h <= 0) rho = 0;
        else rho = m / (VOLNORM * pow(h, (double)NDIM));
        s->pressure[i] = (p->gamma - 1) * s->u[i] * rho;
    }
    s->rho[i] = rho;
    for (int k = 0; k < 3; k++) s->pvel[3 * i + k] = pvl[k];
    s->num_ngb[i] = (NumNgb > 0) ? pow(NumNgb, 1.0 / NDIM) : 0;
}

static int *all_indices(int n)
{
    int *a = (int *)malloc(sizeof(int) * (size_t)(n > 0 ? n : 1));
    for (int i = 0; i < n; i++) a[i] = i;
    return a;
}

static void set_threads(int n_threads)
{
    if (n_threads > 0) omp_set_num_threads(n_threads);
}

int orc_density_sums(const gz_params *p, const orc_state *s, const int *active, int n_active, double *acc, double *pv,
                     int n_threads)
{
    set_threads(n_threads);
    int *all = NULL;
    if (!active) { all = all_indices(s->n); active = all; n_active = s->n; }
    orc_grid g;
    if (orc_grid_build(&g, s->pos, s->h, s->n, p->box_size)) { free(all); return GZ_ERR_ARG; }
    const int mfv = p->method == GZ_METHOD_MFV;
#pragma omp parallel
    {
        int *cand = NULL, cap = 0;
#pragma omp for schedule(dynamic, 64)
        for (int a = 0; a < n_active; a++) {
            const int i = active[a];
            double *ac = acc + 14 * (size_t)a, *pa = pv + 3 * (size_t)a;
            memset(ac, 0, sizeof(double) * 14);
            memset(pa, 0, sizeof(double) * 3);
            const int nc = orc_grid_candidates(&g, s->pos + 3 * (size_t)i, s->h[i], 0, &cand, &cap);
            for (int c = 0; c < nc; c++) {
                const int j = cand[c];
                density_pair(p->kernel, mfv, p->box_size, s->pos + 3 * (size_t)i, s->vel + 3 * (size_t)i, s->h[i],
                             s->pos + 3 * (size_t)j, s->mass[j], s->vel + 3 * (size_t)j, ac, pa);
            }
        }
        free(cand);
    }
    orc_grid_free(&g);
    free(all);
    return 0;
}

/* Largest kernel length at which the last orc_density took sums (seeds after
 * the pre-iteration clamp and every radius the iteration moved to). */
static double g_density_h_iter_max = 0;

double orc_density_h_iter_max(void) { return g_density_h_iter_max; }

int orc_density(const gz_params *p, orc_state *s, const int *active, int n_active, int n_threads)
{
    set_threads(n_threads);
    int *all = NULL;
    if (!active) { all = all_indices(s->n); active = all; n_active = s->n; }
    const int mfv = p->method == GZ_METHOD_MFV;
    /* pre-iteration clamp (density_loop.cc:837-840) */
    for (int a = 0; a < n_active; a++) {
        const int i = active[a];
        const double maxsoft = p->max_kernel_radius;
        if ((s->h[i] < 0) || !isfinite(s->h[i]) || (s->h[i] > 0.99 * maxsoft)) s->h[i] = 0.99 * maxsoft;
    }
    /* grid over positions only: one-way queries need no neighbour h */
    orc_grid g;
    if (orc_grid_build(&g, s->pos, NULL, s->n, p->box_size)) { free(all); return GZ_ERR_ARG; }
    int status = 0;
    double *final_acc = (double *)malloc(sizeof(double) * 14 * (size_t)(n_active > 0 ? n_active : 1));
    double *final_pv = (double *)malloc(sizeof(double) * 3 * (size_t)(n_active > 0 ? n_active : 1));
    double *final_h = (double *)malloc(sizeof(double) * (size_t)(n_active > 0 ? n_active : 1));
    double h_iter_max = 0;
#pragma omp parallel reduction(max : h_iter_max)
    {
        int *cand = NULL, cap = 0;
#pragma omp for schedule(dynamic, 16)
        for (int a = 0; a < n_active; a++) {
            const int i = active[a];
            const double *xi = s->pos + 3 * (size_t)i, *vi = s->vel + 3 * (size_t)i;
            dscratch sc = {0, 0, 0, 0};
            double h = s->h[i], acc[14], pv[3];
            int it = 0, conv = 0, stop = 0;
            for (it = 0; it < MAXITER; it++) {
                if (h > h_iter_max) h_iter_max = h;
                memset(acc, 0, sizeof(acc));
                memset(pv, 0, sizeof(pv));
                const int nc = orc_grid_candidates(&g, xi, h, 0, &cand, &cap);
                for (int c = 0; c < nc; c++) {
                    const int j = cand[c];
                    density_pair(p->kernel, mfv, p->box_size, xi, vi, h, s->pos + 3 * (size_t)j, s->mass[j],
                                 s->vel + 3 * (size_t)j, acc, pv);
                }
                double nh;
                conv = after_iter(p, it, h, acc, s->cond[i], &sc, &nh, &stop);
                /* the runner moves the radius only on AdjustRadius; a converged
                 * slot keeps the radius its last sums were taken at
                 * (neighbor_loop_runner.cc:7353-7361, 7522-7527) */
                if (conv) break;
                h = nh;
            }
            memcpy(final_acc + 14 * (size_t)a, acc, sizeof(acc));
            memcpy(final_pv + 3 * (size_t)a, pv, sizeof(pv));
            final_h[a] = h;
            if (s->iters) s->iters[i] = it + (conv ? 1 : 0);
            int code = stop ? stop : (conv ? 0 : GZ_ERR_DENSITY_MAXITER);
            if (code) {
#pragma omp critical
                { if (!status) status = code; }
            }
        }
        free(cand);
    }
    g_density_h_iter_max = h_iter_max;
    for (int a = 0; a < n_active; a++) density_finalize(p, s, active[a], final_h[a], final_acc + 14 * (size_t)a, final_pv + 3 * (size_t)a);
    free(final_acc); free(final_pv); free(final_h);
    orc_grid_free(&g);
    free(all);
    return status;
}

/* ------------------------------------------------------------- gradients */
/* local_slopelimiter (gradients_loop.cc:76-104, Newtonian branch). */
static void slopelimiter(double *g, double valmax, double valmin, double alim, double h, double shoot_tol,
                         int pos_preserve, double d_max, double val_cen)
{
    double d_abs = g[0] * g[0] + g[1] * g[1] + g[2] * g[2];
    if (d_abs > 0) {
        d_abs = sqrt(d_abs);
        double cfac = 1 / (alim * h * d_abs);
        double fabs_max = fabs(valmax), fabs_min = fabs(valmin), abs_max = fabs_max, abs_min = fabs_min, f_corr;
        if (abs_max < abs_min) { abs_max = fabs_min; abs_min = fabs_max; }
        f_corr = DMIN(abs_min + shoot_tol * abs_max, abs_max);
        cfac *= f_corr;
        if (pos_preserve == 1) {
            double fmin = DMIN(val_cen, DMAX(0, DMAX(MIN_REAL * val_cen, DMIN(0.5 * (val_cen + valmin), val_cen - f_corr))));
            cfac = DMIN(((val_cen - fmin) / d_max) / d_abs, cfac);
        }
        if (cfac < 1) { g[0] *= cfac; g[1] *= cfac; g[2] *= cfac; }
    }
}

/* SymmetricTensor2::matvec (symmetric_tensor2.h:80-84) */
static inline void sym_matvec(const double *s, const double *v, double *o)
{
    const double a = s[0] * v[0] + s[3] * v[1] + s[5] * v[2];
    const double b = s[3] * v[0] + s[1] * v[1] + s[4] * v[2];
    const double c = s[5] * v[0] + s[4] * v[1] + s[2] * v[2];
    o[0] = a; o[1] = b; o[2] = c;
}

#define MINMAX(x, lo, hi) ((x < lo) ? (lo = x) : ((x > hi) ? (hi = x) : (1)))

/* symmetric-support neighbour rows for the active set, from the pyramid */
typedef struct { int *cand; int cap; } candbuf;

int orc_gradients(const gz_params *p, orc_state *s, const int *active, int n_active, int n_threads)
{
    set_threads(n_threads);
    int *all = NULL;
    if (!active) { all = all_indices(s->n); active = all; n_active = s->n; }
    orc_grid g;
    if (orc_grid_build(&g, s->pos, s->h, s->n, p->box_size)) { free(all); return GZ_ERR_ARG; }
    const double box = p->box_size;
#pragma omp parallel
    {
        int *cand = NULL, cap = 0;
#pragma omp for schedule(dynamic, 16)
        for (int a = 0; a < n_active; a++) {
            const int i = active[a];
            if (!(s->mass[i] > 0 && s->rho[i] > 0)) { /* GradientsSpec load_active enabled gate: zero gradients */
                for (int k = 0; k < 3; k++) { s->grad_rho[3 * (size_t)i + k] = 0; s->grad_p[3 * (size_t)i + k] = 0; }
                for (int k = 0; k < 9; k++) s->grad_v[9 * (size_t)i + k] = 0;
                continue;
            }
            const double *xi = s->pos + 3 * (size_t)i, *vi = s->vel + 3 * (size_t)i;
            const double hi = s->h[i], rho_i = s->rho[i], P_i = s->pressure[i];
            double hinv, hinv3, hinv4;
            k_hinv(hi, &hinv, &hinv3, &hinv4);
            double gr[3][5];
            double mx[5] = {0, 0, 0, 0, 0}, mn[5] = {0, 0, 0, 0, 0}, maxdist = 0;
            memset(gr, 0, sizeof(gr));
            const int nc = orc_grid_candidates(&g, xi, hi, 1, &cand, &cap);
            for (int c = 0; c < nc; c++) {
                const int j = cand[c];
                /* GasGrad_isactive_gpu (gradient_functions.h:200-211) */
                if (s->mass[j] <= 0) continue;
                if (s->rho[j] <= 0 || s->h[j] <= 0) continue;
                /* gradient_accumulate_neighbor (gradient_functions.h:304-665) */
                double dp[3] = {xi[0] - s->pos[3 * (size_t)j], xi[1] - s->pos[3 * (size_t)j + 1], xi[2] - s->pos[3 * (size_t)j + 2]};
                wrap3(dp, box);
                const double r2 = dp[0] * dp[0] + dp[1] * dp[1] + dp[2] * dp[2];
                const double hj = s->h[j];
                if (r2 <= 0) continue;
                const double h2_i = hi * hi;
                if ((r2 >= h2_i) && (r2 >= hj * hj)) continue;
                const double r = sqrt(r2);
                double wk_i = 0, dwk_i = 0;
                if (r < hi) { const double u = r * hinv; k_main(p->kernel, u, hinv3, hinv4, &wk_i, &dwk_i); }
                if (r > maxdist) maxdist = r;
                double d[5];
                d[0] = s->rho[j] - rho_i;
                MINMAX(d[0], mn[0], mx[0]);
                d[1] = s->pressure[j] - P_i;
                MINMAX(d[1], mn[1], mx[1]);
                for (int k = 0; k < 3; k++) {
                    d[2 + k] = s->vel[3 * (size_t)j + k] - vi[k];
                    MINMAX(d[2 + k], mn[2 + k], mx[2 + k]);
                }
                if (r < hi) {
                    const double w = wk_i;
                    for (int k = 0; k < 3; k++) {
                        const double wxyz = -w * dp[k];
                        gr[k][0] += wxyz * d[0];
                        gr[k][1] += wxyz * d[1];
                        gr[k][2] += d[2] * wxyz;
                        gr[k][3] += d[3] * wxyz;
                        gr[k][4] += d[4] * wxyz;
                    }
                }
            }
            /* finalize: construct_gradient + limiter (gradients_loop.cc:129-136, 1077-1130) */
            const double *nv = s->nvt + 6 * (size_t)i;
            double grho[3] = {gr[0][0], gr[1][0], gr[2][0]}, gp[3] = {gr[0][1], gr[1][1], gr[2][1]}, gv[3][3];
            for (int c = 0; c < 3; c++) { gv[c][0] = gr[0][2 + c]; gv[c][1] = gr[1][2 + c]; gv[c][2] = gr[2][2 + c]; }
            sym_matvec(nv, grho, grho);
            sym_matvec(nv, gp, gp);
            for (int c = 0; c < 3; c++) sym_matvec(nv, gv[c], gv[c]);
            double stol = 0.0;
            double h_lim = hi;
            const double d_max = DMAX(hi, maxdist);
            h_lim = d_max;
            double a_limiter = 0.25;
            const double CN = s->cond[i];
            if (CN > 100) a_limiter = DMIN(0.5, 0.25 + 0.25 * (CN - 100) / 100);
            if (p->selfgravity_off) { h_lim = hi; stol = 0.1; }
            slopelimiter(grho, mx[0], mn[0], a_limiter, h_lim, 0, 1, d_max, rho_i);
            slopelimiter(gp, mx[1], mn[1], a_limiter, h_lim, stol, 1, d_max, P_i);
            for (int c = 0; c < 3; c++) slopelimiter(gv[c], mx[2 + c], mn[2 + c], a_limiter, h_lim, stol, 0, 0, 0);
            for (int k = 0; k < 3; k++) {
                s->grad_rho[3 * (size_t)i + k] = grho[k];
                s->grad_p[3 * (size_t)i + k] = gp[k];
                for (int c = 0; c < 3; c++) s->grad_v[9 * (size_t)i + 3 * c + k] = gv[c][k];
            }
        }
        free(cand);
    }
    orc_grid_free(&g);
    free(all);
    return 0;
}

/* ---------------------------------------------------------------- Riemann */
typedef struct { double rho, p, v[3], u, cs; } crv;     /* Conserved_var_Riemann (hydro_structs.h:17-38) */
typedef struct { crv L, R; } rvec;                      /* Input_vec_Riemann (reimann.h:33-41) */
typedef struct { double P_M, S_M; crv F; } rout;        /* Riemann_outputs (reimann.h:43-68) */
typedef struct { double G0, G1, G2, G3, G4, G5, G6, G7, G8, G9; int mfv; } gconst; /* reimann.h:1-10 */

static inline double dot3(const double *a, const double *b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }
static inline double nsq3(const double *a) { return a[0] * a[0] + a[1] * a[1] + a[2] * a[2]; }

/* get_wavespeeds_and_pressure_star (reimann.h:485-549) */
static void wavespeeds(const rvec *rv, rout *o, const double *n, double vL, double vR, double cL, double cR, double hL,
                       double hR, double *SLo, double *SRo, double ptl, const gconst *gc)
{
    (void)n;
    double S_L, S_R;
    if ((vR - vL) > DMAX(cL, cR)) {
        o->P_M = MIN_REAL; o->S_M = S_L = S_R = 0;
    } else {
        const double PT_L = rv->L.p, PT_R = rv->R.p;
        S_L = DMIN(vL, vR) - DMAX(cL, cR);
        S_R = DMAX(vL, vR) + DMAX(cL, cR);
        double rho_wt_L = rv->L.rho * (S_L - vL);
        double rho_wt_R = rv->R.rho * (S_R - vR);
        o->S_M = ((PT_R - PT_L) + rho_wt_L * vL - rho_wt_R * vR) / (rho_wt_L - rho_wt_R);
        o->P_M = (PT_L * rho_wt_R - PT_R * rho_wt_L + rho_wt_L * rho_wt_R * (vR - vL)) / (rho_wt_R - rho_wt_L);
        if (o->P_M <= MIN_REAL) { o->P_M = MIN_REAL; o->S_M = S_L = S_R = 0; }
        if ((o->P_M <= 0) || isnan(o->P_M) || (o->P_M > ptl)) {
            const double sL = sqrt(rv->L.rho), sR = sqrt(rv->R.rho);
            const double sinv = 1 / (sL + sR);
            double v_roe[3];
            for (int k = 0; k < 3; k++) v_roe[k] = (rv->L.v[k] * sL + rv->R.v[k] * sR) * sinv;
            const double v_line_roe = dot3(v_roe, n);
            const double h_roe = (sL * hL + sR * hR) * sinv;
            const double cs_roe = sqrt(DMAX(1.e-30, gc->G9 * (h_roe - 0.5 * nsq3(v_roe))));
            S_R = DMAX(vR + cR, v_line_roe + cs_roe);
            S_L = DMIN(vL - cL, v_line_roe - cs_roe);
            rho_wt_R = rv->R.rho * (S_R - vR);
            rho_wt_L = -rv->L.rho * (S_L - vL);
            o->S_M = ((rho_wt_R * vR + rho_wt_L * vL) + (PT_L - PT_R)) / (rho_wt_R + rho_wt_L);
            o->P_M = rv->L.rho * (vL - S_L) * (vL - o->S_M) + PT_L;
            if (o->P_M <= MIN_REAL) { o->P_M = MIN_REAL; o->S_M = S_L = S_R = 0; }
            if ((o->P_M <= 0) || isnan(o->P_M) || (o->P_M > ptl)) {
                o->P_M = 0.5 * ((PT_L + PT_R) + (vL - vR) * 0.25 * (rv->L.rho + rv->R.rho) * (cL + cR));
                o->S_M = 0.5 * (vR + vL) + 2.0 * (PT_L - PT_R) / ((rv->L.rho + rv->R.rho) * (cL + cR));
                const double S_plus = DMAX(DMAX(fabs(vL - cL), fabs(vR - cR)), DMAX(fabs(vL + cL), fabs(vR + cR)));
                S_L = -S_plus; S_R = S_plus;
                if (o->S_M < S_L) o->S_M = S_L;
                if (o->S_M > S_R) o->S_M = S_R;
                if (o->P_M <= MIN_REAL) { o->P_M = MIN_REAL; o->S_M = S_L = S_R = 0; }
            }
        }
    }
    *SLo = S_L;
    *SRo = S_R;
}

/* HLLC_fluxes, MFV (reimann.h:559-615), face frame v_line_frame = 0 */
static void hllc_fluxes(const rvec *rv, rout *o, const double *n, double vL, double vR, double cL, double cR, double hL,
                        double hR, double S_L, double S_R)
{
    (void)cL; (void)cR;
    const double P_M = o->P_M, S_M = o->S_M;
    if ((P_M <= 0) || isnan(P_M)) return;
    double nfac, eK, dv2 = 0, vf = 0;
    {
        const double tol_s = 1.e-12 * (fabs(S_L) + fabs(S_R) + MIN_REAL);
        if ((fabs(S_M - S_L) < tol_s) || (fabs(S_M - S_R) < tol_s) || (fabs(S_M - vf) < tol_s)) {
            o->F.rho = 0;
            o->F.p = o->P_M * o->S_M;
            for (int k = 0; k < 3; k++) o->F.v[k] = n[k] * o->P_M;
            return;
        }
    }
    if (vf < S_L) {
        o->F.rho = rv->L.rho * (vL - vf);
        o->F.p = rv->L.rho * hL * (vL - vf) + rv->L.p * vf;
        for (int k = 0; k < 3; k++) o->F.v[k] = rv->L.v[k] * o->F.rho + n[k] * rv->L.p;
    } else if ((S_L <= vf) && (vf <= S_M)) {
        nfac = rv->L.rho * (S_L - vL) / (S_L - S_M);
        if (nfac < 0) nfac = 0;
        o->F.rho = rv->L.rho * (vL - S_L) + nfac * (S_L - vf);
        eK = rv->L.rho * hL - rv->L.p;
        o->F.p = (rv->L.rho * hL * vL - eK * S_L) +
                 (S_L - vf) * nfac * (eK / rv->L.rho + (S_M - vL) * (S_M + rv->L.p / (rv->L.rho * (S_L - vL))));
        dv2 = nfac * (S_L - vf) * (S_M - vL) + rv->L.p;
        for (int k = 0; k < 3; k++) o->F.v[k] = rv->L.v[k] * o->F.rho + n[k] * dv2;
    } else if ((S_M <= vf) && (vf <= S_R)) {
        nfac = rv->R.rho * (S_R - vR) / (S_R - S_M);
        if (nfac < 0) nfac = 0;
        o->F.rho = rv->R.rho * (vR - S_R) + nfac * (S_R - vf);
        eK = rv->R.rho * hR - rv->R.p;
        o->F.p = (rv->R.rho * hR * vR - eK * S_R) +
                 (S_R - vf) * nfac * (eK / rv->R.rho + (S_M - vR) * (S_M + rv->R.p / (rv->R.rho * (S_R - vR))));
        dv2 = nfac * (S_R - vf) * (S_M - vR) + rv->R.p;
        for (int k = 0; k < 3; k++) o->F.v[k] = rv->R.v[k] * o->F.rho + n[k] * dv2;
    } else {
        o->F.rho = rv->R.rho * (vR - vf);
        o->F.p = rv->R.rho * hR * (vR - vf) + rv->R.p * vf;
        for (int k = 0; k < 3; k++) o->F.v[k] = rv->R.v[k] * o->F.rho + n[k] * rv->R.p;
    }
}

/* Riemann_solver_KurganovTadmor_PWK (reimann.h:445-477), SLOPE_LIMITER_TOLERANCE 1 */
static void riemann_kt(const rvec *rv, rout *o, const double *n, double vL, double vR, double cL, double cR, double hL,
                       double hR, const gconst *gc)
{
    double S_L, S_R, S_M, alpha;
    const double delta_threshold = 0.001 * 0.5 * (rv->L.rho + rv->R.rho) * 0.5 * (cL + cR);
    double dv[3];
    for (int k = 0; k < 3; k++) dv[k] = rv->R.v[k] * rv->R.rho - rv->L.v[k] * rv->L.rho;
    const double dv2 = nsq3(dv);
    const double dvL = fabs(rv->R.rho * vR - rv->L.rho * vL);
    alpha = dvL / sqrt(delta_threshold * delta_threshold + dv2);
    S_L = alpha * cL; if (vL > 0) S_L += vL; else S_L -= vL;
    S_R = alpha * cR; if (vR > 0) S_R += vR; else S_R -= vR;
    S_M = DMAX(S_L, S_R);
    o->S_M = DMAX(cL + fabs(vL), cR + fabs(vR));
    const double f_rho_left = rv->L.rho * (vL + S_M);
    const double f_rho_right = rv->R.rho * (vR - S_M);
    if (gc->mfv) {
        o->P_M = 0.5 * (rv->R.p + rv->L.p);
        o->F.rho = 0.5 * (f_rho_left + f_rho_right);
        for (int k = 0; k < 3; k++) o->F.v[k] = 0.5 * (rv->L.v[k] * f_rho_left + rv->R.v[k] * f_rho_right) + n[k] * o->P_M;
        o->F.p = 0.5 * (f_rho_left * hL + f_rho_right * hR + S_M * (rv->R.p - rv->L.p));
    } else {
        const double denom = 1 / (rv->L.rho * vL - rv->R.rho * vR + S_M * (rv->L.rho + rv->R.rho));
        o->P_M = (f_rho_left * rv->R.p - f_rho_right * rv->L.p) * denom;
        o->F.rho = 0;
        for (int k = 0; k < 3; k++) o->F.v[k] = (rv->R.v[k] - rv->L.v[k]) * (f_rho_left * f_rho_right * denom) + n[k] * o->P_M;
        o->F.p = (S_M * (f_rho_left * rv->R.p + f_rho_right * rv->L.p) + (hR - hL) * f_rho_left * f_rho_right) * denom;
    }
}

/* guess_for_pressure (reimann.h:1025-1062) */
static double guess_pressure(const rvec *rv, double vL, double vR, double cL, double cR, const gconst *gc)
{
    const double pv = 0.5 * (rv->L.p + rv->R.p) - 0.125 * (vR - vL) * (rv->L.p + rv->R.p) * (cL + cR);
    const double pmin = DMIN(rv->L.p, rv->R.p), pmax = DMAX(rv->L.p, rv->R.p);
    if (pmin <= 0) return 0.5 * (pmin + pmax);
    const double qrat = pmax / pmin;
    if (qrat <= 2.0 && (pmin <= pv && pv <= pmax)) return pv;
    if (pv < pmin) {
        const double pnu = (cL + cR) - gc->G7 * (vR - vL);
        const double pde = cL / pow(rv->L.p, gc->G1) + cR / pow(rv->R.p, gc->G1);
        return pow(pnu / pde, gc->G3);
    }
    const double gel = sqrt((gc->G5 / rv->L.rho) / (gc->G6 * rv->L.p + pv));
    const double ger = sqrt((gc->G5 / rv->R.rho) / (gc->G6 * rv->R.p + pv));
    double x = (gel * rv->L.p + ger * rv->R.p - (vR - vL)) / (gel + ger);
    if (x < pmin || x > pmax) x = pmin;
    return x;
}

/* iterative_Riemann_solver (reimann.h:965-1020) */
static int riemann_iterative(const rvec *rv, rout *o, double vL, double vR, double cL, double cR, const gconst *gc)
{
    double Pg, Pg_prev, W_L, W_R, Z_L, Z_R, tol, pratio;
    int niter = 0;
    const double dvel = vR - vL;
    const double check_vel = gc->G4 * (cR + cL) - dvel;
    if (check_vel < 0) return 0;
    tol = 100.0;
    Pg = guess_pressure(rv, vL, vR, cL, cR, gc);
    while ((tol > 1.e-6) && (niter < 1000)) {
        Pg_prev = Pg;
        if (Pg > rv->L.p) {
            const double a0 = gc->G5 / rv->L.rho, a1 = gc->G6 * rv->L.p, a2 = sqrt(a0 / (Pg + a1));
            W_L = (Pg - rv->L.p) * a2;
            Z_L = a2 * (1.0 - 0.5 * (Pg - rv->L.p) / (a1 + Pg));
        } else {
            pratio = Pg / rv->L.p;
            W_L = gc->G4 * cL * (pow(pratio, gc->G1) - 1);
            Z_L = 1 / (rv->L.rho * cL) * pow(Pg / rv->L.p, -gc->G2);
        }
        if (Pg > rv->R.p) {
            const double a0 = gc->G5 / rv->R.rho, a1 = gc->G6 * rv->R.p, a2 = sqrt(a0 / (Pg + a1));
            W_R = (Pg - rv->R.p) * a2;
            Z_R = a2 * (1.0 - 0.5 * (Pg - rv->R.p) / (a1 + Pg));
        } else {
            pratio = Pg / rv->R.p;
            W_R = gc->G4 * cR * (pow(pratio, gc->G1) - 1);
            Z_R = 1 / (rv->R.rho * cR) * pow(pratio, -gc->G2);
        }
        if (niter < 1000 / 2) Pg -= (W_L + W_R + dvel) / (Z_L + Z_R);
        else Pg -= 0.5 * (W_L + W_R + dvel) / (Z_L + Z_R);
        if (Pg < 0.1 * Pg_prev) Pg = 0.1 * Pg_prev;
        tol = 2.0 * fabs((Pg - Pg_prev) / (Pg + Pg_prev));
        niter++;
    }
    if (niter < 1000) {
        o->P_M = Pg;
        o->S_M = 0.5 * (vL + vR) + 0.5 * (W_R - W_L);
        return 1;
    }
    return 0;
}

/* vacuum / fan sampling at S = 0 (reimann.h:672-840) */
static void sample_vac_left(const rvec *rv, rout *o, const double *n, double vR, double cR, const gconst *gc)
{
    const double S = 0.0, S_R = vR - gc->G4 * cR;
    if (!gc->mfv) { o->P_M = 0; o->S_M = S_R; return; }
    if (S_R > S) { o->P_M = 0; o->S_M = S_R; o->F.rho = 0; }
    else {
        if (vR + cR > S) {
            const double C_eff = gc->G5 * (cR - gc->G7 * (vR - S));
            o->P_M = rv->R.p * pow(C_eff / cR, gc->G3);
            o->S_M = gc->G5 * (-cR + gc->G7 * vR + S);
            o->F.rho = rv->R.rho * pow(C_eff / cR, gc->G4);
        } else { o->P_M = rv->R.p; o->S_M = vR; o->F.rho = rv->R.rho; }
    }
    o->F.p = o->P_M;
    for (int k = 0; k < 3; k++) o->F.v[k] = rv->R.v[k] + n[k] * (o->S_M - vR);
}

static void sample_vac_right(const rvec *rv, rout *o, const double *n, double vL, double cL, const gconst *gc)
{
    const double S = 0.0, S_L = vL + gc->G4 * cL;
    if (!gc->mfv) { o->P_M = 0; o->S_M = S_L; return; }
    if (S_L < S) { o->P_M = 0; o->S_M = S_L; o->F.rho = 0; }
    else {
        if (vL - cL < S) {
            const double C_eff = gc->G5 * (cL + gc->G7 * (vL - S));
            o->P_M = rv->L.p * pow(C_eff / cL, gc->G3);
            o->S_M = gc->G5 * (cL + gc->G7 * vL + S);
            o->F.rho = rv->L.rho * pow(C_eff / cL, gc->G4);
        } else { o->P_M = rv->L.p; o->S_M = vL; o->F.rho = rv->L.rho; }
    }
    o->F.p = o->P_M;
    for (int k = 0; k < 3; k++) o->F.v[k] = rv->L.v[k] + n[k] * (o->S_M - vL);
}

static void sample_vac_internal(const rvec *rv, rout *o, const double *n, double vL, double vR, double cL, double cR,
                                const gconst *gc)
{
    const double S = 0.0, S_L = vL + gc->G4 * cL, S_R = vR - gc->G4 * cR;
    if (S <= S_L) sample_vac_right(rv, o, n, vL, cL, gc);
    else if (S >= S_R) sample_vac_left(rv, o, n, vR, cR, gc);
    else {
        o->P_M = 0;
        o->S_M = S;
        if (gc->mfv) {
            o->F.rho = 0;
            o->F.p = o->P_M;
            for (int k = 0; k < 3; k++)
                o->F.v[k] = (rv->L.v[k] + (rv->R.v[k] - rv->L.v[k]) * (S - S_L) / (S_R - S_L)) * (1 - n[k]) + S * n[k];
        }
    }
}

static void sample_standard(const rvec *rv, rout *o, const double *n, double vL, double vR, double cL, double cR,
                            const gconst *gc)
{
    if (!gc->mfv) return;
    const double S = 0.0;
    double C_eff, S_eff;
    if (S <= o->S_M) {
        if (o->P_M <= rv->L.p) {
            if (S <= vL - cL) { o->F.p = rv->L.p; o->F.rho = rv->L.rho; for (int k = 0; k < 3; k++) o->F.v[k] = rv->L.v[k]; return; }
            const double C_eff_L = cL * pow(o->P_M / rv->L.p, gc->G1);
            if (S > o->S_M - C_eff_L) {
                o->F.rho = rv->L.rho * pow(o->P_M / rv->L.p, gc->G8);
                o->F.p = o->P_M;
                for (int k = 0; k < 3; k++) o->F.v[k] = rv->L.v[k] + n[k] * (o->S_M - vL);
                return;
            }
            S_eff = gc->G5 * (cL + gc->G7 * vL + S);
            C_eff = gc->G5 * (cL + gc->G7 * (vL - S));
            o->F.rho = rv->L.rho * pow(C_eff / cL, gc->G4);
            o->F.p = rv->L.p * pow(C_eff / cL, gc->G3);
            for (int k = 0; k < 3; k++) o->F.v[k] = rv->L.v[k] + n[k] * (S_eff - vL);
            return;
        }
        if (rv->L.p > 0) {
            const double pml = o->P_M / rv->L.p;
            const double S_L = vL - cL * sqrt(gc->G2 * pml + gc->G1);
            if (S <= S_L) { o->F.p = rv->L.p; o->F.rho = rv->L.rho; for (int k = 0; k < 3; k++) o->F.v[k] = rv->L.v[k]; return; }
            o->F.rho = rv->L.rho * (pml + gc->G6) / (pml * gc->G6 + 1.0);
            o->F.p = o->P_M;
            for (int k = 0; k < 3; k++) o->F.v[k] = rv->L.v[k] + n[k] * (o->S_M - vL);
            return;
        }
        o->F.rho = rv->L.rho / gc->G6;
        o->F.p = o->P_M;
        for (int k = 0; k < 3; k++) o->F.v[k] = rv->L.v[k] + n[k] * (o->S_M - vL);
        return;
    }
    if (o->P_M > rv->R.p) {
        if (rv->R.p > 0) {
            const double pmr = o->P_M / rv->R.p;
            const double S_R = vR + cR * sqrt(gc->G2 * pmr + gc->G1);
            if (S >= S_R) { o->F.p = rv->R.p; o->F.rho = rv->R.rho; for (int k = 0; k < 3; k++) o->F.v[k] = rv->R.v[k]; return; }
            o->F.rho = rv->R.rho * (pmr + gc->G6) / (pmr * gc->G6 + 1.0);
            o->F.p = o->P_M;
            for (int k = 0; k < 3; k++) o->F.v[k] = rv->R.v[k] + n[k] * (o->S_M - vR);
            return;
        }
        o->F.rho = rv->R.rho / gc->G6;
        o->F.p = o->P_M;
        for (int k = 0; k < 3; k++) o->F.v[k] = rv->R.v[k] + n[k] * (o->S_M - vR);
        return;
    }
    if (S >= vR + cR) { o->F.p = rv->R.p; o->F.rho = rv->R.rho; for (int k = 0; k < 3; k++) o->F.v[k] = rv->R.v[k]; return; }
    const double C_eff_R = cR * pow(o->P_M / rv->R.p, gc->G1);
    if (S <= o->S_M + C_eff_R) {
        o->F.rho = rv->R.rho * pow(o->P_M / rv->R.p, gc->G8);
        o->F.p = o->P_M;
        for (int k = 0; k < 3; k++) o->F.v[k] = rv->R.v[k] + n[k] * (o->S_M - vR);
        return;
    }
    S_eff = gc->G5 * (-cR + gc->G7 * vR + S);
    C_eff = gc->G5 * (cR - gc->G7 * (vR - S));
    o->F.rho = rv->R.rho * pow(C_eff / cR, gc->G4);
    o->F.p = rv->R.p * pow(C_eff / cR, gc->G3);
    for (int k = 0; k < 3; k++) o->F.v[k] = rv->R.v[k] + n[k] * (S_eff - vR);
}

/* convert_face_to_flux (reimann.h:1070-1083) */
static void face_to_flux(rout *o, const double *n, const gconst *gc)
{
    const double rho = o->F.rho, P = o->F.p;
    double v[3] = {o->F.v[0], o->F.v[1], o->F.v[2]};
    const double v_line = dot3(v, n) - 0;
    double h = 0.5 * rho * nsq3(v);
    h += (gc->G0 / gc->G9) * P;
    o->F.p = h * v_line;
    o->F.rho = rho * v_line;
    for (int k = 0; k < 3; k++) o->F.v[k] = v[k] * o->F.rho + n[k] * P;
}

/* Riemann_solver_exact (reimann.h:625-664) */
static void riemann_exact(const rvec *rv, rout *o, const double *n, double vL, double vR, double cL, double cR,
                          const gconst *gc, int *stop)
{
    if ((rv->L.p == 0 && rv->R.p == 0) || (rv->L.rho == 0 && rv->R.rho == 0)) {
        o->P_M = o->S_M = 0;
        if (gc->mfv) { o->F.rho = o->F.p = o->F.v[0] = o->F.v[1] = o->F.v[2] = 0; }
        return;
    }
    if ((rv->L.rho > 0) && (rv->R.rho > 0)) {
        if (riemann_iterative(rv, o, vL, vR, cL, cR, gc)) sample_standard(rv, o, n, vL, vR, cL, cR, gc);
        else sample_vac_internal(rv, o, n, vL, vR, cL, cR, gc);
    } else {
        if ((rv->L.rho < 0) || (rv->R.rho < 0)) { *stop = 1234545; return; }
        if (rv->L.rho > 0) sample_vac_right(rv, o, n, vL, cL, gc);
        if (rv->R.rho > 0) sample_vac_left(rv, o, n, vR, cR, gc);
    }
    if (gc->mfv) face_to_flux(o, n, gc);
}

/* Pair evaluations of the last force pass that took each rare branch of the
 * Riemann cascade (test instrumentation: which fallbacks a case exercises):
 * [0] Kurganov-Tadmor, [1] the exact iterative solver, [2] the second attempt
 * (cell-centred states), [3] the third attempt (at rest). */
static long long g_riemann_branches[4];

void orc_riemann_branches(long long out[4])
{
    for (int k = 0; k < 4; k++) out[k] = g_riemann_branches[k];
}

static void count_branch(int k)
{
#pragma omp atomic
    g_riemann_branches[k]++;
}

/* Riemann_solver, hydro branch (reimann.h:282-370); rv by value as in the reference */
static void riemann_solver(rvec rv, rout *o, const double *n, double ptl, const gconst *gc, int *stop)
{
    if ((rv.L.p < 0 && rv.R.p < 0) || (rv.L.rho < 0) || (rv.R.rho < 0)) { o->P_M = 0; return; }
    rv.L.cs = sqrt(gc->G0 * rv.L.p / rv.L.rho);
    rv.R.cs = sqrt(gc->G0 * rv.R.p / rv.R.rho);
    rv.L.u = rv.L.p / (gc->G9 * rv.L.rho);
    rv.R.u = rv.R.p / (gc->G9 * rv.R.rho);
    const double cL = rv.L.cs, cR = rv.R.cs;
    const double hL = rv.L.p / rv.L.rho + rv.L.u + 0.5 * nsq3(rv.L.v);
    const double hR = rv.R.p / rv.R.rho + rv.R.u + 0.5 * nsq3(rv.R.v);
    const double vL = dot3(rv.L.v, n), vR = dot3(rv.R.v, n);
    /* HLLC_Riemann_solver (reimann.h:382-396) */
    double S_L, S_R;
    wavespeeds(&rv, o, n, vL, vR, cL, cR, hL, hR, &S_L, &S_R, ptl, gc);
    if (gc->mfv) {
        if ((o->P_M >= 0) && (!isnan(o->P_M))) hllc_fluxes(&rv, o, n, vL, vR, cL, cR, hL, hR, S_L, S_R);
    } else {
        o->F.rho = 0;
        for (int k = 0; k < 3; k++) o->F.v[k] = n[k] * o->P_M;
        o->F.p = o->P_M * o->S_M;
    }
    if ((o->P_M < 0) || isnan(o->P_M)) { count_branch(0); riemann_kt(&rv, o, n, vL, vR, cL, cR, hL, hR, gc); }
    if ((o->P_M < 0) || isnan(o->P_M) || (o->P_M > ptl)) {
        count_branch(1);
        riemann_exact(&rv, o, n, vL, vR, cL, cR, gc, stop);
    }
}

/* reconstruct_face_states, non-MHD (reimann.h:125-244) */
static void reconstruct(double Q_i, const double *g_i, double Q_j, const double *g_j, const double *d_i, const double *d_j,
                        double *Q_L, double *Q_R, int mode)
{
    if (mode == 0) { *Q_R = Q_i; *Q_L = Q_j; return; }
    if (Q_i == Q_j) { *Q_L = *Q_R = Q_i; return; }
    *Q_R = Q_i + g_i[0] * d_i[0] + g_i[1] * d_i[1] + g_i[2] * d_i[2];
    *Q_L = Q_j + g_j[0] * d_j[0] + g_j[1] * d_j[1] + g_j[2] * d_j[2];
    double Qmin, Qmax, Qmed, Qmax_eff, Qmin_eff, fac, Qmed_max, Qmed_min;
    const double fac_minmax = 0.5, fac_meddev = 0.375;
    Qmed = 0.5 * (Q_i + Q_j);
    if (Q_i < Q_j) { Qmax = Q_j; Qmin = Q_i; } else { Qmax = Q_i; Qmin = Q_j; }
    fac = fac_minmax * (Qmax - Qmin);
    Qmax_eff = Qmax + fac;
    Qmin_eff = Qmin - fac;
    if (mode > 0) {
        if (Qmax < 0) { if (Qmax_eff > 0) Qmax_eff = Qmax * Qmax / (Qmax - (Qmax_eff - Qmax)); }
        if (Qmin > 0) { if (Qmin_eff < 0) Qmin_eff = Qmin * Qmin / (Qmin + (Qmin - Qmin_eff)); }
    }
    fac = fac_meddev * (Qmax - Qmin);
    Qmed_max = Qmed + fac;
    Qmed_min = Qmed - fac;
    if (Qmed_max > Qmax_eff) Qmed_max = Qmax_eff;
    if (Qmed_min < Qmin_eff) Qmed_min = Qmin_eff;
    if (Q_i < Q_j) {
        if (*Q_R < Qmin_eff) *Q_R = Qmin_eff;
        if (*Q_R > Qmed_max) *Q_R = Qmed_max;
        if (*Q_L > Qmax_eff) *Q_L = Qmax_eff;
        if (*Q_L < Qmed_min) *Q_L = Qmed_min;
    } else {
        if (*Q_R > Qmax_eff) *Q_R = Qmax_eff;
        if (*Q_R < Qmed_min) *Q_R = Qmed_min;
        if (*Q_L < Qmin_eff) *Q_L = Qmin_eff;
        if (*Q_L > Qmed_max) *Q_L = Qmed_max;
    }
}

/* ------------------------------------------------------------------ force */
typedef struct {
    double acc[3], dtE, vsig, dtmass, dmass, gw[3];
} fout;

typedef struct {
    const double *x, *v, *pv, *nvt, *grho, *gp, *gv;
    double m, rho, P, h, cs, cond, fce, drk, dt;
} fside;

static inline void load_side(const orc_state *s, int i, double gamma, fside *f)
{
    f->x = s->pos + 3 * (size_t)i;
    f->v = s->vel + 3 * (size_t)i;
    f->pv = s->pvel + 3 * (size_t)i;
    f->nvt = s->nvt + 6 * (size_t)i;
    f->grho = s->grad_rho + 3 * (size_t)i;
    f->gp = s->grad_p + 3 * (size_t)i;
    f->gv = s->grad_v + 9 * (size_t)i;
    f->m = s->mass[i];
    f->rho = s->rho[i];
    f->P = s->pressure[i];
    f->h = s->h[i];
    f->cs = (f->rho > 0) ? sqrt(gamma * f->P / f->rho) : 0; /* effective_soundspeed (cell_data.h:703-713) */
    f->cond = s->cond[i];
    f->fce = s->fce[i];
    f->drk = s->drkern[i];
    f->dt = s->dt[i];
}

/* hydro_accumulate_neighbor (hydro_functions.h:56-546) with the meshless
 * core (hydro_core_meshless_functions.h:48-616) and the face construction
 * (compute_finitevol_faces_functions.h:46-168) inlined; i is the active
 * (R state), j the neighbour (L state). Returns the MFV j-side dMass write
 * through *dmass_j (0 when none). */
static void force_pair(const gz_params *p, const gconst *gc, const fside *I, const fside *J, fout *out, double *dmass_j,
                       int *stop, double *vsig_pair)
{
    *dmass_j = 0;
    *vsig_pair = -1; /* set below for a pair that reaches the wake-up test (hydro_functions.h:534-544) */
    if (J->m <= 0) return;
    if (J->rho <= 0) return;
    const int kf = p->kernel, mfv = gc->mfv;
    double dp[3] = {I->x[0] - J->x[0], I->x[1] - J->x[1], I->x[2] - J->x[2]};
    wrap3(dp, p->box_size);
    const double r2 = dp[0] * dp[0] + dp[1] * dp[1] + dp[2] * dp[2];
    if ((r2 >= I->h * I->h) && (r2 >= J->h * J->h)) return;
    if (r2 <= 0) return;
    const double r = sqrt(r2);
    const double rinv = 1.0 / r;
    double dv[3] = {I->v[0] - J->v[0], I->v[1] - J->v[1], I->v[2] - J->v[2]};
    double vsig = I->cs + J->cs;
    double hinv_i, hinv3_i, hinv4_i, hinv_j, hinv3_j, hinv4_j;
    double wk_i = 0, dwk_i = 0, wk_j = 0, dwk_j = 0;
    k_hinv(I->h, &hinv_i, &hinv3_i, &hinv4_i);
    if (r < I->h) k_main(kf, r * hinv_i, hinv3_i, hinv4_i, &wk_i, &dwk_i);
    k_hinv(J->h, &hinv_j, &hinv3_j, &hinv4_j);
    if (r < J->h) k_main(kf, r * hinv_j, hinv3_j, hinv4_j, &wk_j, &dwk_j);
    const double cnumcrit2 = ((double)CN_DANGER) * ((double)CN_DANGER) - I->cond * I->cond;
    double eps_big = 0.5, eps_small = 1.e-3;
    if (!mfv && !p->selfgravity_off) { eps_small = 1.e-2; eps_big = 0.6; }
    const double vdotr2 = dot3(dp, dv);
    if (vdotr2 < 0) {
        if (mfv) vsig -= 3 * 1.0 * vdotr2 * rinv;
        else vsig -= 1.0 * vdotr2 * rinv;
    }
    const double V_i = I->m / I->rho;
    double V_j = J->m / J->rho;
    double FAN = 0, FA[3] = {0, 0, 0}, face_vel_i = 0, face_vel_j = 0, face_area_dot_vel = 0;
    crv Fl;
    memset(&Fl, 0, sizeof(Fl));
    rvec rv;
    rout ro;
    memset(&rv, 0, sizeof(rv));
    memset(&ro, 0, sizeof(ro));
    /* ---- meshless core ---- */
    do {
        const double leak_vs_tol = 0.5 * (I->fce + J->fce);
        const double Pressure_i = I->P, Pressure_j = J->P;
        V_j = J->m / J->rho;
        /* compute_finitevol_faces */
        {
            double wt_i = V_i, wt_j = V_j;
            if ((fabs(V_i - V_j) / DMIN(V_i, V_j)) / NDIM > 1.25)
                wt_i = wt_j = V_i * V_j * (wk_i + wk_j) / (V_i * wk_i + V_j * wk_j);
            double ai[3], aj[3];
            sym_matvec(I->nvt, dp, ai);
            sym_matvec(J->nvt, dp, aj);
            const double si = wk_i * wt_i, sj = wk_j * wt_j;
            for (int k = 0; k < 3; k++) FA[k] = (ai[k] * si + aj[k] * sj) * (1.0 * 1.0);
            FAN = nsq3(FA);
            const double fn_dot_dp = dot3(FA, dp);
            if ((J->cond * J->cond > 1.0e12 + cnumcrit2) || (fn_dot_dp < 0)) {
                double fk = -(wt_i * V_i * dwk_i + wt_j * V_j * dwk_j) / r;
                fk *= 1.0 * 1.0;
                for (int k = 0; k < 3; k++) FA[k] = dp[k] * fk;
                FAN = fk * fk * r2;
            }
            FAN = sqrt(FAN);
        }
        if (FAN == 0) { memset(&Fl, 0, sizeof(Fl)); break; }
        double n[3];
        {
            const double inv = 1.0 / FAN;
            for (int k = 0; k < 3; k++) n[k] = FA[k] * inv;
        }
        double s_i = 0.5 * r, s_j = -0.5 * r;
        s_i = 0 - s_i;
        s_j = 0 - s_j;
        double d_i[3], d_j[3];
        for (int k = 0; k < 3; k++) d_i[k] = dp[k] * rinv;
        for (int k = 0; k < 3; k++) { d_j[k] = d_i[k] * s_j; d_i[k] *= s_i; }
        double vframe[3];
        const double *wj = mfv ? J->pv : J->v, *wi = mfv ? I->pv : I->v;
        for (int k = 0; k < 3; k++) vframe[k] = (wj[k] * (-s_i) + wi[k] * s_j) * rinv;
        face_vel_i += dot3(I->v, n);
        face_vel_j += dot3(J->v, n);
        face_vel_i /= 1.0;
        face_vel_j /= 1.0;
        face_area_dot_vel = ((-s_i) * face_vel_j + s_j * face_vel_i) * rinv;
        double v2_approach = 0;
        double vdotr2_phys = vdotr2;
        vdotr2_phys *= 1.0 / (r * 1.0);
        if (vdotr2_phys < 0) v2_approach = vdotr2_phys * vdotr2_phys;
        const double vdotf2_phys = face_vel_i - face_vel_j;
        if (vdotf2_phys < 0) v2_approach = DMAX(v2_approach, vdotf2_phys * vdotf2_phys);
        int recon_mode = 1;
        if (leak_vs_tol > 1) recon_mode = 0;
        const double rho_i = I->rho, rho_j = J->rho, P_i = Pressure_i, P_j = Pressure_j;
        reconstruct(rho_i, I->grho, rho_j, J->grho, d_i, d_j, &rv.L.rho, &rv.R.rho, recon_mode);
        reconstruct(P_i, I->gp, P_j, J->gp, d_i, d_j, &rv.L.p, &rv.R.p, recon_mode);
        for (int k = 0; k < 3; k++)
            reconstruct(I->v[k] - vframe[k], I->gv + 3 * k, J->v[k] - vframe[k], J->gv + 3 * k, d_i, d_j, &rv.L.v[k],
                        &rv.R.v[k], recon_mode);
        const double press_i_tot = Pressure_i + I->rho * v2_approach;
        const double press_j_tot = Pressure_j + J->rho * v2_approach;
        double ptl = 1.1 * 1.0 * DMAX(press_i_tot, press_j_tot);
        if (mfv) ptl *= 2.0;
        if (recon_mode == 0) ptl = DMAX(ptl, DMAX(DMAX(Pressure_i, Pressure_j), 2. * DMAX(I->rho, J->rho) * v2_approach));
        riemann_solver(rv, &ro, n, ptl, gc, stop);
        if ((ro.P_M < 0) || isnan(ro.P_M) || (ro.P_M > 1.4 * ptl)) {
            count_branch(2);
            rv.R.p = Pressure_i; rv.L.p = Pressure_j;
            rv.R.rho = I->rho; rv.L.rho = J->rho;
            for (int k = 0; k < 3; k++) { rv.R.v[k] = I->v[k] - vframe[k]; rv.L.v[k] = J->v[k] - vframe[k]; }
            riemann_solver(rv, &ro, n, 1.4 * ptl, gc, stop);
            if ((ro.P_M < 0) || isnan(ro.P_M)) {
                count_branch(3);
                rv.R.p = Pressure_i; rv.L.p = Pressure_j;
                rv.R.rho = I->rho; rv.L.rho = J->rho;
                for (int k = 0; k < 3; k++) { rv.R.v[k] = 0; rv.L.v[k] = 0; }
                riemann_solver(rv, &ro, n, 2.0 * ptl, gc, stop);
                if ((ro.P_M < 0) || isnan(ro.P_M)) *stop = GZ_ERR_RIEMANN;
            }
        }
        if (!((ro.P_M > 0) && (!isnan(ro.P_M)))) { memset(&Fl, 0, sizeof(Fl)); break; }
        /* de-boost (hydro_core_meshless_functions.h:459-468) */
        ro.F.p += dot3(vframe, ro.F.v);
        if (mfv) {
            ro.F.p += 0.5 * nsq3(vframe) * ro.F.rho;
            for (int k = 0; k < 3; k++) ro.F.v[k] += vframe[k] * ro.F.rho;
        }
        if (mfv) Fl.rho = FAN * ro.F.rho;
        Fl.p = FAN * ro.F.p;
        for (int k = 0; k < 3; k++) Fl.v[k] = ro.F.v[k] * FAN;
        /* MFM face entropic switch (hydro_core_meshless_functions.h:515-574) */
        if (!mfv) {
            const double SM_over_ceff = fabs(ro.S_M) / DMIN(I->cs, J->cs);
            if ((SM_over_ceff < eps_big && 0 >= 0) || (leak_vs_tol > 1)) {
                int use = 1;
                const double facenorm_pm = ro.P_M * FAN;
                const double PdV_fac = ro.P_M * vdotr2_phys / 1.0;
                const double PdV_i = dwk_i * V_i * V_i * I->drk * PdV_fac;
                const double PdV_j = dwk_j * V_j * V_j * J->drk * PdV_fac;
                const double du_old = facenorm_pm * (ro.S_M + face_area_dot_vel);
                const double du_new = 0.5 * (PdV_i - PdV_j + facenorm_pm * (face_vel_i + face_vel_j));
                const double cnum2 = J->cond * J->cond;
                const double ratio = 1.001;
                const double to_i = Pressure_i / I->rho, to_j = Pressure_j / J->rho;
                if (use && SM_over_ceff > eps_small && cnum2 < cnumcrit2) {
                    if (to_i > ratio * to_j) {
                        const double dtoj = -du_old + facenorm_pm * face_vel_j;
                        if (dtoj > 0) use = 0;
                        else { if (dtoj < 0) { if (dtoj > -du_new + facenorm_pm * face_vel_j) use = 0; } }
                    } else if (ratio * to_i < to_j) {
                        const double dtoi = +du_old - facenorm_pm * face_vel_i;
                        if (dtoi > 0) use = 0;
                        else { if (dtoi < 0) { if (dtoi > +du_new - facenorm_pm * face_vel_i) use = 0; } }
                    } else {
                        const double dtoj = -du_old + facenorm_pm * face_vel_j;
                        const double dtoi = +du_old - facenorm_pm * face_vel_i;
                        if (dtoj < 0) { if (dtoj > -du_new + facenorm_pm * face_vel_j) use = 0; }
                        if (dtoi < 0) { if (dtoi > +du_new - facenorm_pm * face_vel_i) use = 0; }
                    }
                }
                if (cnum2 >= cnumcrit2) use = 1;
                if (use) Fl.p += du_new - du_old;
            }
        }
    } while (0);
    /* flux assignment (hydro_functions.h:419-448) */
    if (mfv) {
        double dmass_holder = Fl.rho * I->dt, lim;
        if (dmass_holder > 0) lim = J->m; else lim = I->m;
        lim *= 0.1;
        double accepted = Fl.rho;
        if (fabs(dmass_holder) > lim) {
            accepted *= lim / fabs(dmass_holder);
            dmass_holder *= lim / fabs(dmass_holder);
        }
        if (I->dt < J->dt) out->dmass += dmass_holder;
        else if (I->dt == J->dt) { out->dmass += 0.5 * dmass_holder; accepted *= 0.5; }
        else accepted = 0;
        out->dtmass += Fl.rho;
        for (int k = 0; k < 3; k++) out->gw[k] += dp[k] * accepted;
    }
    for (int k = 0; k < 3; k++) out->acc[k] += Fl.v[k];
    out->dtE += Fl.p;
    const double vsig_ts = vsig + fabs(I->cs - J->cs);
    if (vsig_ts > out->vsig) out->vsig = vsig_ts;
    *vsig_pair = vsig_ts;
    if (mfv) {
        /* j-side write (hydro_functions.h:511-532) */
        double dmass_holder = Fl.rho * I->dt, lim;
        if (dmass_holder > 0) lim = J->m; else lim = I->m;
        lim *= 0.1;
        if (fabs(dmass_holder) > lim) dmass_holder *= lim / fabs(dmass_holder);
        if (I->dt < J->dt) *dmass_j = -dmass_holder;
        else if (I->dt == J->dt) *dmass_j = -0.5 * dmass_holder;
    }
}

static void make_gconst(const gz_params *p, gconst *gc)
{
    const double G0 = p->gamma;
    gc->G0 = G0;
    gc->G1 = (G0 - 1.0) / (2.0 * G0);
    gc->G2 = (G0 + 1.0) / (2.0 * G0);
    gc->G3 = (2.0 * G0 / (G0 - 1.0));
    gc->G4 = 2.0 / (G0 - 1.0);
    gc->G5 = 2.0 / (G0 + 1.0);
    gc->G6 = (G0 - 1.0) / (G0 + 1.0);
    gc->G7 = 0.5 * (G0 - 1.0);
    gc->G8 = 1.0 / G0;
    gc->G9 = G0 - 1.0;
    gc->mfv = p->method == GZ_METHOD_MFV;
}

int orc_force(const gz_params *p, orc_state *s, const int *active, int n_active, int n_threads)
{
    return orc_force_wakeup(p, s, active, n_active, n_threads, NULL);
}

#define WAKEUP 4.1 /* declarations/constants.h:11-13 (SLOPE_LIMITER_TOLERANCE > 0, no GR) */

int orc_force_wakeup(const gz_params *p, orc_state *s, const int *active, int n_active, int n_threads,
                     const int *bin_active)
{
    set_threads(n_threads);
    int *all = NULL;
    if (!active) { all = all_indices(s->n); active = all; n_active = s->n; }
    gconst gc;
    make_gconst(p, &gc);
    const int mfv = gc.mfv;
    for (int k = 0; k < 4; k++) g_riemann_branches[k] = 0;
    /* preloop (hydro_toplevel.cc:457-565) */
    for (int a = 0; a < n_active; a++) {
        const int i = active[a];
        s->vsig[i] = MIN_REAL;
        s->dudt[i] = 0;
        for (int k = 0; k < 3; k++) s->accel[3 * (size_t)i + k] = 0;
        if (mfv) { s->dtmass[i] = 0; s->dmass[i] = 0; for (int k = 0; k < 3; k++) s->gravwork[3 * (size_t)i + k] = 0; }
    }
    orc_grid g;
    if (orc_grid_build(&g, s->pos, s->h, s->n, p->box_size)) { free(all); return GZ_ERR_ARG; }
    int status = 0;
    fout *outs = (fout *)calloc((size_t)(n_active > 0 ? n_active : 1), sizeof(fout));
#pragma omp parallel
    {
        int *cand = NULL, cap = 0;
#pragma omp for schedule(dynamic, 16)
        for (int a = 0; a < n_active; a++) {
            const int i = active[a];
            if (!(s->mass[i] > 0 && s->rho[i] > 0)) continue; /* HydroForceSpec enabled gate */
            fside I, J;
            load_side(s, i, p->gamma, &I);
            fout *o = outs + a;
            if (o->vsig < I.cs) o->vsig = I.cs;
            int stop = 0;
            const int nc = orc_grid_candidates(&g, I.x, I.h, 1, &cand, &cap);
            for (int c = 0; c < nc; c++) {
                const int j = cand[c];
                if (j == i) continue;
                load_side(s, j, p->gamma, &J);
                double dmj, vsig_pair;
                force_pair(p, &gc, &I, &J, o, &dmj, &stop, &vsig_pair);
                if (mfv && dmj != 0) {
#pragma omp atomic
                    s->dmass[j] += dmj;
                }
                /* wake-up (hydro_functions.h:534-544): an inactive neighbour whose stored signal
                 * speed is too slow for this pair is flagged with this target's bin + 1
                 * (wakeup_flag_from_timebin, core/proto.h:181) */
                if (bin_active && vsig_pair >= 0 && !bin_active[s->timebin[j]] &&
                    vsig_pair > WAKEUP * s->vsig[j]) {
                    const int w = s->timebin[i] + 1;
#pragma omp critical(orc_wakeup)
                    { if (s->wakeup[j] < w) s->wakeup[j] = w; }
                }
            }
            if (stop) {
#pragma omp critical
                { if (!status) status = stop; }
            }
        }
        free(cand);
    }
    /* writeback (hydro_force_loop.cc:227-391) + final operations (hydro_toplevel.cc:133-253) */
    for (int a = 0; a < n_active; a++) {
        const int i = active[a];
        const fout *o = outs + a;
        double *ac = s->accel + 3 * (size_t)i;
        for (int k = 0; k < 3; k++) ac[k] += o->acc[k];
        s->dudt[i] += o->dtE;
        if (mfv) {
            s->dtmass[i] += o->dtmass;
            s->dmass[i] += o->dmass;
            for (int k = 0; k < 3; k++) s->gravwork[3 * (size_t)i + k] += o->gw[k];
        }
        const double cs_i = (s->rho[i] > 0) ? sqrt(p->gamma * s->pressure[i] / s->rho[i])
                                            : sqrt(p->gamma * (p->gamma - 1.) * s->u[i]);
        const double max_sig = fmax(o->vsig, cs_i);
        if (s->vsig[i] < max_sig) s->vsig[i] = max_sig;
    }
    for (int a = 0; a < n_active; a++) {
        const int i = active[a];
        if (!(s->mass[i] > 0)) continue;
        const double *v = s->vel + 3 * (size_t)i;
        double *ac = s->accel + 3 * (size_t)i;
        if (mfv) {
            const double *pv = s->pvel + 3 * (size_t)i;
            const double d[3] = {v[0] - pv[0], v[1] - pv[1], v[2] - pv[2]};
            const double v2_p = s->vsig[i] * s->vsig[i] + nsq3(d);
            s->vsig[i] = sqrt(v2_p);
        }
        double vp[3];
        {
            const double inv = 1.0 / 1.0;
            for (int k = 0; k < 3; k++) vp[k] = v[k] * inv;
        }
        s->dudt[i] -= dot3(vp, ac);
        if (mfv) {
            s->dudt[i] += 0.5 * nsq3(vp) * s->dtmass[i];
            for (int k = 0; k < 3; k++) ac[k] -= vp[k] * s->dtmass[i];
        }
        {
            const double inv = 1.0 / s->mass[i];
            for (int k = 0; k < 3; k++) ac[k] *= inv;
        }
        if (mfv) s->dudt[i] -= s->u[i] * s->dtmass[i];
        s->dudt[i] /= s->mass[i];
        if (mfv) {
            const double inv = 1.0 / s->mass[i];
            for (int k = 0; k < 3; k++) s->gravwork[3 * (size_t)i + k] *= inv;
        }
        if (s->h[i] >= 0.99 * p->max_kernel_radius) s->dudt[i] = 0;
    }
    free(outs);
    orc_grid_free(&g);
    free(all);
    return status;
}

/* ------------------------------------------------------------ neighbour sets */
static int cmp_int(const void *a, const void *b)
{
    const int x = *(const int *)a, y = *(const int *)b;
    return (x > y) - (x < y);
}

int orc_neighbors(const gz_params *p, const orc_state *s, const int *active, int n_active, int mode, orc_csr *out,
                  int n_threads)
{
    set_threads(n_threads);
    int *all = NULL;
    if (!active) { all = all_indices(s->n); active = all; n_active = s->n; }
    orc_grid g;
    if (orc_grid_build(&g, s->pos, s->h, s->n, p->box_size)) { free(all); return GZ_ERR_ARG; }
    int **rows = (int **)calloc((size_t)(n_active > 0 ? n_active : 1), sizeof(int *));
    int *cnt = (int *)calloc((size_t)(n_active > 0 ? n_active : 1), sizeof(int));
    const double box = p->box_size;
#pragma omp parallel
    {
        int *cand = NULL, cap = 0;
#pragma omp for schedule(dynamic, 16)
        for (int a = 0; a < n_active; a++) {
            const int i = active[a];
            const double *xi = s->pos + 3 * (size_t)i;
            const double hi = s->h[i];
            const int nc = orc_grid_candidates(&g, xi, hi, mode, &cand, &cap);
            int *row = (int *)malloc(sizeof(int) * (size_t)(nc > 0 ? nc : 1));
            int k = 0;
            for (int c = 0; c < nc; c++) {
                const int j = cand[c];
                double dp[3] = {xi[0] - s->pos[3 * (size_t)j], xi[1] - s->pos[3 * (size_t)j + 1], xi[2] - s->pos[3 * (size_t)j + 2]};
                wrap3(dp, box);
                const double r2 = dp[0] * dp[0] + dp[1] * dp[1] + dp[2] * dp[2];
                if (mode == 0) {
                    if (r2 < hi * hi) row[k++] = j;
                } else {
                    const double hj = s->h[j];
                    if (r2 > 0 && !((r2 >= hi * hi) && (r2 >= hj * hj))) row[k++] = j;
                }
            }
            qsort(row, (size_t)k, sizeof(int), cmp_int);
            rows[a] = row;
            cnt[a] = k;
        }
        free(cand);
    }
    out->n_rows = n_active;
    out->offsets = (long long *)malloc(sizeof(long long) * (size_t)(n_active + 1));
    out->offsets[0] = 0;
    for (int a = 0; a < n_active; a++) out->offsets[a + 1] = out->offsets[a] + cnt[a];
    out->nbrs = (int *)malloc(sizeof(int) * (size_t)(out->offsets[n_active] > 0 ? out->offsets[n_active] : 1));
    for (int a = 0; a < n_active; a++) {
        memcpy(out->nbrs + out->offsets[a], rows[a], sizeof(int) * (size_t)cnt[a]);
        free(rows[a]);
    }
    free(rows);
    free(cnt);
    orc_grid_free(&g);
    free(all);
    return 0;
}

void orc_csr_free(orc_csr *c)
{
    free(c->offsets);
    free(c->nbrs);
    c->offsets = NULL;
    c->nbrs = NULL;
    c->n_rows = 0;
}

double orc_full_pass_seconds(const gz_params *p, orc_state *s, const int *active, int n_active, int n_threads, int *status)
{
    struct timespec t0, t1;
    clock_gettime(CLOCK_MONOTONIC, &t0);
    int st = orc_density(p, s, active, n_active, n_threads);
    if (!st) st = orc_gradients(p, s, active, n_active, n_threads);
    if (!st) st = orc_force(p, s, active, n_active, n_threads);
    clock_gettime(CLOCK_MONOTONIC, &t1);
    if (status) *status = st;
    return (double)(t1.tv_sec - t0.tv_sec) + 1e-9 * (double)(t1.tv_nsec - t0.tv_nsec);
}

/* -------------------------------------------------------------------- kick */
/* do_the_kick (core/kicks.cc:284-545) for gas cells of the configuration
 * above (non-comoving: cf_atime = cf_a2inv = cf_hubble_a = 1; no timestep
 * dilation, cooling, entropy switch, special boundaries or extra physics):
 *   MFV conserved-mass update      kicks.cc:290-323
 *   thermal update                 kicks.cc:331-358, 466-478, with
 *     internal_energy_positivity_catch (core/proto.h:417-421, no u_floor)
 *     and enforce_temperature_floor (declarations/cell_data.h:604-611)
 *   momentum kick                  kicks.cc:480-490
 *   mass check, predicted reset    kicks.cc:521-543
 * unit_integertime_in_physical is Timebase_interval (core/timestep_functions.h:43-46)
 * and the non-comoving gravkick factor is (time1 - time0) * Timebase_interval
 * (timestep_functions.h:203-206, 253-256). Vec3 updates are per component.
 * The loops of do_first/second_halfstep_kick (kicks.cc:59-77, 144-162) kick
 * only particles with P.Mass > 0; so does this. */
int orc_kick(const gz_params *p, orc_kick_state *k, int mode, double timebase, double min_egy_spec)
{
    const int mfv = p->method == GZ_METHOD_MFV;
    for (int i = 0; i < k->n; i++) {
        if (!(k->mass[i] > 0)) continue; /* the loops call do_the_kick only then: kicks.cc:69, 153 */
        double mass_old, mass_pred, mass_new;
        mass_old = mass_pred = mass_new = k->mass[i];
        const long long span = k->tend[i] - k->tstart[i];
        if (mfv && k->dmass[i] != 0) {
            double dm = 0;
            if (mode != 0) {
                dm = ((double)span * timebase) * k->dtmass[i];
                if (dm * k->dmass[i] < 0) dm = 0;
                if (fabs(dm) > fabs(k->dmass[i])) dm = k->dmass[i];
                k->dmass[i] -= dm;
            } else {
                dm = k->dmass[i];
            }
            if (dm < -0.99 * k->mass_true[i]) dm = -0.99 * k->mass_true[i];
            mass_old = k->mass_true[i];
            mass_pred = k->mass[i];
            mass_new = mass_old + dm;
            k->mass_true[i] = mass_new;
            if (mode == 0) k->dmass[i] = 0;
        }
        if (!k->active[i]) continue;

        const double dt_hydro = (double)span * timebase;
        const double dt_grav = (double)span * timebase;
        const double *g = k->grav + 3 * (size_t)i;
        double dent_grav = 0;
        if (mfv) {
            const double *w = k->gravwork + 3 * (size_t)i;
            dent_grav += (w[0] * g[0] + w[1] * g[1] + w[2] * g[2]) * dt_hydro;
        }
        const double du_tot = k->dudt[i] * dt_hydro + dent_grav;
        const double dent = k->u[i] + du_tot;
        k->u[i] = (dent < 0.5 * k->u[i]) ? 0.5 * k->u[i] : dent;
        if (min_egy_spec != 0 && k->u[i] < min_egy_spec) {
            k->u[i] = min_egy_spec;
            k->dudt[i] = 0;
        }

        double dp[3];
        const double *a = k->accel + 3 * (size_t)i;
        for (int c = 0; c < 3; c++) {
            dp[c] = 0;
            dp[c] += g[c] * (mass_pred * dt_grav);
            dp[c] += a[c] * (mass_pred * dt_hydro);
        }
        const double inv_mass = 1.0 / mass_new;
        double *v = k->vel + 3 * (size_t)i;
        for (int c = 0; c < 3; c++) v[c] += dp[c] * inv_mass;
        if (k->mass[i] <= 0 || !isfinite(k->mass[i])) continue;
        if (mode == 1) {
            for (int c = 0; c < 3; c++) k->vel_pred[3 * (size_t)i + c] = v[c];
            if (mfv) k->mass[i] = k->mass_true[i];
            k->u_pred[i] = k->u[i];
        }
        for (int c = 0; c < 3; c++) k->dp[3 * (size_t)i + c] += dp[c];
    }
    return 0;
}

/* ------------------------------------------------------------------- drift */
/* drift_particle_impl (core/drift_particle_functions.h:86-260) for gas cells
 * of the configuration above, HYDRO_FIX_MESH_MOTION = 5 (declarations/
 * precompiler_logic.h:78), no timestep dilation, no special boundaries:
 *   time checks                         drift_particle_functions.h:90-97
 *   position step: MFV with ParticleVel (advect_mesh_point_body, core/
 *     timestep_functions.h:979), MFM with Vel (particle_drift_velocity,
 *     drift_straight_displacement, timestep_functions.h:649-652)
 *   capped log change, radius factor    timestep_functions.h:312, 323-335
 *   VelPred, MFV mass (mfv_drifted_mass, timestep_functions.h:993-996),
 *   density, InternalEnergyPred with internal_energy_positivity_catch
 *   (core/proto.h:417-421) and the MinEgySpec floor, kernel radius and its
 *   clamps                              drift_particle_functions.h:158-233
 *   ideal-gas pressure (gamma - 1) u rho  eos/eos_functions.h:873 (set_eos_pressure_impl)
 * The drift factor, the gravkick factor and the hydro kick time are all
 * (time1 - time0) * Timebase_interval here (timestep_functions.h:43-46, 203-206). */
int orc_drift(const gz_params *p, orc_drift_state *d, long long time1, double timebase, double min_egy_spec)
{
    const int mfv = p->method == GZ_METHOD_MFV;
    int code = 0;
    for (int i = 0; i < d->n; i++) {
        const long long time0 = d->ti_current[i];
        if (time1 < time0) {
            if (!code) code = GZ_ERR_NO_PAST_DRIFT;
            continue;
        }
        if (time1 == time0) continue;
        const double dt_drift = (double)(time1 - time0) * timebase;
        double *x = d->pos + 3 * (size_t)i;
        const double *w = mfv ? d->pvel + 3 * (size_t)i : d->vel + 3 * (size_t)i;
        for (int c = 0; c < 3; c++) x[c] += w[c] * dt_drift;

        double lc = d->divvel[i] * dt_drift;
        if (lc > 0.3) lc = 0.3;
        if (lc < -0.3) lc = -0.3;
        const double h_fac = exp(lc / 3.0);

        if (d->mass[i] > 0) {
            const double dt_entr = (double)(time1 - time0) * timebase;
            double *vp = d->vel_pred + 3 * (size_t)i;
            const double *g = d->grav + 3 * (size_t)i;
            const double *a = d->accel + 3 * (size_t)i;
            for (int c = 0; c < 3; c++) vp[c] += g[c] * dt_drift + a[c] * dt_entr;
            if (mfv) {
                const double m = d->mass[i] + d->dtmass[i] * dt_entr;
                const double lo = 0.5 * d->mass_true[i];
                d->mass[i] = m > lo ? m : lo;
            }
            d->rho[i] *= exp(-lc);
            const double etmp = d->u_pred[i] + d->dudt[i] * dt_entr;
            d->u_pred[i] = (etmp < 0.5 * d->u_pred[i]) ? 0.5 * d->u_pred[i] : etmp;
            if (d->u_pred[i] < min_egy_spec) d->u_pred[i] = min_egy_spec;
            d->h[i] *= h_fac;
            if (d->h[i] < p->min_kernel_radius) d->h[i] = p->min_kernel_radius;
            if (d->h[i] > p->max_kernel_radius) d->h[i] = p->max_kernel_radius;
            d->pressure[i] = (p->gamma - 1) * d->u_pred[i] * d->rho[i];
        }
        d->ti_current[i] = time1;
    }
    return code;
}

/* ---------------------------------------------------------------- timestep */
#define ORC_TIMEBINS 60
#define ORC_TIMEBASE (((long long)1) << ORC_TIMEBINS) /* declarations/typedefs.h:8-9 */

/* get_timestep_bin (core/timestep.cc:1525-1545): the bin whose integer step is ti_step. */
static int orc_timestep_bin(long long ti_step)
{
    if (ti_step == 0) return 0;
    int bin = -1;
    while (ti_step) {
        bin++;
        ti_step >>= 1;
    }
    return bin;
}

/* get_timestep (core/timestep.cc:357-1416) as it compiles for gas cells of
 * this configuration: cf_a2inv = cf_atime = cf_hubble_a = 1, no PM, no
 * dilation, STOP_WHEN_BELOW_MINTIMESTEP, dt_displacement = MaxSizeTimestep
 * (find_dt_displacement_constraint, timestep.cc:1425-1434, non-comoving):
 *   acceleration criterion   :421-487 (KERNEL_CORE_SIZE of the kernel)
 *   Courant criterion         :711-729 (Get_Particle_Size, declarations/particle_data.h:461-469)
 *   divergence criterion      :1093-1098
 *   caps, floor, integer step :1334-1414
 * then the per-particle binning of find_timesteps (:176-215, 265-270): a power
 * of two below the wanted step, a larger bin only where it is synchronised. */
int orc_timestep(const gz_params *p, const orc_timestep_params *tp, orc_timestep_state *t)
{
    /* KERNEL_CORE_SIZE: 1/2 for the cubic spline, 2/5 for Wendland C2 (mesh/kernel.h:59, 113) */
    const double core = p->kernel == GZ_KERNEL_CUBIC ? (1.0 / 2.0) : (2.0 / 5.0);
    int code = 0;
    const double tb = tp->timebase;
    for (int i = 0; i < t->n; i++) {
        const double *g = t->grav + 3 * (size_t)i;
        const double *a = t->accel + 3 * (size_t)i;
        double ax = 1.0 * g[0], ay = 1.0 * g[1], az = 1.0 * g[2];
        ax += a[0];
        ay += a[1];
        az += a[2];
        double ac = sqrt(ax * ax + ay * ay + az * az);
        t->aphys[i] = ac;
        if (ac == 0) ac = 1.0e-30;
        double h_acc = core * t->softening[i];
        if (h_acc <= 0) h_acc = (1.61199 * t->h[i] / t->num_ngb[i]) * 1.0;
        double dt = sqrt(2 * tp->err_tol_int_accuracy * 1.0 * h_acc / ac);
        if (t->mass[i] > 0) {
            const double csnd = 0.5 * t->vsig[i];
            const double L = 1.61199 * t->h[i] / t->num_ngb[i];
            const double dt_courant = tp->courant_fac * (L * 1.0) / csnd;
            if (dt_courant < dt) dt = dt_courant;
            const double divv = t->divvel[i];
            if (divv != 0) {
                const double dt_divv = 1.5 / fabs(1.0 * divv);
                if (dt_divv < dt) dt = dt_divv;
            }
        }
        dt *= 1.0;
        if (dt >= tp->max_size_timestep) dt = tp->max_size_timestep;
        if (dt >= tp->max_size_timestep) dt = tp->max_size_timestep; /* dt_displacement */
        if ((dt < tp->min_size_timestep) || !(dt / tb >= 2.0)) {
            if (t->mass[i] > 0 && !code) code = 888;
            dt = tp->min_size_timestep;
        }
        if (dt > 0.5 * ORC_TIMEBASE * tb) dt = 0.5 * ORC_TIMEBASE * tb;
        long long ti_step = (long long)(dt / tb);
        if (ti_step <= 1) ti_step = 2;
        if (!(ti_step > 0 && ti_step < ORC_TIMEBASE)) ti_step = 2;
        t->ti_want[i] = ti_step;

        ti_step = (long long)(((double)ti_step) / 1.0);
        long long ti_min = ORC_TIMEBASE;
        while (ti_min > ti_step) ti_min >>= 1;
        ti_step = ti_min;
        int bin = orc_timestep_bin(ti_step);
        const int binold = t->bin[i];
        if (bin > binold) {
            while (tp->bin_active[bin] == 0 && bin > binold) bin--;
            ti_step = bin ? ((long long)1 << bin) : 0;
        }
        if (tp->ti_current >= ORC_TIMEBASE) {
            ti_step = 0;
            bin = 0;
        }
        if ((ORC_TIMEBASE - tp->ti_current) < ti_step) {
            if (!code) code = 90001005;
            ti_step = ORC_TIMEBASE - tp->ti_current;
            ti_min = ORC_TIMEBASE;
            while (ti_min > ti_step) ti_min >>= 1;
            ti_step = ti_min;
        }
        t->bin[i] = bin;
        t->ti_begstep[i] += t->dt_step[i];
        t->dt_step[i] = ti_step;
    }
    return code;
}


/* ------------------------------------------------------------- active sets */
/* make_list_of_active_particles (core/run.cc:997-1010): the cells whose
 * TimeBin is active and whose mass is positive, here in ascending index order
 * (the reference walks the bins' linked lists; the passes do not depend on the
 * order). Returns the count; out may be NULL. */
int orc_active_list(int n, const int *timebin, const double *mass, const int *bin_active, int *out)
{
    int k = 0;
    for (int i = 0; i < n; i++) {
        if (bin_active[timebin[i]] && mass[i] > 0) {
            if (out) out[k] = i;
            k++;
        }
    }
    return k;
}

/* The new timebin of each cell the last force pass woke up (P.wakeup > 0), by
 * the rule of process_wake_ups (core/timestep.cc:1565-1700) for gas: the
 * waker's bin (wakeup_timebin_from_flag, core/proto.h:182) less the bins that
 * WAKEUP spans (the smallest k with 2^k >= WAKEUP), floored at the lowest
 * occupied active bin, capped at the highest bin active at the next kick, and
 * never above the cell's own bin; active cells and cells without mass keep
 * theirs. The linked-list moves, the step truncation and the kicks that
 * follow stay with the caller. Returns the number of cells moved. */
int orc_wakeup_bins(int n, const int *timebin, const int *wakeup, const double *mass, const int *bin_active,
                    int max_time_bin_active, int lowest_occupied_active_bin, int *out)
{
    int offset = 0;
    while ((1ll << offset) < (long long)WAKEUP) offset++;
    int moved = 0;
    for (int i = 0; i < n; i++) {
        int bin = timebin[i];
        out[i] = bin;
        if (!wakeup[i] || !(mass[i] > 0)) continue;
        const int binold = timebin[i];
        if (bin_active[binold]) continue;
        if (wakeup[i] > 0) {
            const int waker_bin = wakeup[i] - 1;
            bin = waker_bin - offset > 0 ? waker_bin - offset : 0;
            if (bin < lowest_occupied_active_bin) bin = lowest_occupied_active_bin;
        } else {
            bin = max_time_bin_active;
        }
        if (bin > max_time_bin_active) bin = max_time_bin_active;
        if (bin >= binold) bin = binold;
        out[i] = bin;
        if (bin != binold) moved++;
    }
    return moved;
}

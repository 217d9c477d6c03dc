// gizmo_b200/csrc/kick.cu -- the half-step kick (gz_kick in include/gizmo_hydro.h).
//
// do_the_kick (core/kicks.cc:284-545) for gas cells of the build this library
// serves: non-comoving (cf_atime = cf_a2inv = cf_hubble_a = 1), no timestep
// dilation, no cooling, no entropy switch, no special boundaries. One thread
// per particle over the caller's own device arrays; the update is a handful
// of FP64 operations per ~330 bytes moved, so the kernel is HBM-bound and its
// only design points are coalesced access and a grid that fills the SMs.
//
// Built with -fmad=false: every product and sum rounds as the reference
// writes it, so the result is bit-identical to the reference's kick.
#include <cuda_runtime.h>

#include <cmath>

#include "../../include/gizmo_hydro.h"

namespace {

constexpr int kKickBlock = 256;

struct KickArgs {
    gz_kick_fields f;
    int mode;
    int mfv;
    double timebase;
    double min_egy_spec;
};

// kicks.cc:290-323 (MFV conserved mass), :331-358 and :466-478 (thermal
// update through internal_energy_positivity_catch, core/proto.h:417-421, and
// enforce_temperature_floor, declarations/cell_data.h:604-611), :480-490
// (momentum), :521-543 (mass check and the predicted values after the second
// half kick). unit_integertime_in_physical and the non-comoving gravkick
// factor are both (tend - tstart) * Timebase_interval
// (core/timestep_functions.h:43-46, 203-206, 253-256).
__global__ void __launch_bounds__(kKickBlock) k_kick(const KickArgs a)
{
    const gz_kick_fields &f = a.f;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < f.n; i += stride) {
        // Every input of the particle is loaded before the first branch on loaded data, so that
        // all of its loads are in flight together; the branches below only choose what is stored.
        const double mass = f.mass[i];
        const int64_t t0 = f.tstart[i], t1 = f.tend[i];
        const int active = f.active ? f.active[i] : 1;
        double mass_true = 0, dmass = 0, dtmass = 0;
        if (a.mfv) {
            mass_true = f.mass_true[i];
            dmass = f.dmass[i];
            dtmass = f.dtmass[i];
        }
        double g[3] = {0, 0, 0}, w[3] = {0, 0, 0}, acc[3], vel[3], dp_old[3];
#pragma unroll
        for (int c = 0; c < 3; c++) {
            if (f.grav) g[c] = f.grav[3 * i + c];
            if (a.mfv && f.gravwork) w[c] = f.gravwork[3 * i + c];
            acc[c] = f.accel[3 * i + c];
            vel[c] = f.vel[3 * i + c];
            dp_old[c] = f.dp[3 * i + c];
        }
        const double u_old = f.u[i];
        const double dudt = f.dudt[i];

        if (!(mass > 0)) continue;  // the kick loops skip these cells (kicks.cc:69, 153)
        const double mass_pred = mass;
        double mass_new = mass;
        const double dt = (double)(t1 - t0) * a.timebase;
        if (a.mfv && dmass != 0) {
            double dm;
            if (a.mode != 0) {
                dm = dt * dtmass;
                if (dm * dmass < 0) dm = 0;
                if (fabs(dm) > fabs(dmass)) dm = dmass;
                dmass -= dm;
            } else {
                dm = dmass;
                dmass = 0;
            }
            if (dm < -0.99 * mass_true) dm = -0.99 * mass_true;
            mass_new = mass_true + dm;
            mass_true = mass_new;
            f.mass_true[i] = mass_true;
            f.dmass[i] = dmass;
        }
        if (!active) continue;

        double dent_grav = 0;
        if (a.mfv) dent_grav += (w[0] * g[0] + w[1] * g[1] + w[2] * g[2]) * dt;
        const double du_tot = dudt * dt + dent_grav;
        const double dent = u_old + du_tot;
        double u = (dent < 0.5 * u_old) ? 0.5 * u_old : dent;
        if (a.min_egy_spec != 0 && u < a.min_egy_spec) {
            u = a.min_egy_spec;
            f.dudt[i] = 0;
        }
        f.u[i] = u;

        const double inv_mass = 1.0 / mass_new;
        double dp[3], v[3];
#pragma unroll
        for (int c = 0; c < 3; c++) {
            dp[c] = 0;
            dp[c] += g[c] * (mass_pred * dt);
            dp[c] += acc[c] * (mass_pred * dt);
            v[c] = vel[c] + dp[c] * inv_mass;
            f.vel[3 * i + c] = v[c];
        }
        if (mass <= 0 || !isfinite(mass)) continue;
        if (a.mode == 1) {
#pragma unroll
            for (int c = 0; c < 3; c++) f.vel_pred[3 * i + c] = v[c];
            if (a.mfv) f.mass[i] = mass_true;
            f.u_pred[i] = u;
        }
#pragma unroll
        for (int c = 0; c < 3; c++) f.dp[3 * i + c] = dp_old[c] + dp[c];
    }
}

}  // namespace

extern "C" int gz_kick(const gz_params *params, const gz_kick_fields *f, int mode, double timebase,
                       double min_egy_spec, void *stream)
{
    if (!params || !f || f->n < 0 || (mode != 0 && mode != 1)) return GZ_ERR_ARG;
    if (params->method != GZ_METHOD_MFM && params->method != GZ_METHOD_MFV) return GZ_ERR_ARG;
    if (!(timebase >= 0) || !std::isfinite(timebase) || !std::isfinite(min_egy_spec)) return GZ_ERR_ARG;
    if (f->n == 0) return GZ_OK;
    if (!f->vel || !f->u || !f->mass || !f->accel || !f->dudt || !f->vel_pred || !f->u_pred || !f->dp ||
        !f->tstart || !f->tend)
        return GZ_ERR_ARG;
    const int mfv = params->method == GZ_METHOD_MFV;
    if (mfv && (!f->mass_true || !f->dmass || !f->dtmass)) return GZ_ERR_ARG;
    int dev = 0, sms = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return GZ_ERR_NO_DEVICE;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || sms <= 0)
        return GZ_ERR_CUDA;
    KickArgs a;
    a.f = *f;
    a.mode = mode;
    a.mfv = mfv;
    a.timebase = timebase;
    a.min_egy_spec = min_egy_spec;
    // one wave of resident blocks at most: the grid-stride loop takes the rest
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_kick, kKickBlock, 0) != cudaSuccess || per_sm <= 0)
        return GZ_ERR_CUDA;
    const int64_t want = (f->n + kKickBlock - 1) / kKickBlock;
    const int64_t cap = (int64_t)sms * per_sm;
    const int blocks = (int)(want < cap ? want : cap);
    k_kick<<<blocks, kKickBlock, 0, (cudaStream_t)stream>>>(a);
    return cudaGetLastError() == cudaSuccess ? GZ_OK : GZ_ERR_CUDA;
}

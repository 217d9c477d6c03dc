// gizmo_b200/csrc/drift.cu -- the drift (gz_drift in include/gizmo_hydro.h).
//
// drift_particle_impl (core/drift_particle_functions.h:86-260) for the gas
// cells of the build this library serves: non-comoving, no timestep dilation,
// ideal gas, HYDRO_FIX_MESH_MOTION = 5 (an MFV cell moves with its smoothed
// ParticleVel, an MFM cell with its velocity), no special boundaries. One
// thread per cell over the caller's own device arrays; ~300 bytes and two
// exponentials per cell, so the kernel is HBM-bound. As in the kick, every
// input of a cell is loaded before the first branch on loaded data, so that
// all of its loads are in flight together.
//
// Built with -fmad=false; the two exponentials are the correctly rounded
// gz::cr::exp, so every field matches the reference's arithmetic bit for bit
// wherever its libm exp rounds correctly.
#include <cuda_runtime.h>

#include <cmath>

#include "../../include/gizmo_hydro.h"
#include "crmath.cuh"

namespace {

constexpr int kDriftBlock = 256;
constexpr double kMaxLogChange = 0.3;  // KERNEL_RADIUS_DRIFT_MAX_LOG_CHANGE, core/timestep_functions.h:312

struct DriftArgs {
    gz_drift_fields f;
    int64_t time1;
    int mfv;
    double timebase;
    double min_egy_spec;
    double min_h, max_h, gamma_m1;
};

// drift_particle_functions.h:90-97 (time checks), :106-112 with
// advect_mesh_point_body / drift_straight_displacement (timestep_functions.h:979,
// 649-652: the position step), :115-116 with timestep_functions.h:323-335 (the
// capped log change and radius factor), :158-233 (VelPred, mfv_drifted_mass
// timestep_functions.h:993-996, density, InternalEnergyPred through
// internal_energy_positivity_catch core/proto.h:417-421 and the MinEgySpec
// floor, kernel radius and its clamps), :235 set_eos_pressure_impl (ideal gas,
// eos/eos_functions.h:873). The drift factor, the gravkick factor and the hydro
// kick time are all (time1 - time0) * Timebase_interval here.
__global__ void __launch_bounds__(kDriftBlock) k_drift(const DriftArgs a)
{
    const gz_drift_fields &f = a.f;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < f.n; i += stride) {
        const int64_t time0 = f.ti_current[i];
        const double mass = f.mass[i];
        const double divvel = f.divvel[i];
        double x[3], w[3], vp[3], g[3] = {0, 0, 0}, acc[3];
        const double *move = a.mfv ? f.pvel : f.vel;
#pragma unroll
        for (int c = 0; c < 3; c++) {
            x[c] = f.pos[3 * i + c];
            w[c] = move[3 * i + c];
            vp[c] = f.vel_pred[3 * i + c];
            if (f.grav) g[c] = f.grav[3 * i + c];
            acc[c] = f.accel[3 * i + c];
        }
        double dtmass = 0, mass_true = 0;
        if (a.mfv) {
            dtmass = f.dtmass[i];
            mass_true = f.mass_true[i];
        }
        const double rho = f.rho[i];
        const double u_pred = f.u_pred[i];
        const double dudt = f.dudt[i];
        const double h = f.h[i];

        if (a.time1 < time0) {
            atomicCAS(f.status, 0, GZ_ERR_NO_PAST_DRIFT);
            continue;
        }
        if (a.time1 == time0) continue;
        const double dt = (double)(a.time1 - time0) * a.timebase;
#pragma unroll
        for (int c = 0; c < 3; c++) f.pos[3 * i + c] = x[c] + w[c] * dt;

        double lc = divvel * dt;
        if (lc > kMaxLogChange) lc = kMaxLogChange;
        if (lc < -kMaxLogChange) lc = -kMaxLogChange;

        if (mass > 0) {
#pragma unroll
            for (int c = 0; c < 3; c++) f.vel_pred[3 * i + c] = vp[c] + (g[c] * dt + acc[c] * dt);
            if (a.mfv) {
                const double m = mass + dtmass * dt;
                const double lo = 0.5 * mass_true;
                f.mass[i] = m > lo ? m : lo;
            }
            const double rho_new = rho * gz::cr::exp(-lc);
            f.rho[i] = rho_new;
            const double etmp = u_pred + dudt * dt;
            double u = (etmp < 0.5 * u_pred) ? 0.5 * u_pred : etmp;
            if (u < a.min_egy_spec) u = a.min_egy_spec;
            f.u_pred[i] = u;
            double h_new = h * gz::cr::exp(lc / 3.0);
            if (h_new < a.min_h) h_new = a.min_h;
            if (h_new > a.max_h) h_new = a.max_h;
            f.h[i] = h_new;
            f.pressure[i] = a.gamma_m1 * u * rho_new;
        }
        f.ti_current[i] = a.time1;
    }
}

}  // namespace

extern "C" int gz_drift(const gz_params *params, const gz_drift_fields *f, int64_t time1, double timebase,
                        double min_egy_spec, void *stream)
{
    if (!params || !f || f->n < 0) return GZ_ERR_ARG;
    if (params->method != GZ_METHOD_MFM && params->method != GZ_METHOD_MFV) return GZ_ERR_ARG;
    if (!(timebase >= 0) || !std::isfinite(timebase) || !std::isfinite(min_egy_spec)) return GZ_ERR_ARG;
    if (f->n == 0) return GZ_OK;
    const int mfv = params->method == GZ_METHOD_MFV;
    if (!f->pos || !(mfv ? f->pvel : f->vel) || !f->vel_pred || !f->accel || !f->divvel || !f->mass || !f->rho ||
        !f->u_pred || !f->dudt || !f->h || !f->pressure || !f->ti_current || !f->status)
        return GZ_ERR_ARG;
    if (mfv && (!f->dtmass || !f->mass_true)) return GZ_ERR_ARG;
    int dev = 0, sms = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return GZ_ERR_NO_DEVICE;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || sms <= 0)
        return GZ_ERR_CUDA;
    DriftArgs a;
    a.f = *f;
    a.time1 = time1;
    a.mfv = mfv;
    a.timebase = timebase;
    a.min_egy_spec = min_egy_spec;
    a.min_h = params->min_kernel_radius;
    a.max_h = params->max_kernel_radius;
    a.gamma_m1 = params->gamma - 1;
    // one wave of resident blocks at most: the grid-stride loop takes the rest
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_drift, kDriftBlock, 0) != cudaSuccess || per_sm <= 0)
        return GZ_ERR_CUDA;
    const int64_t want = (f->n + kDriftBlock - 1) / kDriftBlock;
    const int64_t cap = (int64_t)sms * per_sm;
    const int blocks = (int)(want < cap ? want : cap);
    k_drift<<<blocks, kDriftBlock, 0, (cudaStream_t)stream>>>(a);
    return cudaGetLastError() == cudaSuccess ? GZ_OK : GZ_ERR_CUDA;
}

// gizmo_b200/csrc/timestep.cu -- the timestep criterion (gz_timestep in include/gizmo_hydro.h).
//
// get_timestep (core/timestep.cc:357-1416) for gas cells of the build this
// library serves -- non-comoving (cf_atime = cf_a2inv = cf_hubble_a = 1), no
// PM step, no timestep dilation, STOP_WHEN_BELOW_MINTIMESTEP, and the
// displacement limit of find_dt_displacement_constraint (timestep.cc:
// 1425-1434) equal to MaxSizeTimestep as it is without comoving integration --
// followed by the per-particle binning of find_timesteps (timestep.cc:176-215,
// 265-270): the largest power of two not above the wanted step, a larger bin
// only where it is synchronised, and the end of the timeline. One thread per
// cell over the caller's own device arrays, like gz_kick and gz_drift; the
// criteria read the force pass's outputs (HydroAccel, MaxSignalVel,
// Particle_DivVel) and the density pass's (KernelRadius, NumNgb).
//
// Built with -fmad=false: the products, sums, the square roots and divisions
// round as the reference writes them (IEEE in both), so the integer steps and
// bins are the reference's exactly.
#include <cuda_runtime.h>

#include <cmath>

#include "../../include/gizmo_hydro.h"

namespace {

constexpr int kStepBlock = 256;
constexpr long long kTimebase = 1ll << GZ_TIMEBINS;  // TIMEBASE, declarations/typedefs.h:8-9

struct StepArgs {
    gz_timestep_fields f;
    gz_timestep_params tp;
    double core;  // KERNEL_CORE_SIZE: 1/2 cubic, 2/5 Wendland C2 (mesh/kernel.h:59, 113)
};

// get_timestep_bin (core/timestep.cc:1525-1545): the bin whose integer step is ti_step
__device__ int step_bin(long long ti_step)
{
    if (ti_step == 0) return 0;
    int bin = -1;
    while (ti_step) {
        bin++;
        ti_step >>= 1;
    }
    return bin;
}

__device__ void record(int32_t *status, int code)
{
    if (status) atomicCAS(status, 0, code);
}

__global__ void __launch_bounds__(kStepBlock) k_timestep(const StepArgs a)
{
    const gz_timestep_fields &f = a.f;
    const gz_timestep_params &tp = a.tp;
    const double tb = tp.timebase;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < f.n; i += stride) {
        double g[3] = {0, 0, 0}, acc[3];
#pragma unroll
        for (int c = 0; c < 3; c++) {
            if (f.grav) g[c] = f.grav[3 * i + c];
            acc[c] = f.accel[3 * i + c];
        }
        const double vsig = f.vsig[i], h = f.h[i], num_ngb = f.num_ngb[i], divv = f.divvel[i], mass = f.mass[i];
        const double soft = f.softening ? f.softening[i] : 0.0;
        const int binold = f.bin[i];
        const long long ti_begstep = f.ti_begstep[i], dt_step = f.dt_step[i];

        // acceleration criterion (timestep.cc:421-487)
        double ax = 1.0 * g[0], ay = 1.0 * g[1], az = 1.0 * g[2];
        ax += acc[0];
        ay += acc[1];
        az += acc[2];
        double ac = sqrt(ax * ax + ay * ay + az * az);
        if (f.aphys) f.aphys[i] = ac;
        if (ac == 0) ac = 1.0e-30;
        double h_acc = a.core * soft;
        if (h_acc <= 0) h_acc = (1.61199 * h / num_ngb) * 1.0;  // Get_Particle_Size (particle_data.h:461-469)
        double dt = sqrt(2 * tp.err_tol_int_accuracy * 1.0 * h_acc / ac);
        if (mass > 0) {
            // Courant criterion (timestep.cc:711-729) and the divergence limit (:1093-1098)
            const double csnd = 0.5 * vsig;
            const double L = 1.61199 * h / num_ngb;
            const double dt_courant = tp.courant_fac * (L * 1.0) / csnd;
            if (dt_courant < dt) dt = dt_courant;
            if (divv != 0) {
                const double dt_divv = 1.5 / fabs(1.0 * divv);
                if (dt_divv < dt) dt = dt_divv;
            }
        }
        // caps, floor and the integer step (timestep.cc:1334-1414)
        dt *= 1.0;
        if (dt >= tp.max_size_timestep) dt = tp.max_size_timestep;
        if (dt >= tp.max_size_timestep) dt = tp.max_size_timestep;  // the displacement limit
        if ((dt < tp.min_size_timestep) || !(dt / tb >= 2.0)) {
            if (mass > 0) record(f.status, 888);
            dt = tp.min_size_timestep;
        }
        if (dt > 0.5 * (double)kTimebase * tb) dt = 0.5 * (double)kTimebase * tb;
        long long ti_step = (long long)(dt / tb);
        if (ti_step <= 1) ti_step = 2;
        if (!(ti_step > 0 && ti_step < kTimebase)) ti_step = 2;
        if (f.ti_want) f.ti_want[i] = ti_step;

        // the per-particle binning of find_timesteps (timestep.cc:176-215, 265-270)
        ti_step = (long long)(((double)ti_step) / 1.0);
        long long ti_min = kTimebase;
        while (ti_min > ti_step) ti_min >>= 1;
        ti_step = ti_min;
        int bin = step_bin(ti_step);
        if (bin > binold) {
            while (tp.bin_active[bin] == 0 && bin > binold) bin--;
            ti_step = bin ? (1ll << bin) : 0;
        }
        if (tp.ti_current >= kTimebase) {
            ti_step = 0;
            bin = 0;
        }
        if ((kTimebase - tp.ti_current) < ti_step) {
            record(f.status, GZ_ERR_END_OF_TIMELINE);
            ti_step = kTimebase - tp.ti_current;
            ti_min = kTimebase;
            while (ti_min > ti_step) ti_min >>= 1;
            ti_step = ti_min;
        }
        f.bin[i] = bin;
        f.ti_begstep[i] = ti_begstep + dt_step;
        f.dt_step[i] = ti_step;
    }
}

}  // namespace

extern "C" int gz_timestep(const gz_params *params, const gz_timestep_params *tp, const gz_timestep_fields *f,
                           void *stream)
{
    if (!params || !tp || !f || f->n < 0) return GZ_ERR_ARG;
    if (params->kernel != GZ_KERNEL_CUBIC && params->kernel != GZ_KERNEL_WENDLAND_C2) return GZ_ERR_ARG;
    if (!(tp->timebase > 0) || !std::isfinite(tp->timebase) || tp->ti_current < 0) return GZ_ERR_ARG;
    if (f->n == 0) return GZ_OK;
    if (!f->accel || !f->vsig || !f->h || !f->num_ngb || !f->divvel || !f->mass || !f->bin || !f->ti_begstep ||
        !f->dt_step)
        return GZ_ERR_ARG;
    int dev = 0, sms = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return GZ_ERR_NO_DEVICE;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || sms <= 0)
        return GZ_ERR_CUDA;
    StepArgs a;
    a.f = *f;
    a.tp = *tp;
    a.core = params->kernel == GZ_KERNEL_CUBIC ? (1.0 / 2.0) : (2.0 / 5.0);
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_timestep, kStepBlock, 0) != cudaSuccess ||
        per_sm <= 0)
        return GZ_ERR_CUDA;
    const int64_t want = (f->n + kStepBlock - 1) / kStepBlock;
    const int64_t cap = (int64_t)sms * per_sm;
    const int blocks = (int)(want < cap ? want : cap);
    k_timestep<<<blocks, kStepBlock, 0, (cudaStream_t)stream>>>(a);
    return cudaGetLastError() == cudaSuccess ? GZ_OK : GZ_ERR_CUDA;
}

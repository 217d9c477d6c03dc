// gizmo_b200/csrc/noalloc.cu -- density sums for callers that cannot allocate
// device memory (gz_density_sums_noalloc in include/gizmo_hydro.h).
//
// Some callers own all device memory themselves -- a host code whose memory
// pool has reserved the device, or a loop that cannot accept the device-wide
// synchronisation a cudaMalloc/cudaFree implies -- and so cannot use a
// gz_context, which allocates its buffers. This entry point computes the same
// fixed-h density sums as gz_density_sums for a particle set that the caller
// already holds in device memory, and allocates nothing: its only scratch is
// the packed neighbour-record array below, a file-scope device array of
// kMaxParticles records (4 MiB) that every GPU loading this library holds
// until the process exits.
//
// The neighbour loop is all-pairs (the set is small by construction), tiled
// through shared memory; the pair arithmetic is the one of k_density_sums in
// FP64 (this file is built with -fmad=false like passes_fp64.cu), so the sums
// agree with gz_density_sums up to summation order.
#include <cuda_runtime.h>

#include <mutex>

#include "../../include/gizmo_hydro.h"
#include "state.cuh"

using namespace gz;

namespace {

constexpr int kMaxParticles = GZ_NOALLOC_MAX_PARTICLES;
constexpr int kTile = 128;
constexpr int kMaxDevices = 128;

// The only scratch of the entry point: one packed record per particle of the
// current call. Shared by every call on a device; fully rewritten by each call
// for the particles it covers, so nothing in it needs clearing.
static __device__ __align__(256) DensRec g_records[kMaxParticles];

std::mutex g_setup_mutex;
DensRec *g_records_ptr[kMaxDevices] = {};  // device address of g_records, per device

__global__ void k_noalloc_pack(int n, const double *__restrict__ pos, const double *__restrict__ vel,
                               const double *__restrict__ mass, DensRec *rec)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    DensRec r;
    r.x = pos[3 * (size_t)i]; r.y = pos[3 * (size_t)i + 1]; r.z = pos[3 * (size_t)i + 2];
    r.m = mass[i];
    r.vx = vel[3 * (size_t)i]; r.vy = vel[3 * (size_t)i + 1]; r.vz = vel[3 * (size_t)i + 2];
    r.pad = 0.0;
    rec[i] = r;
}

// One thread per target; every particle of the set is a candidate, streamed
// through shared memory kTile records at a time and accepted on r^2 < h^2
// (DensitySpec::pair_kernel, density_loop.h:1140-1385).
__global__ void __launch_bounds__(kTile) k_noalloc_density_sums(PassParams p, int n, const double *__restrict__ pos,
                                                                 const double *__restrict__ vel,
                                                                 const double *__restrict__ hs,
                                                                 const DensRec *__restrict__ rec, double *acc,
                                                                 double *pv)
{
    __shared__ DensRec tile[kTile];
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const bool valid = i < n;
    double xi = 0, yi = 0, zi = 0, hd = 0, vix = 0, viy = 0, viz = 0;
    if (valid) {
        xi = pos[3 * (size_t)i]; yi = pos[3 * (size_t)i + 1]; zi = pos[3 * (size_t)i + 2];
        vix = vel[3 * (size_t)i]; viy = vel[3 * (size_t)i + 1]; viz = vel[3 * (size_t)i + 2];
        hd = hs[i];
    }
    const double h2 = hd * hd;
    double hinv = 0, hinv3 = 0, hinv4 = 0;
    if (valid) k_hinv(hd, hinv, hinv3, hinv4);
    const int mfv = p.method == 1;
    double a[17];
#pragma unroll
    for (int k = 0; k < 17; k++) a[k] = 0;
    for (int t0 = 0; t0 < n; t0 += kTile) {
        if (t0 + (int)threadIdx.x < n) tile[threadIdx.x] = rec[t0 + threadIdx.x];
        __syncthreads();
        const int m = min(kTile, n - t0);
        if (valid) {
            for (int k = 0; k < m; k++) {
                const DensRec rj = tile[k];
                if (rj.m <= 0) continue;
                double dx, dy, dz;
                const double r2 = sep2(xi, yi, zi, rj.x, rj.y, rj.z, p.box, p.half, dx, dy, dz);
                if (r2 >= h2) continue;
                const double r = sqrt(r2);
                const double u = r * hinv;
                double wk, dwk;
                k_main(p.kernel, u, hinv3, hinv4, wk, dwk);
                const double mj_wk = rj.m * wk;
                a[0] += wk;
                a[1] += mj_wk;
                if (mfv && r == 0.0) {
                    a[14] += mj_wk * rj.vx;
                    a[15] += mj_wk * rj.vy;
                    a[16] += mj_wk * rj.vz;
                }
                a[2] += -(3.0 * hinv * wk + u * dwk);
                if (r > 0.0) {
                    a[4] += dx * dx * wk;
                    a[5] += dy * dy * wk;
                    a[6] += dz * dz * wk;
                    a[7] += dx * dy * wk;
                    a[8] += dy * dz * wk;
                    a[9] += dx * dz * wk;
                    a[10] += wk * dx;
                    a[11] += wk * dy;
                    a[12] += wk * dz;
                    const double dvx = vix - rj.vx, dvy = viy - rj.vy, dvz = viz - rj.vz;
                    if (mfv) {
                        a[14] += mj_wk * (vix - dvx);
                        a[15] += mj_wk * (viy - dvy);
                        a[16] += mj_wk * (viz - dvz);
                    }
                    a[3] -= dwk * (dx * dvx + dy * dvy + dz * dvz) / r;
                }
            }
        }
        __syncthreads();
    }
    if (!valid) return;
#pragma unroll
    for (int k = 0; k < 13; k++) acc[14 * (size_t)i + k] = a[k];
    acc[14 * (size_t)i + 13] = 0.0;
    if (pv)
        for (int k = 0; k < 3; k++) pv[3 * (size_t)i + k] = a[14 + k];
}

// Device address of g_records on the current device, looked up once per
// device (host code must not pass the symbol itself: on the host it names a
// stand-in, not device memory).
int records_address(DensRec **out)
{
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return GZ_ERR_NO_DEVICE;
    if (dev < 0 || dev >= kMaxDevices) return GZ_ERR_ARG;
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    if (!g_records_ptr[dev]) {
        void *p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_records);
        if (e != cudaSuccess || !p) return GZ_ERR_CUDA;
        g_records_ptr[dev] = (DensRec *)p;
    }
    *out = g_records_ptr[dev];
    return GZ_OK;
}

}  // namespace

extern "C" int gz_density_sums_noalloc(const gz_params *params, int n, const double *pos, const double *vel,
                                       const double *mass, const double *h, double *acc, double *pv, void *stream)
{
    if (!params || n < 0) return GZ_ERR_ARG;
    if (params->kernel != GZ_KERNEL_CUBIC && params->kernel != GZ_KERNEL_WENDLAND_C2) return GZ_ERR_ARG;
    if (params->method != GZ_METHOD_MFM && params->method != GZ_METHOD_MFV) return GZ_ERR_ARG;
    if (!(params->box_size > 0)) return GZ_ERR_ARG;
    if (n > kMaxParticles) return GZ_ERR_CAPACITY;
    if (n == 0) return GZ_OK;
    if (!pos || !vel || !mass || !h || !acc) return GZ_ERR_ARG;
    DensRec *rec = nullptr;
    const int rc = records_address(&rec);
    if (rc) return rc;
    PassParams p{};
    p.kernel = params->kernel;
    p.method = params->method;
    p.first_step = params->first_step;
    p.selfgravity_off = params->selfgravity_off;
    p.box = params->box_size;
    p.half = 0.5 * params->box_size;
    p.gamma = params->gamma;
    p.des_num_ngb = params->des_num_ngb;
    p.max_num_ngb_dev = params->max_num_ngb_dev;
    p.min_kernel_radius = params->min_kernel_radius;
    p.max_kernel_radius = params->max_kernel_radius;
    cudaStream_t s = (cudaStream_t)stream;
    const unsigned blocks = (unsigned)((n + kTile - 1) / kTile);
    k_noalloc_pack<<<blocks, kTile, 0, s>>>(n, pos, vel, mass, rec);
    k_noalloc_density_sums<<<blocks, kTile, 0, s>>>(p, n, pos, vel, h, rec, acc, pv);
    return cudaGetLastError() == cudaSuccess ? GZ_OK : GZ_ERR_CUDA;
}

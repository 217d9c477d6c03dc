// gizmo_b200/csrc/passes.cuh -- the three pair kernels, templated on pair arithmetic T.
//
// Included by passes_fp64.cu (T = double, built without FMA contraction) and
// passes_mixed.cu (T = float). Layout: a group of TPT consecutive lanes owns
// one target row; lanes stride over the row's neighbours, gather neighbour
// fields from the sorted SoA mirror (Morton order keeps them in L1/L2),
// evaluate the pair in T, accumulate in FP64 registers and combine with
// __shfl_xor within the group. Lane 0 of the group runs the per-particle
// epilogue (finalize) in FP64.
#pragma once

#include <cooperative_groups.h>

#include "launch.h"

namespace gz {

// Stores one record per thread of the block, for the consecutive particles
// [first, first + count), through shared memory, so that the block writes one
// contiguous run with 16-byte stores instead of each lane a record-sized stride.
// Every thread of the block takes part (it synchronises the block).
template <typename R>
GZ_DEV void store_block_records(R *dst, const R &r, int first, int count, int4 *smem)
{
    static_assert(sizeof(R) % 16 == 0, "records are whole 16-byte words");
    constexpr int kWords = (int)(sizeof(R) / 16);
    if ((int)threadIdx.x < count) reinterpret_cast<R *>(smem)[threadIdx.x] = r;
    __syncthreads();
    int4 *out = reinterpret_cast<int4 *>(dst + first);
    for (int k = threadIdx.x; k < count * kWords; k += blockDim.x) out[k] = smem[k];
    __syncthreads();
}

constexpr int kPackBlock = 128;

// ---------------------------------------------------------------- density
// DensitySpec::pair_kernel (density_loop.h:1140-1385), gas i, gas j; the
// row is a superset (buffered radius) and r2 < h^2 is re-tested exactly.
constexpr int kDensityBlock = 128;

// A record through the read-only data path, in 16-byte pieces.
template <typename R> GZ_DEV R ldg_record(const R *__restrict__ p)
{
    static_assert(sizeof(R) % 16 == 0, "records are whole 16-byte words");
    R r;
    int4 *d = reinterpret_cast<int4 *>(&r);
    const int4 *s = reinterpret_cast<const int4 *>(p);
#pragma unroll
    for (int k = 0; k < (int)(sizeof(R) / 16); k++) d[k] = __ldg(s + k);
    return r;
}

// A neighbour's density record through the read-only data path, in 16-byte
// pieces, without its padding word.
GZ_DEV DensRec load_dens_rec(const DensRec *__restrict__ rec, int j)
{
    const double2 *q = reinterpret_cast<const double2 *>(rec + j);
    const double2 q0 = __ldg(q), q1 = __ldg(q + 1), q2 = __ldg(q + 2);
    DensRec r;
    r.x = q0.x; r.y = q0.y; r.z = q1.x; r.m = q1.y; r.vx = q2.x; r.vy = q2.y;
    r.vz = __ldg(reinterpret_cast<const double *>(q + 3));
    r.pad = 0.0;
    return r;
}

// The sums of target t's density row, by the TPT lanes (`lane` of them, on
// `mask`) that own it; lane 0 stores them.
template <typename T, int TPT>
GZ_DEV void density_row(const PassParams &p, const Particles &ps, const DensityWork &w, int t, int lane,
                        unsigned mask)
{
    const double xi = ps.x[t], yi = ps.y[t], zi = ps.z[t];
    const double hd = ps.h[t];
    const double h2 = hd * hd;
    const T h = T(hd);
    T hinv, hinv3, hinv4;
    k_hinv(h, hinv, hinv3, hinv4);
    const T vix = T(ps.vx[t]), viy = T(ps.vy[t]), viz = T(ps.vz[t]);
    const int mfv = p.method == 1;
    double a[17];
#pragma unroll
    for (int k = 0; k < 17; k++) a[k] = 0;
    // one neighbour's contribution; the lane visits its entries in row order
    auto pair = [&](const DensRec &rj) {
        const double mjd = rj.m;
        if (mjd <= 0) return;
        double dx, dy, dz;
        const double r2 = sep2(xi, yi, zi, rj.x, rj.y, rj.z, p.box, p.half, dx, dy, dz);
        if (r2 >= h2) return;
        const T r = Real<T>::sqrt_(T(r2));
        const T u = r * hinv;
        T wk, dwk;
        k_main(p.kernel, u, hinv3, hinv4, wk, dwk);
        const T mj = T(mjd);
        const T mj_wk = mj * wk;
        a[0] += (double)wk;
        a[1] += (double)mj_wk;
        const T vjx = T(rj.vx), vjy = T(rj.vy), vjz = T(rj.vz);
        if (mfv && r == T(0)) {
            a[14] += (double)(mj_wk * vjx);
            a[15] += (double)(mj_wk * vjy);
            a[16] += (double)(mj_wk * vjz);
        }
        a[2] += (double)(-(T(3) * hinv * wk + u * dwk));
        if (r > T(0)) {
            const T px = T(dx), py = T(dy), pz = T(dz);
            a[4] += (double)(px * px * wk);
            a[5] += (double)(py * py * wk);
            a[6] += (double)(pz * pz * wk);
            a[7] += (double)(px * py * wk);
            a[8] += (double)(py * pz * wk);
            a[9] += (double)(px * pz * wk);
            a[10] += (double)(wk * px);
            a[11] += (double)(wk * py);
            a[12] += (double)(wk * pz);
            const T dvx = vix - vjx, dvy = viy - vjy, dvz = viz - vjz;
            if (mfv) {
                a[14] += (double)(mj_wk * (vix - dvx));
                a[15] += (double)(mj_wk * (viy - dvy));
                a[16] += (double)(mj_wk * (viz - dvz));
            }
            a[3] -= (double)(dwk * (px * dvx + py * dvy + pz * dvz) / r);
        }
    };
    // one record in flight per lane: the register budget goes to resident
    // warps (six 128-thread blocks per multiprocessor), which hide the
    // gather latency better than a second record per lane does; the next
    // entry's index is loaded a step ahead, so the record load does not wait
    // on it
    const long long b0 = w.beg[t], b1 = w.end[t];
    const int *__restrict__ nbr = w.nbr;
    long long e = b0 + lane;
    int j = e < b1 ? __ldg(nbr + e) : 0;
    for (; e < b1; e += TPT) {
        const long long en = e + TPT;
        const int jn = en < b1 ? __ldg(nbr + en) : 0;
        pair(load_dens_rec(w.rec, j));
        j = jn;
    }
#pragma unroll
    for (int k = 0; k < 17; k++) a[k] = warp_sum(a[k], mask, TPT);
    if (lane == 0) {
        const size_t n = (size_t)ps.n;
#pragma unroll
        for (int k = 0; k < 17; k++) w.acc[k * n + t] = a[k];
    }
}

template <typename T, int TPT>
__global__ void __launch_bounds__(kDensityBlock, 6) k_density_sums(PassParams p, Particles ps, DensityWork w)
{
    const int gtid = blockIdx.x * blockDim.x + threadIdx.x;
    const int slot = gtid / TPT, lane = gtid % TPT;
    if (slot >= w.n_todo) return;
    const unsigned mask = (TPT == 32) ? 0xffffffffu : (((1u << TPT) - 1u) << ((threadIdx.x & 31) & ~(TPT - 1)));
    density_row<T, TPT>(p, ps, w, w.todo[slot], lane, mask);
}

// The same rows for a captured pass: the iteration's target count and lane
// count come from the device state. A fixed number of blocks stand in for the
// plain launch's grid: each takes the next block-sized chunk of rows (the
// plain grid's next block) from a counter, so the rows in flight are a
// contiguous run of the list and the chunks go to whichever block is free, as
// the hardware hands out the blocks of a plain launch. An instance whose TPT
// is not the iteration's returns at once. Each row is summed by the same
// lanes in the same order as k_density_sums sums it.
template <typename T, int TPT>
__global__ void __launch_bounds__(kDensityBlock, 6) k_density_sums_graph(PassParams p, Particles ps, DensityWork w,
                                                                         GraphState *gs,
                                                                         const int *__restrict__ todo)
{
    __shared__ int s_chunk;
    if (gs->fail || gs->tpt != TPT) return;
    const int n_todo = gs->n_todo;
    constexpr int kRows = kDensityBlock / TPT;
    const unsigned mask = (TPT == 32) ? 0xffffffffu : (((1u << TPT) - 1u) << ((threadIdx.x & 31) & ~(TPT - 1)));
    const int lane = threadIdx.x % TPT;
    for (;;) {
        if (threadIdx.x == 0) s_chunk = atomicAdd(&gs->sums_next, 1);
        __syncthreads();
        const int chunk = s_chunk;
        __syncthreads();  // read by every thread before the next draw
        if ((long long)chunk * kRows >= n_todo) break;
        const int slot = chunk * kRows + (int)threadIdx.x / TPT;
        if (slot < n_todo) density_row<T, TPT>(p, ps, w, todo[slot], lane, mask);
    }
}

template <typename T>
void launch_density_sums(const PassParams &p, const Particles &ps, const DensityWork &w, int tpt, cudaStream_t s)
{
    if (w.n_todo <= 0) return;
    const long long threads = (long long)w.n_todo * tpt;
    const unsigned blocks = (unsigned)((threads + kDensityBlock - 1) / kDensityBlock);
    switch (tpt) {
        case 4: k_density_sums<T, 4><<<blocks, kDensityBlock, 0, s>>>(p, ps, w); break;
        case 8: k_density_sums<T, 8><<<blocks, kDensityBlock, 0, s>>>(p, ps, w); break;
        case 32: k_density_sums<T, 32><<<blocks, kDensityBlock, 0, s>>>(p, ps, w); break;
        default: k_density_sums<T, 16><<<blocks, kDensityBlock, 0, s>>>(p, ps, w); break;
    }
}

// -------------------------------------------------------------- gradients
// What a gradient row reads of each neighbour: position, h, mass, density,
// pressure and velocity, all FP64 (80 bytes). The pair takes the differences
// q_j - q_i in FP64 and only then rounds them to the pair type: in a smooth
// field q_j and q_i agree to many digits, and rounding them to FP32 first
// would keep only the few that differ.
template <typename T> struct __align__(16) GradRec {
    double x, y, z, h, m, rho;
    double P, vx, vy, vz;
};

template <typename T> __global__ void __launch_bounds__(kPackBlock) k_pack_gradient(Particles ps, GradRec<T> *rec)
{
    extern __shared__ int4 s_pack[];
    const int first = blockIdx.x * blockDim.x;
    const int i = first + threadIdx.x;
    GradRec<T> r{};
    if (i < ps.n) {
        r.x = ps.x[i]; r.y = ps.y[i]; r.z = ps.z[i]; r.h = ps.h[i]; r.m = ps.m[i]; r.rho = ps.rho[i];
        r.P = ps.pressure[i]; r.vx = ps.vx[i]; r.vy = ps.vy[i]; r.vz = ps.vz[i];
    }
    store_block_records(rec, r, first, min((int)blockDim.x, ps.n - first), s_pack);
}

// gradient_accumulate_neighbor (gradient_functions.h:304-665) + the
// finalize: construct_gradient (gradients_loop.cc:129-136) and
// local_slopelimiter (gradients_loop.cc:1077-1130).
template <typename T, int TPT>
__global__ void __launch_bounds__(128, 4) k_gradients(PassParams p, Particles ps, const int *__restrict__ targets,
                                                   int n_targets, Csr rows, const GradRec<T> *__restrict__ rec)
{
    const int gtid = blockIdx.x * blockDim.x + threadIdx.x;
    const int slot = gtid / TPT, lane = gtid % TPT;
    if (slot >= n_targets) return;
    const unsigned mask = (TPT == 32) ? 0xffffffffu : (((1u << TPT) - 1u) << ((threadIdx.x & 31) & ~(TPT - 1)));
    const int i = targets[slot];
    const size_t n = (size_t)ps.n;
    const double mi = ps.m[i], rhoi = ps.rho[i], Pi = ps.pressure[i], hid = ps.h[i];
    const bool enabled = (mi > 0 && rhoi > 0);
    const double xi = ps.x[i], yi = ps.y[i], zi = ps.z[i];
    const double hi2 = hid * hid;
    const T hi = T(hid);
    T hinv, hinv3, hinv4;
    k_hinv(hi, hinv, hinv3, hinv4);
    const double vi[3] = {ps.vx[i], ps.vy[i], ps.vz[i]};
    double gr[15];  // [k][q]: q = rho, P, v0, v1, v2
    // the extrema and MaxDistance only ever hold values of type T (differences
    // and distances computed in T), so they are kept in T
    T mx[5], mn[5], maxdist = T(0);
#pragma unroll
    for (int k = 0; k < 15; k++) gr[k] = 0;
#pragma unroll
    for (int k = 0; k < 5; k++) { mx[k] = T(0); mn[k] = T(0); }
    if (enabled) {
        const long long b0 = rows.off[slot], b1 = rows.off[slot + 1];
        long long e = b0 + lane;
        int jn = e < b1 ? __ldg(rows.nbr + e) : 0;
        for (; e < b1; e += TPT) {
            const int jc = jn;
            jn = e + TPT < b1 ? __ldg(rows.nbr + e + TPT) : 0;  // the next index is in flight during this pair
            const GradRec<T> rj = ldg_record(rec + jc);
            const double mj = rj.m, rhoj = rj.rho, hjd = rj.h;
            if (mj <= 0) continue;
            if (rhoj <= 0 || hjd <= 0) continue;
            double dx, dy, dz;
            const double r2 = sep2(xi, yi, zi, rj.x, rj.y, rj.z, p.box, p.half, dx, dy, dz);
            if (r2 <= 0) continue;
            if ((r2 >= hi2) && (r2 >= hjd * hjd)) continue;
            const T r = Real<T>::sqrt_(T(r2));
            T wk_i = T(0), dwk_i = T(0);
            const bool in_i = Real<T>::inside(Real<T>::support_r(r, r2), r2, hi, hid);
            if (in_i) k_main(p.kernel, Real<T>::below_one(r * hinv), hinv3, hinv4, wk_i, dwk_i);
            if (r > maxdist) maxdist = r;
            T d[5];
            d[0] = T(rhoj - rhoi);  // differences in FP64, then rounded once
            d[1] = T(rj.P - Pi);
            d[2] = T(rj.vx - vi[0]);
            d[3] = T(rj.vy - vi[1]);
            d[4] = T(rj.vz - vi[2]);
#pragma unroll
            for (int q = 0; q < 5; q++) {
                if (d[q] < mn[q]) mn[q] = d[q]; else if (d[q] > mx[q]) mx[q] = d[q];
            }
            if (in_i) {
                const T dp[3] = {T(dx), T(dy), T(dz)};
#pragma unroll
                for (int k = 0; k < 3; k++) {
                    const T wxyz = -wk_i * dp[k];
                    gr[5 * k + 0] += (double)(wxyz * d[0]);
                    gr[5 * k + 1] += (double)(wxyz * d[1]);
                    gr[5 * k + 2] += (double)(d[2] * wxyz);
                    gr[5 * k + 3] += (double)(d[3] * wxyz);
                    gr[5 * k + 4] += (double)(d[4] * wxyz);
                }
            }
        }
    }
#pragma unroll
    for (int k = 0; k < 15; k++) gr[k] = warp_sum(gr[k], mask, TPT);
    double mxd[5], mnd[5];
#pragma unroll
    for (int q = 0; q < 5; q++) { mxd[q] = warp_max((double)mx[q], mask, TPT); mnd[q] = warp_min((double)mn[q], mask, TPT); }
    const double maxdistd = warp_max((double)maxdist, mask, TPT);
    if (lane != 0) return;
    double g_rho[3] = {0, 0, 0}, g_p[3] = {0, 0, 0}, g_v[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
    if (enabled) {
        double nv[6];
#pragma unroll
        for (int k = 0; k < 6; k++) nv[k] = ps.nvt[k * n + i];
        double s_rho[3] = {gr[0], gr[5], gr[10]}, s_p[3] = {gr[1], gr[6], gr[11]};
        sym_matvec(nv, s_rho, g_rho);
        sym_matvec(nv, s_p, g_p);
        for (int c = 0; c < 3; c++) {
            double s_v[3] = {gr[2 + c], gr[7 + c], gr[12 + c]};
            sym_matvec(nv, s_v, g_v[c]);
        }
        double stol = 0.0, h_lim = hid;
        const double d_max = dmax(hid, maxdistd);
        h_lim = d_max;
        double a_limiter = 0.25;
        const double CN = ps.cond[i];
        if (CN > 100) a_limiter = dmin(0.5, 0.25 + 0.25 * (CN - 100) / 100);
        if (p.selfgravity_off) { h_lim = hid; stol = 0.1; }
        slopelimiter(g_rho, mxd[0], mnd[0], a_limiter, h_lim, 0, 1, d_max, rhoi);
        slopelimiter(g_p, mxd[1], mnd[1], a_limiter, h_lim, stol, 1, d_max, Pi);
        for (int c = 0; c < 3; c++) slopelimiter(g_v[c], mxd[2 + c], mnd[2 + c], a_limiter, h_lim, stol, 0, 0, 0);
    }
    for (int k = 0; k < 3; k++) {
        ps.grad[(0 + k) * n + i] = g_rho[k];
        ps.grad[(3 + k) * n + i] = g_p[k];
        for (int c = 0; c < 3; c++) ps.grad[(6 + 3 * c + k) * n + i] = g_v[c][k];
    }
}

template <typename T>
void launch_gradients(const PassParams &p, const Particles &ps, const int *targets, int n_targets, Csr rows, int tpt,
                      void *recbuf, const EventPair *ev, cudaStream_t s)
{
    if (n_targets <= 0) return;
    GradRec<T> *rec = (GradRec<T> *)recbuf;
    k_pack_gradient<T><<<(ps.n + kPackBlock - 1) / kPackBlock, kPackBlock, kPackBlock * sizeof(GradRec<T>), s>>>(ps, rec);
    const long long threads = (long long)n_targets * tpt;
    const unsigned blocks = (unsigned)((threads + 127) / 128);  // 128-thread blocks: finer register granularity
    if (ev) cudaEventRecord(ev->start, s);
    switch (tpt) {
        case 1: k_gradients<T, 1><<<blocks, 128, 0, s>>>(p, ps, targets, n_targets, rows, rec); break;
        case 2: k_gradients<T, 2><<<blocks, 128, 0, s>>>(p, ps, targets, n_targets, rows, rec); break;
        case 4: k_gradients<T, 4><<<blocks, 128, 0, s>>>(p, ps, targets, n_targets, rows, rec); break;
        case 8: k_gradients<T, 8><<<blocks, 128, 0, s>>>(p, ps, targets, n_targets, rows, rec); break;
        case 32: k_gradients<T, 32><<<blocks, 128, 0, s>>>(p, ps, targets, n_targets, rows, rec); break;
        default: k_gradients<T, 16><<<blocks, 128, 0, s>>>(p, ps, targets, n_targets, rows, rec); break;
    }
    if (ev) cudaEventRecord(ev->stop, s);
}

// ------------------------------------------------------------------ force
template <typename T> GZ_DEV void load_side(const Particles &ps, int i, double gamma, Side<T> &S)
{
    const size_t n = (size_t)ps.n;
    S.v[0] = T(ps.vx[i]); S.v[1] = T(ps.vy[i]); S.v[2] = T(ps.vz[i]);
    S.pv[0] = T(ps.pv[i]); S.pv[1] = T(ps.pv[n + i]); S.pv[2] = T(ps.pv[2 * n + i]);
#pragma unroll
    for (int k = 0; k < 6; k++) S.nvt[k] = T(ps.nvt[k * n + i]);
#pragma unroll
    for (int k = 0; k < 3; k++) { S.grho[k] = T(ps.grad[k * n + i]); S.gp[k] = T(ps.grad[(3 + k) * n + i]); }
#pragma unroll
    for (int k = 0; k < 9; k++) S.gv[k] = T(ps.grad[(6 + k) * n + i]);
    const double rho = ps.rho[i], P = ps.pressure[i];
    S.m = T(ps.m[i]);
    S.rho = T(rho);
    S.P = T(P);
    S.h = T(ps.h[i]);
    S.cs = T((rho > 0) ? sqrt(gamma * P / rho) : 0.0);  // effective_soundspeed, cell_data.h:703-713
    S.cond = T(ps.cond[i]);
    S.fce = T(ps.fce[i]);
    S.drk = T(ps.drkern[i]);
    S.dt = ps.dt[i];
    S.Vd = ps.m[i] / rho;
    S.condd = ps.cond[i];
    S.fced = ps.fce[i];
    S.prd = P / rho;
}

// Gas-gamma constants of the Riemann solvers (GAMMA_G0..G9, reimann.h:1-10).
template <typename T> GZ_DEV GConst<T> make_gconst(double G0, int mfv)
{
    GConst<T> gc;
    gc.G0 = T(G0); gc.G1 = T((G0 - 1.0) / (2.0 * G0)); gc.G2 = T((G0 + 1.0) / (2.0 * G0));
    gc.G3 = T((2.0 * G0 / (G0 - 1.0))); gc.G4 = T(2.0 / (G0 - 1.0)); gc.G5 = T(2.0 / (G0 + 1.0));
    gc.G6 = T((G0 - 1.0) / (G0 + 1.0)); gc.G7 = T(0.5 * (G0 - 1.0)); gc.G8 = T(1.0 / G0); gc.G9 = T(G0 - 1.0);
    gc.mfv = mfv;
    return gc;
}

// What a force row reads of each neighbour: FP64 position, h, mass and
// density (membership, the j filters, the MFV mass bookkeeping), the
// particle's side of the face in the pair type, and whether it is active
// (208 bytes in FP32, 352 in FP64).
template <typename T> struct __align__(16) ForceRec {
    double x, y, z, h, m, rho;
    Side<T> s;
    int active;
};

// What the gathering force pass reads of each neighbour for the MFV mass
// bookkeeping and the GravWorkTerm: FP64 position, mass and dt, and whether it
// is active (48 bytes: three 16-byte loads, in place of four sectors of the
// neighbour's force record).
struct __align__(16) GatherRec {
    double x, y, z, m, dt;
    int active, pad;
};


template <typename T> __global__ void __launch_bounds__(kPackBlock) k_pack_force(Particles ps, double gamma,
                                                                                ForceRec<T> *rec, GatherRec *grec)
{
    extern __shared__ int4 s_pack[];
    const int first = blockIdx.x * blockDim.x;
    const int i = first + threadIdx.x;
    const int count = min((int)blockDim.x, ps.n - first);
    ForceRec<T> r{};
    GatherRec g{};
    if (i < ps.n) {
        r.x = ps.x[i]; r.y = ps.y[i]; r.z = ps.z[i]; r.h = ps.h[i]; r.m = ps.m[i]; r.rho = ps.rho[i];
        load_side(ps, i, gamma, r.s);
        r.active = ps.active[i];
        g.x = r.x; g.y = r.y; g.z = r.z; g.m = r.m; g.dt = ps.dt[i];
        g.active = r.active;
        g.pad = 0;
    }
    store_block_records(rec, r, first, count, s_pack);
    store_block_records(grec, g, first, count, s_pack);
}

// Row i of the symmetric list: every pair is evaluated in one canonical
// orientation (lower sorted index as the i side of the face) so the flux seen
// from i and from j are exact negatives -- mass and momentum are conserved to
// roundoff of the FP64 accumulation. i-side accumulation follows
// hydro_functions.h:419-509, j-side dMass writes hydro_functions.h:511-532.
// The row's sums go to `sums`; k_force_finish then does the writeback
// (hydro_force_loop.cc:227-391) and the final operations
// (hydro_toplevel.cc:133-253).
//
// MODE kBoth: row i evaluates all its pairs (as the reference does: each pair
//   twice, once per row). Used for active subsets.
// MODE kGather: a pass over every particle evaluates each pair once, in
//   k_force_pairs, which stores its flux at both of the pair's row entries;
//   row i then reads the flux of every entry in place and accumulates it with
//   i's sign. Both rows use the identical flux.
constexpr int kBoth = 0, kGather = 1;
constexpr int kRowSums = 13;  // per row: acc(3) dtE dtm dm gw(3) vs, then the flux_abs diagnostic(3)

template <typename T, int TPT, int MODE>
__global__ void __launch_bounds__(128) k_force(PassParams p, Particles ps, const int *__restrict__ targets,
                                               int n_targets, Csr rows, DevStatus *st,
                                               const ForceRec<T> *__restrict__ rec,
                                               const GatherRec *__restrict__ grec,
                                               const PairFlux<T> *__restrict__ flux, double *sums)
{
    const int gtid = blockIdx.x * blockDim.x + threadIdx.x;
    const int slot = gtid / TPT, lane = gtid % TPT;
    if (slot >= n_targets) return;
    const unsigned mask = (TPT == 32) ? 0xffffffffu : (((1u << TPT) - 1u) << ((threadIdx.x & 31) & ~(TPT - 1)));
    const int i = targets[slot];
    const size_t n = (size_t)ps.n;
    const int mfv = p.method == 1;
    const GConst<T> gc = make_gconst<T>(p.gamma, mfv);
    const double mi = ps.m[i], rhoi = ps.rho[i];
    const bool enabled = (mi > 0 && rhoi > 0);
    const double xi = ps.x[i], yi = ps.y[i], zi = ps.z[i], hid = ps.h[i], dti = ps.dt[i];
    const ForceRec<T> *rip = rec + i;
    double acc[3] = {0, 0, 0}, dtE = 0, dtm = 0, dm = 0, gw[3] = {0, 0, 0}, vs = 0;
    double fa[3] = {0, 0, 0};  // scale of the sums: |F_rho|, |F_v|, |F_E| summed over the row
    int stop = 0;
    if (enabled) {
        vs = (double)rip->s.cs;
        const long long b0 = rows.off[slot], b1 = rows.off[slot + 1];
        long long e = b0 + lane;
        int jn = e < b1 ? rows.nbr[e] : 0;
        // kGather: the next entry's flux and neighbour record are in flight
        // while this entry is accumulated, its index one entry further ahead
        PairFlux<T> Fn{};
        GatherRec gn{};
        int jnn = 0;
        if (MODE == kGather) {
            if (e < b1) {
                Fn = flux[e];
                if (mfv) gn = grec[jn];
            }
            jnn = e + TPT < b1 ? rows.nbr[e + TPT] : 0;
        }
        for (; e < b1; e += TPT) {
            const int j = jn;
            PairFlux<T> F;
            double mj, dtj, dx, dy, dz;
            int j_active;
            if (MODE == kGather) {
                F = Fn;  // valid only if both particles have mass and density
                const GatherRec g = gn;
                jn = jnn;
                if (e + TPT < b1) {
                    Fn = flux[e + TPT];
                    if (mfv) gn = grec[jn];
                }
                jnn = e + 2 * TPT < b1 ? rows.nbr[e + 2 * TPT] : 0;
                if (!F.valid) continue;
                if (mfv) {  // only the MFV bookkeeping reads the neighbour
                    mj = g.m;
                    dtj = g.dt;
                    j_active = g.active;
                    sep2(xi, yi, zi, g.x, g.y, g.z, p.box, p.half, dx, dy, dz);
                }
            } else {
                jn = e + TPT < b1 ? rows.nbr[e + TPT] : 0;  // the next index is in flight during this entry
                const ForceRec<T> *rjp = rec + j;
                mj = rjp->m;
                const double rhoj = rjp->rho;
                if (!(mj > 0 && rhoj > 0)) continue;
                const double r2 = sep2(xi, yi, zi, rjp->x, rjp->y, rjp->z, p.box, p.half, dx, dy, dz);
                const double hjd = rjp->h;
                dtj = rjp->s.dt;
                j_active = rjp->active;
                // one call site for both orientations: the lower sorted index is
                // the i side of the face, so rows i and j run the identical
                // instruction sequence on identical operands and get
                // bit-identical fluxes
                const bool fwd = i < j;
                const double sgn = fwd ? 1.0 : -1.0;
                const T dp[3] = {T(sgn * dx), T(sgn * dy), T(sgn * dz)};
                // both sides are read from the records in place (global memory, L1-resident)
                const ForceRec<T> *pl = fwd ? rip : rjp, *pr = fwd ? rjp : rip;
                Guard<T> g;  // kBoth runs in the FP64 form only (the mixed form goes through the flux buffer)
                force_pair(p.kernel, mfv, p.selfgravity_off, gc, pl->s, pr->s, dp, r2, fwd ? hid : hjd,
                           fwd ? hjd : hid, F, stop, g);
                if (!F.valid) continue;
                wakeup_test(ps, i, j, (double)F.vsig_ts);
            }
            const double sign = (i < j) ? 1.0 : -1.0;
            const double frho = sign * (double)F.rho;
            acc[0] += sign * (double)F.v[0];
            acc[1] += sign * (double)F.v[1];
            acc[2] += sign * (double)F.v[2];
            dtE += sign * (double)F.p;
            if (p.diag_flux_abs) {
                fa[0] += fabs(frho);
                fa[1] += sqrt((double)F.v[0] * (double)F.v[0] + (double)F.v[1] * (double)F.v[1] +
                              (double)F.v[2] * (double)F.v[2]);
                fa[2] += fabs((double)F.p);
            }
            if ((double)F.vsig_ts > vs) vs = (double)F.vsig_ts;
            if (mfv) {
                double self_dm, accepted, other_dm;
                mfv_mass_side(frho, dti, dtj, mi, mj, self_dm, accepted, other_dm);
                dtm += frho;
                dm += self_dm;
                gw[0] += dx * accepted;
                gw[1] += dy * accepted;
                gw[2] += dz * accepted;
                if (j_active) {
                    double sj, aj, oj;  // j's own evaluation writes onto i
                    mfv_mass_side(-frho, dtj, dti, mj, mi, sj, aj, oj);
                    dm += oj;
                } else if (other_dm != 0) {
                    atomicAdd(ps.dmass + j, other_dm);
                }
            }
        }
    }
    if (stop) record_status(st, stop, i);
#pragma unroll
    for (int k = 0; k < 3; k++) {
        acc[k] = warp_sum(acc[k], mask, TPT);
        gw[k] = warp_sum(gw[k], mask, TPT);
        fa[k] = warp_sum(fa[k], mask, TPT);
    }
    dtE = warp_sum(dtE, mask, TPT);
    dtm = warp_sum(dtm, mask, TPT);
    dm = warp_sum(dm, mask, TPT);
    vs = warp_max(vs, mask, TPT);
    if (lane != 0) return;
    const double row[kRowSums] = {acc[0], acc[1], acc[2], dtE, dtm, dm, gw[0], gw[1], gw[2], vs, fa[0], fa[1], fa[2]};
#pragma unroll
    for (int k = 0; k < kRowSums - 3; k++) sums[k * n + i] = row[k];
    if (p.diag_flux_abs)
#pragma unroll
        for (int k = kRowSums - 3; k < kRowSums; k++) sums[k * n + i] = row[k];
}

// The writeback of a force row from its sums, one thread per target: the
// preloop zeros + the row's sums, the MaxSignalVel floor
// (hydro_force_loop.cc:227-391) and the final operations
// (hydro_toplevel.cc:133-253). A separate kernel, because in the row kernel
// only one lane of each row would run it.
template <typename T>
__global__ void __launch_bounds__(256) k_force_finish(PassParams p, Particles ps, const int *__restrict__ targets,
                                                      int n_targets, const double *__restrict__ sums)
{
    const int slot = blockIdx.x * blockDim.x + threadIdx.x;
    if (slot >= n_targets) return;
    const int i = targets[slot];
    const size_t n = (size_t)ps.n;
    const int mfv = p.method == 1;
    const double mi = ps.m[i], rhoi = ps.rho[i], hid = ps.h[i];
    const double acc[3] = {sums[i], sums[n + i], sums[2 * n + i]};
    const double dtE = sums[3 * n + i], dtm = sums[4 * n + i], dm = sums[5 * n + i];
    const double gw[3] = {sums[6 * n + i], sums[7 * n + i], sums[8 * n + i]};
    const double vs = sums[9 * n + i];
    const double cs_i = (rhoi > 0) ? sqrt(p.gamma * ps.pressure[i] / rhoi) : sqrt(p.gamma * (p.gamma - 1.) * ps.u[i]);
    double vsig = kMinReal;
    const double max_sig = fmax(vs, cs_i);
    if (vsig < max_sig) vsig = max_sig;
    double a3[3] = {acc[0], acc[1], acc[2]}, du = dtE, g3[3] = {gw[0], gw[1], gw[2]};
    if (mi > 0) {
        const double v[3] = {ps.vx[i], ps.vy[i], ps.vz[i]};
        if (mfv) {
            const double d[3] = {v[0] - ps.pv[i], v[1] - ps.pv[n + i], v[2] - ps.pv[2 * n + i]};
            const double v2_p = vsig * vsig + (d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
            vsig = sqrt(v2_p);
        }
        du -= (v[0] * a3[0] + v[1] * a3[1] + v[2] * a3[2]);
        if (mfv) {
            du += 0.5 * (v[0] * v[0] + v[1] * v[1] + v[2] * v[2]) * dtm;
            for (int k = 0; k < 3; k++) a3[k] -= v[k] * dtm;
        }
        const double inv = 1.0 / mi;
        for (int k = 0; k < 3; k++) a3[k] *= inv;
        if (mfv) du -= ps.u[i] * dtm;
        du /= mi;
        if (mfv) for (int k = 0; k < 3; k++) g3[k] *= inv;
        if (hid >= 0.99 * p.max_kernel_radius) du = 0;
    }
    for (int k = 0; k < 3; k++) { ps.accel[k * n + i] = a3[k]; ps.gw[k * n + i] = g3[k]; }
    if (p.diag_flux_abs)
        for (int k = 0; k < 3; k++) ps.fabs[k * n + i] = sums[(10 + k) * n + i];
    ps.dudt[i] = du;
    ps.vsig[i] = vsig;
    ps.dtmass[i] = dtm;
    ps.dmass[i] += dm;
}

// Each pair of the symmetric rows once, for a pass over every particle
// (targets[s] = s, rows sorted). A warp takes kPairRows consecutive rows and
// spreads the pairs j > i of all of them over its lanes, one pair per lane per
// round, so no lane idles on a short row. The pair is evaluated in the
// canonical orientation (lower index as the i side), and its flux is stored at
// the pair's entry in row i and at i's entry in row j (a binary search of the
// sorted row j); a pair of which either particle has no mass or density stores
// an invalid flux. k_force<kGather> then accumulates both rows from the stored
// fluxes.
constexpr int kPairRows = 32;

// Queues this lane's pair for the FP64 re-evaluation when `fragile`. Called by
// every lane that reaches it; the lanes that arrive together take one atomic
// for all of their pushes (the count is one address for the whole launch).
GZ_DEV void push_refine(const RefineQueue &q, bool fragile, long long e, long long a, int i, int j, int t)
{
    namespace cg = cooperative_groups;
    if (!q.item) return;
    const cg::coalesced_group grp = cg::coalesced_threads();
    const unsigned want = grp.ballot(fragile);
    if (!want) return;
    const unsigned below = want & ((1u << grp.thread_rank()) - 1u);
    unsigned long long base = 0;
    if (grp.thread_rank() == (unsigned)(__ffs(want) - 1)) base = atomicAdd(q.count, (unsigned long long)__popc(want));
    base = grp.shfl(base, __ffs(want) - 1);
    if (fragile) {
        const unsigned long long k = base + __popc(below);
        if ((long long)k < q.cap) q.item[k] = RefineItem{e, a, i, j, t, 0};
    }
}

// Resident 128-thread blocks per multiprocessor the pair kernel asks of the
// register allocator, each measured at 256^3 against its neighbours. FP32:
// five (at most 96 registers a thread). FP64: four (at most 128): 96.8 ms
// against 99.0 at three, 102.8 at two, 101.3 at five.
template <typename T> constexpr int kForcePairsMinBlocks = sizeof(T) == 4 ? 5 : 4;

template <typename T>
__global__ void __launch_bounds__(128, kForcePairsMinBlocks<T>) k_force_pairs(PassParams p, Particles ps, int n_rows,
                                                                              Csr rows, DevStatus *st,
                                                                              const ForceRec<T> *__restrict__ rec,
                                                                              PairFlux<T> *flux, RefineQueue q)
{
    const long long warp = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    const long long r0 = warp * kPairRows;
    if (r0 >= n_rows) return;  // the whole warp leaves together
    const unsigned full = 0xffffffffu;
    // lane k: row r0 + k, its first entry with j > i and the number of such entries
    long long split = 0;
    int cnt = 0;
    if (lane < kPairRows && r0 + lane < n_rows) {
        const int i = (int)(r0 + lane);
        long long a = rows.off[i], b = rows.off[i + 1];
        const long long end = b;
        while (a < b) {
            const long long mid = a + ((b - a) >> 1);
            if (rows.nbr[mid] <= i) a = mid + 1; else b = mid;
        }
        split = a;
        cnt = (int)(end - a);
    }
    int incl = cnt;  // inclusive scan of the counts over the warp
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        const int v = __shfl_up_sync(full, incl, d);
        if (lane >= d) incl += v;
    }
    const int total = __shfl_sync(full, incl, 31);
    const int mfv = p.method == 1;
    const GConst<T> gc = make_gconst<T>(p.gamma, mfv);
    int stop = 0, stop_index = -1;
    for (int base = 0; base < total; base += 32) {
        const int f = base + lane;
        // the row of pair f: the number of rows whose inclusive count is <= f
        int k = 0;
#pragma unroll
        for (int step = 16; step > 0; step >>= 1) {
            const int v = __shfl_sync(full, incl, k + step - 1);
            if (v <= f) k += step;
        }
        const int excl_k = __shfl_sync(full, incl - cnt, k);
        const long long split_k = __shfl_sync(full, split, k);
        if (f >= total) continue;
        const int i = (int)(r0 + k);
        const long long e = split_k + (f - excl_k);
        const int j = rows.nbr[e];
        const ForceRec<T> *rip = rec + i;  // shared by the lanes of the row: cached
        const ForceRec<T> rj = ldg_record(rec + j);
        const ForceRec<T> *rjp = &rj;
        PairFlux<T> F;
        F.valid = 0;
        F.rho = F.p = T(0);
        F.v[0] = F.v[1] = F.v[2] = T(0);
        F.vsig_ts = T(0);
        Guard<T> g;
        if (rip->m > 0 && rip->rho > 0 && rjp->m > 0 && rjp->rho > 0) {
            double dx, dy, dz;
            const double r2 = sep2(rip->x, rip->y, rip->z, rjp->x, rjp->y, rjp->z, p.box, p.half, dx, dy, dz);
            const T dp[3] = {T(dx), T(dy), T(dz)};
            int pstop = 0;
            force_pair(p.kernel, mfv, p.selfgravity_off, gc, rip->s, rjp->s, dp, r2, rip->h, rjp->h, F, pstop, g);
            // a fragile pair's flux (and stop code) comes from its FP64 evaluation, queued below
            if (g.fragile()) pstop = 0;
            if (pstop && !stop) { stop = pstop; stop_index = i; }
        }
        flux[e] = F;
        // i's entry in row j
        const long long b_end = rows.off[j + 1];
        long long a = rows.off[j], b = b_end;
        while (a < b) {
            const long long mid = a + ((b - a) >> 1);
            if (rows.nbr[mid] < i) a = mid + 1; else b = mid;
        }
        if (a >= b_end || rows.nbr[a] != i) {  // rows not symmetric: cannot happen for rows built here
            if (!stop) { stop = 6 /* GZ_ERR_INTERNAL */; stop_index = i; }
            continue;
        }
        flux[a] = F;
        push_refine(q, g.fragile(), e, a, i, j, -1);
    }
    if (stop) record_status(st, stop, stop_index);
}

// Every entry of the rows of a pass over an active subset, each written at its
// own entry: a pair of two active particles is evaluated once per row, as the
// reference does, in the canonical orientation (lower sorted index as the i
// side), so both evaluations are bit-identical. A warp takes kPairRows rows and
// spreads their entries over its lanes, one entry per lane per round; the flux
// goes to k_force<kGather> like the pairs of a pass over every particle. The
// wake-up test of an inactive neighbour (hydro_functions.h:534-544) runs here.
template <typename T>
__global__ void __launch_bounds__(128) k_force_entries(PassParams p, Particles ps, const int *__restrict__ targets,
                                                       int n_rows, Csr rows, DevStatus *st,
                                                       const ForceRec<T> *__restrict__ rec, PairFlux<T> *flux,
                                                       RefineQueue q)
{
    const long long warp = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    const long long r0 = warp * kPairRows;
    if (r0 >= n_rows) return;  // the whole warp leaves together
    const unsigned full = 0xffffffffu;
    long long first = 0;
    int cnt = 0;
    if (lane < kPairRows && r0 + lane < n_rows) {
        first = rows.off[r0 + lane];
        cnt = (int)(rows.off[r0 + lane + 1] - first);
    }
    int incl = cnt;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        const int v = __shfl_up_sync(full, incl, d);
        if (lane >= d) incl += v;
    }
    const int total = __shfl_sync(full, incl, 31);
    const int mfv = p.method == 1;
    const GConst<T> gc = make_gconst<T>(p.gamma, mfv);
    int stop = 0, stop_index = -1;
    for (int base = 0; base < total; base += 32) {
        const int f = base + lane;
        int k = 0;
#pragma unroll
        for (int step = 16; step > 0; step >>= 1) {
            const int v = __shfl_sync(full, incl, k + step - 1);
            if (v <= f) k += step;
        }
        const int excl_k = __shfl_sync(full, incl - cnt, k);
        const long long first_k = __shfl_sync(full, first, k);
        if (f >= total) continue;
        const int t = targets[r0 + k];
        const long long e = first_k + (f - excl_k);
        const int j = rows.nbr[e];
        const int lo = t < j ? t : j, hi = t < j ? j : t;
        const ForceRec<T> rl = ldg_record(rec + lo), rh = ldg_record(rec + hi);
        PairFlux<T> F;
        F.valid = 0;
        F.rho = F.p = T(0);
        F.v[0] = F.v[1] = F.v[2] = T(0);
        F.vsig_ts = T(0);
        Guard<T> g;
        if (rl.m > 0 && rl.rho > 0 && rh.m > 0 && rh.rho > 0) {
            double dx, dy, dz;
            const double r2 = sep2(rl.x, rl.y, rl.z, rh.x, rh.y, rh.z, p.box, p.half, dx, dy, dz);
            const T dp[3] = {T(dx), T(dy), T(dz)};
            int pstop = 0;
            force_pair(p.kernel, mfv, p.selfgravity_off, gc, rl.s, rh.s, dp, r2, rl.h, rh.h, F, pstop, g);
            // the wake-up test of an inactive neighbour, on the pair's signal speed
            const bool wake_test = F.valid && ps.bin_active && !ps.bin_active[ps.timebin[j]];
            const double wake_at = wake_test ? kWakeup * ps.vsig_prev[j] : 0.0;
            if (wake_test) g.near(F.vsig_ts, T(wake_at), F.vsig_ts, 38);
            if (g.fragile()) pstop = 0;
            else if (wake_test && (double)F.vsig_ts > wake_at) atomicMax(ps.wakeup + j, ps.timebin[t] + 1);
            if (pstop && !stop) { stop = pstop; stop_index = t; }
        }
        flux[e] = F;
        push_refine(q, g.fragile(), e, -1, lo, hi, t);
    }
    if (stop) record_status(st, stop, stop_index);
}

template <typename T, int MODE>
void launch_force_mode(const PassParams &p, const Particles &ps, const int *targets, int n_targets, Csr rows, int tpt,
                       DevStatus *st, const ForceRec<T> *rec, const GatherRec *grec, const PairFlux<T> *flux,
                       double *sums, cudaStream_t s)
{
    const long long threads = (long long)n_targets * tpt;
    const unsigned blocks = (unsigned)((threads + 127) / 128);
    switch (tpt) {
        case 1: k_force<T, 1, MODE><<<blocks, 128, 0, s>>>(p, ps, targets, n_targets, rows, st, rec, grec, flux, sums); break;
        case 4: k_force<T, 4, MODE><<<blocks, 128, 0, s>>>(p, ps, targets, n_targets, rows, st, rec, grec, flux, sums); break;
        case 8: k_force<T, 8, MODE><<<blocks, 128, 0, s>>>(p, ps, targets, n_targets, rows, st, rec, grec, flux, sums); break;
        case 32: k_force<T, 32, MODE><<<blocks, 128, 0, s>>>(p, ps, targets, n_targets, rows, st, rec, grec, flux, sums); break;
        default: k_force<T, 16, MODE><<<blocks, 128, 0, s>>>(p, ps, targets, n_targets, rows, st, rec, grec, flux, sums); break;
    }
    k_force_finish<T><<<(unsigned)((n_targets + 255) / 256), 256, 0, s>>>(p, ps, targets, n_targets, sums);
}

// With `fluxbuf` (one PairFlux<T> per row entry) the pairs are evaluated into
// it -- each pair once when `all` (every particle a target, targets[s] = s),
// otherwise each row entry -- the mixed form's fragile pairs are evaluated
// again in FP64 (force_refine), and k_force<kGather> accumulates the rows;
// without it (the FP64 form only) each row evaluates all its pairs in place.
// `sums`: kRowSums x n doubles of scratch.
template <typename T>
void launch_force(const PassParams &p, const Particles &ps, const int *targets, int n_targets, Csr rows, int tpt,
                  DevStatus *st, void *recbuf, void *fluxbuf, bool all, const RefineQueue &q, double *sums,
                  const EventPair *ev, cudaStream_t s)
{
    if (n_targets <= 0) return;
    // the record scratch holds the force records, then the gather records
    ForceRec<T> *rec = (ForceRec<T> *)recbuf;
    GatherRec *grec = (GatherRec *)(rec + ps.n);
    k_pack_force<T><<<(ps.n + kPackBlock - 1) / kPackBlock, kPackBlock, kPackBlock * sizeof(ForceRec<T>), s>>>(
        ps, p.gamma, rec, grec);
    if (fluxbuf) {
        PairFlux<T> *flux = (PairFlux<T> *)fluxbuf;
        const long long warps = (n_targets + kPairRows - 1) / kPairRows;
        if (ev) cudaEventRecord(ev->start, s);
        if (all) k_force_pairs<T><<<(unsigned)((warps + 3) / 4), 128, 0, s>>>(p, ps, n_targets, rows, st, rec, flux, q);
        else k_force_entries<T><<<(unsigned)((warps + 3) / 4), 128, 0, s>>>(p, ps, targets, n_targets, rows, st, rec,
                                                                            flux, q);
        if (ev) cudaEventRecord(ev->stop, s);
        if constexpr (sizeof(T) == sizeof(float)) force_refine(p, ps, q, flux, st, s);
        // one thread per row: the gather's per-entry work is short, and lanes
        // sharing a row would spend more on the cross-lane reduction and on
        // idling at the row's end than on the entries themselves
        launch_force_mode<T, kGather>(p, ps, targets, n_targets, rows, 1, st, rec, grec, flux, sums, s);
    } else if constexpr (sizeof(T) == sizeof(double)) {
        if (ev) cudaEventRecord(ev->start, s);  // (also spans the writeback kernel)
        launch_force_mode<T, kBoth>(p, ps, targets, n_targets, rows, tpt, st, rec, grec, nullptr, sums, s);
        if (ev) cudaEventRecord(ev->stop, s);
    }
}

}  // namespace gz

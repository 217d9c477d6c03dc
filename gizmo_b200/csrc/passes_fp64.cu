// gizmo_b200/csrc/passes_fp64.cu -- FP64 form of the pair kernels plus the
// per-particle FP64 epilogues shared by both forms. Built with -fmad=false so
// every product and sum rounds as in the reference's CPU build.
#include "passes.cuh"

namespace gz {

size_t gradient_record_bytes(int mixed) { return mixed ? sizeof(GradRec<float>) : sizeof(GradRec<double>); }
size_t force_record_bytes(int mixed)
{
    return (mixed ? sizeof(ForceRec<float>) : sizeof(ForceRec<double>)) + sizeof(GatherRec);
}
size_t pair_flux_bytes(int mixed) { return mixed ? sizeof(PairFlux<float>) : sizeof(PairFlux<double>); }

__global__ void __launch_bounds__(kPackBlock) k_pack_density(Particles ps, DensRec *rec)
{
    extern __shared__ int4 s_pack[];
    const int first = blockIdx.x * blockDim.x;
    const int i = first + threadIdx.x;
    DensRec r{};
    if (i < ps.n) {
        r.x = ps.x[i]; r.y = ps.y[i]; r.z = ps.z[i]; r.m = ps.m[i];
        r.vx = ps.vx[i]; r.vy = ps.vy[i]; r.vz = ps.vz[i]; r.pad = 0.0;
    }
    store_block_records(rec, r, first, min((int)blockDim.x, ps.n - first), s_pack);
}

void density_pack(const Particles &ps, DensRec *rec, cudaStream_t s)
{
    if (ps.n > 0)
        k_pack_density<<<(ps.n + kPackBlock - 1) / kPackBlock, kPackBlock, kPackBlock * sizeof(DensRec), s>>>(ps, rec);
}

void density_sums_fp64(const PassParams &p, const Particles &ps, const DensityWork &w, int tpt, cudaStream_t s)
{
    launch_density_sums<double>(p, ps, w, tpt, s);
}

void density_sums_graph(const PassParams &p, const Particles &ps, const DensityWork &w, GraphState *gs,
                        const int *todo, int blocks, cudaStream_t s)
{
    k_density_sums_graph<double, 4><<<blocks, kDensityBlock, 0, s>>>(p, ps, w, gs, todo);
    k_density_sums_graph<double, 8><<<blocks, kDensityBlock, 0, s>>>(p, ps, w, gs, todo);
    k_density_sums_graph<double, 16><<<blocks, kDensityBlock, 0, s>>>(p, ps, w, gs, todo);
}

void gradients_fp64(const PassParams &p, const Particles &ps, const int *targets, int n_targets, Csr rows, int tpt,
                    void *rec, const EventPair *ev, cudaStream_t s)
{
    launch_gradients<double>(p, ps, targets, n_targets, rows, tpt, rec, ev, s);
}

void force_fp64(const PassParams &p, const Particles &ps, const int *targets, int n_targets, Csr rows, int tpt,
                DevStatus *st, void *rec, void *flux, bool all, double *sums, const EventPair *ev, cudaStream_t s)
{
    const RefineQueue none{nullptr, nullptr, 0};
    launch_force<double>(p, ps, targets, n_targets, rows, tpt, st, rec, flux, all, none, sums, ev, s);
}

// force_refine: one thread per queued pair, grid-stride over the count the
// pair kernel left on the device. The pair is the FP64 form's: Side<double>
// from the FP64 mirror exactly as k_pack_force<double> packs it, the same
// minimum-image separation and the same force_pair<double> call in this
// unit's arithmetic (no contraction), so the flux is the FP64 form's bit for
// bit before it is rounded to the FP32 flux entry. The wake-up test of a pair
// of an active-subset pass is taken here too, on the FP64 signal speed.
__global__ void __launch_bounds__(128) k_force_refine(PassParams p, Particles ps, RefineQueue q,
                                                      PairFlux<float> *flux, DevStatus *st)
{
    const unsigned long long pushed = *q.count;  // beyond cap: the host redoes the pass with a longer queue
    const long long n = (long long)pushed < q.cap ? (long long)pushed : q.cap;
    const int mfv = p.method == 1;
    const GConst<double> gc = make_gconst<double>(p.gamma, mfv);
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x) {
        const RefineItem it = q.item[k];
        Side<double> A, B;
        load_side(ps, it.i, p.gamma, A);
        load_side(ps, it.j, p.gamma, B);
        double dx, dy, dz;
        const double r2 = sep2(ps.x[it.i], ps.y[it.i], ps.z[it.i], ps.x[it.j], ps.y[it.j], ps.z[it.j], p.box, p.half,
                               dx, dy, dz);
        const double dp[3] = {dx, dy, dz};
        PairFlux<double> F64;
        int stop = 0;
        Guard<double> g;
        force_pair(p.kernel, mfv, p.selfgravity_off, gc, A, B, dp, r2, ps.h[it.i], ps.h[it.j], F64, stop, g);
        if (stop) record_status(st, stop, it.i);
        PairFlux<float> F;
        F.rho = (float)F64.rho;
        F.p = (float)F64.p;
        F.v[0] = (float)F64.v[0]; F.v[1] = (float)F64.v[1]; F.v[2] = (float)F64.v[2];
        F.vsig_ts = (float)F64.vsig_ts;
        F.valid = F64.valid;
        flux[it.e] = F;
        if (it.a >= 0) flux[it.a] = F;
        if (it.t >= 0 && F64.valid) wakeup_test(ps, it.t, it.t == it.i ? it.j : it.i, F64.vsig_ts);
    }
}

void force_refine(const PassParams &p, const Particles &ps, const RefineQueue &q, PairFlux<float> *flux,
                  DevStatus *st, cudaStream_t s)
{
    if (!q.item) return;
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    k_force_refine<<<sms * 4, 128, 0, s>>>(p, ps, q, flux, st);
}

// DensitySpec::after_iter_body for one target of iteration `iter`, plus the
// runner's radius update (neighbor_loop_runner.cc:7340-7372): returns whether
// it still iterates, sets `regrow` when its new radius outgrew its row and
// `moved` to that radius.
GZ_DEV bool after_iter_target(const PassParams &p, const Particles &ps, const DensityWork &w, int iter, int t,
                              DevStatus *st, bool &regrow, double &moved)
{
    const size_t n = (size_t)ps.n;
    double acc[14];
    for (int k = 0; k < 14; k++) acc[k] = w.acc[k * n + t];
    const double h = ps.h[t];
    DensityScratch sc = w.scratch[t];
    double nh = h;
    int stop = 0;
    const int conv = after_iter(p, iter, h, acc, ps.cond[t], sc, nh, stop);
    w.scratch[t] = sc;
    ps.iters[t] = iter + 1;
    if (stop) record_status(st, stop, t);
    regrow = false;
    if (!conv) {
        ps.h[t] = nh;
        moved = nh;
        regrow = nh > w.h_built[t];
    }
    return !conv;
}

// after_iter per iterating particle, with the compaction flags
// (neighbor_loop_runner.cc:7340-7372).
__global__ void k_after_iter(PassParams p, Particles ps, DensityWork w, DevStatus *st)
{
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    double moved = 0;  // the radius this particle moves to (0: none), for the iteration's largest
    if (s < w.n_todo) {
        bool regrow = false;
        const bool keep = after_iter_target(p, ps, w, w.iter, w.todo[s], st, regrow, moved);
        if (regrow) atomicExch(w.rebuild, 1);
        w.keep[s] = keep ? 1 : 0;
        w.regrow[s] = (unsigned char)regrow;
    }
    if (w.h_iter_max) warp_atomic_max_nonneg(w.h_iter_max, moved);  // every lane of the block
}

// after_iter for a captured pass: the iteration and its target count come
// from the device state; the flags (still iterating, radius outgrew its row)
// are per slot, as k_after_iter writes them, for the compaction that follows.
// Blocks take block-sized chunks of the list from a counter, in order, as
// the hardware hands out the blocks of the plain launch.
__global__ void __launch_bounds__(128) k_after_iter_graph(PassParams p, Particles ps, DensityWork w, DevStatus *st,
                                                          GraphState *gs, const int *__restrict__ todo)
{
    __shared__ int s_chunk;
    if (gs->fail) return;
    const int iter = gs->iter, n_todo = gs->n_todo;
    double moved = 0;
    for (;;) {
        if (threadIdx.x == 0) s_chunk = atomicAdd(&gs->after_next, 1);
        __syncthreads();
        const int chunk = s_chunk;
        __syncthreads();
        if ((long long)chunk * blockDim.x >= n_todo) break;
        const int s = chunk * blockDim.x + threadIdx.x;
        if (s < n_todo) {
            bool regrow = false;
            double mv = 0;
            const bool keep = after_iter_target(p, ps, w, iter, todo[s], st, regrow, mv);
            moved = fmax(moved, mv);
            w.keep[s] = keep ? 1 : 0;
            w.regrow[s] = (unsigned char)regrow;
        }
    }
    if (w.h_iter_max) warp_atomic_max_nonneg(w.h_iter_max, moved);
}

void density_after_iter(const PassParams &p, const Particles &ps, const DensityWork &w, DevStatus *st, cudaStream_t s)
{
    if (w.n_todo <= 0) return;
    k_after_iter<<<(w.n_todo + 127) / 128, 128, 0, s>>>(p, ps, w, st);
}

void density_after_iter_graph(const PassParams &p, const Particles &ps, const DensityWork &w, DevStatus *st,
                              GraphState *gs, const int *todo, int blocks, cudaStream_t s)
{
    k_after_iter_graph<<<blocks, 128, 0, s>>>(p, ps, w, st, gs, todo);
}

// density_finalize_post_runner (density_loop.cc:303-733), gas, non-SPH.
__global__ void k_density_finalize(PassParams p, Particles ps, const double *__restrict__ accb,
                                   const int *__restrict__ targets, int n_targets)
{
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n_targets) return;
    const int i = targets[s];
    const size_t n = (size_t)ps.n;
    double acc[17];
    for (int k = 0; k < 17; k++) acc[k] = accb[k * n + i];
    const double h = ps.h[i];
    double NumNgb = acc[0], Drk = acc[2], DivV = acc[3];
    if (NumNgb > 0) {
        Drk *= h / (3 * NumNgb);
        DivV /= NumNgb;
        NumNgb *= kVolNorm * cr::pow(h, 3.0);
    } else { NumNgb = Drk = DivV = 0; }
    if (Drk > -0.9) Drk = 1.0 / (1.0 + Drk); else Drk = 1.0;
    DivV *= Drk;
    ps.drkern[i] = Drk;
    ps.divvel[i] = DivV;
    double rho = acc[1];
    double pvl[3] = {acc[14], acc[15], acc[16]};
    double CN, fce, Tn[3][3];
    nvt_invert(h, NumNgb, acc + 4, acc + 10, CN, Tn, fce);
    ps.nvt[0 * n + i] = Tn[0][0]; ps.nvt[1 * n + i] = Tn[1][1]; ps.nvt[2 * n + i] = Tn[2][2];
    ps.nvt[3 * n + i] = Tn[0][1]; ps.nvt[4 * n + i] = Tn[1][2]; ps.nvt[5 * n + i] = Tn[0][2];
    ps.cond[i] = CN;
    ps.fce[i] = fce;
    const double m = ps.m[i];
    if (m > 0) {
        if (rho > 0 && p.method == 1) {
            const double eps = 0.3;
            const double v[3] = {ps.vx[i], ps.vy[i], ps.vz[i]};
            for (int k = 0; k < 3; k++) pvl[k] = v[k] * (1.0 - eps) + pvl[k] * (eps / rho);
        }
        if ((h > 0) && (NumNgb > 0)) rho = m * NumNgb / (kVolNorm * cr::pow(h, 3.0));
        else if (h <= 0) rho = 0;
        else rho = m / (kVolNorm * cr::pow(h, 3.0));
        ps.pressure[i] = (p.gamma - 1) * ps.u[i] * rho;
    }
    ps.rho[i] = rho;
    for (int k = 0; k < 3; k++) ps.pv[k * n + i] = pvl[k];
    ps.num_ngb[i] = (NumNgb > 0) ? cr::pow(NumNgb, 1.0 / 3) : 0;
}

void density_finalize(const PassParams &p, const Particles &ps, const double *acc, const int *targets, int n_targets,
                      cudaStream_t s)
{
    if (n_targets <= 0) return;
    k_density_finalize<<<(n_targets + 127) / 128, 128, 0, s>>>(p, ps, acc, targets, n_targets);
}

// hydro_force_initial_operations_preloop (hydro_toplevel.cc:457-565): the
// running dMass of every active cell restarts at zero (the other preloop
// fields are assigned outright by the force kernel).
__global__ void k_force_preloop(Particles ps, const int *__restrict__ targets, int n_targets)
{
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n_targets) return;
    ps.dmass[targets[s]] = 0;
}

void force_preloop(const PassParams &p, const Particles &ps, const int *targets, int n_targets, cudaStream_t s)
{
    (void)p;
    if (n_targets <= 0) return;
    k_force_preloop<<<(n_targets + 255) / 256, 256, 0, s>>>(ps, targets, n_targets);
}

}  // namespace gz

// gizmo_b200/csrc/capi.cu -- the C ABI (include/gizmo_hydro.h): context,
// device-resident particle mirror, and the pass orchestration that replaces
// run_neighbor_loop_iterative<DensitySpec>, run_neighbor_loop<GradientsSpec>
// and run_neighbor_loop<HydroForceSpec> (src/mesh/neighbor_loop_runner.h:1614-1629)
// inside density() / hydro_gradient_calc() / hydro_force().
#include <cub/cub.cuh>

#include <algorithm>
#include <cmath>
#include <map>
#include <mutex>
#include <tuple>
#include <cstdio>
#include <cstring>
#include <vector>

#include "../../include/gizmo_hydro.h"
#include "launch.h"

using namespace gz;

namespace {

struct DevBuf {
    void *p = nullptr;
    size_t bytes = 0;
};

// Search radius of the density rows, as a factor of h (the pair body re-filters
// r < h exactly, so any factor >= 1 gives the same sums). The reference's runner
// uses 1.3 (DensitySpec::mode_a_csr_buffer_factor, density_loop.h:316). From a
// previous step's h the first rows need less: 1.15 x h holds the whole iteration
// of ~98.6% of particles (Plummer mixture) at 0.66 x the candidates of 1.3 x h;
// a particle whose h outgrows its row gets a new one at 1.3 x its new h.
constexpr double kDensityBufferFirst = 1.15;
constexpr double kDensityBuffer = 1.3;

}  // namespace

struct gz_context {
    gz_params prm{};
    PassParams pp{};
    int device = 0;
    cudaStream_t stream = nullptr;
    int n = 0;
    // sorted SoA mirror
    DevBuf x, y, z, vx, vy, vz, m, u, dt, h, cond, num_ngb, drkern, divvel, rho, pressure, fce, nvt, pv, grad, accel,
        dudt, vsig, dtmass, dmass, gw, fabs3, iters, active;
    // original-order staging and permutation
    DevBuf stage, stage3, perm, inv, keys, keys_sorted, idx, cub_tmp, targets_orig, targets, targets_tmp;
    // resident copies of the uploaded inputs, original order (gz_restage source)
    DevBuf o_vel, o_mass, o_u, o_dt, o_h, o_cond;
    // individual timesteps: resident inputs (original order), sorted copies, wake-up flags, TimeBinActive
    DevBuf o_timebin, o_vsig, timebin, vsig_prev, wakeup, binact, sel_flags, sel_out;
    bool have_bins = false;          // timebin (and vsig) were uploaded
    bool binact_on = false;          // gz_set_bin_active gave a table
    DevBuf dl;                       // download staging, [9][n] doubles (widest output field)
    DevBuf rec;                      // packed neighbour records of the running pass
    DevBuf work;                     // work counter of the persistent walks
    long long launches = 0;          // kernels of this library launched by the context
    // octree over the sorted particles
    DevBuf t_node, t_lo, t_hi, t_parent, t_done, t_nch, t_cpos, t_build;
    int t_nodes = 0, t_levels = 0;
    bool grid_valid = false;
    // density work: rows are [d_beg[t], d_end[t]) in d_nbr; d_used entries are taken
    DevBuf acc, h_built, scratch, keep, regrow, todo_a, todo_b, grow, d_beg, d_end, flag, counts, d_off, d_nbr, n_sel;
    DevBuf hmax;                     // largest kernel length the density iteration took sums at (double bits)
    DevBuf refined, rq;              // mixed form: count and queue of the force pairs evaluated again in FP64
    long long pairs_refined = 0;
    double h_iter_max = 0;           // ... read back after the pass
    long long d_nbr_cap = 0, d_used = 0;
    bool dens_all = false;           // the density rows cover every particle (last pass had no active list)
    DevBuf pad_over, pad_list, pad_sum, pad_counts;  // padded single-walk density rows
    DevBuf s_acnt, s_bcnt, s_tmp;    // symmetric rows derived from the density rows
    DevBuf pflux;                    // force pass evaluating each pair once: the flux per row entry
    // symmetric rows (shared by gradients and force)
    DevBuf s_off, s_nbr, s_counts;
    long long s_nbr_cap = 0;
    int sym_rows = 0;
    bool sym_valid = false;
    std::vector<int> sym_active;     // active list the symmetric rows were built for
    bool sym_all = false;            // ... or all particles
    DevBuf status;
    // host record
    int err = 0, err_index = -1;
    char msg[256] = {0};
    int last_iters = 0;
    long long pairs_density = 0, pairs_symmetric = 0;
    bool have_density = false, have_gradients = false;
    int tpt_force = 8;               // lanes per force row (fixed: measured best at every size)
    int diag = 0;                    // GZ_DIAG_* flags
    bool timing = false;             // gz_kernel_timing on
    struct Timer {
        std::vector<EventPair> ev;   // event pairs, one per timed launch since the last read
        size_t used = 0;
        long long units = 0;
    } timers[GZ_TIMERS];
    bool fabs_valid = false;         // the last force pass summed flux_abs
    int sms = 148;                   // multiprocessors of the device
    // walk tuning (gz_tuning): neither changes a result, both change the walk's cost
    int leaf_max = kLeafMax;         // octree leaf size
    double row_slots = 2.5;          // padded density-row slots per expected row entry
    // the pass over every particle captured as one CUDA graph (gz_hydro_pass)
    struct Graph {
        cudaGraph_t graph = nullptr;
        cudaGraphExec_t exec = nullptr;
        cudaStream_t body[2] = {nullptr, nullptr};  // streams the conditional bodies are captured on
        std::vector<unsigned long long> sig;        // what the graph was captured for (buffers, sizes, settings)
        long long kernels_top = 0, kernels_loop = 0, kernels_sym = 0, kernels_tail = 0;
        long long rq_cap = 0;                       // refine-queue room the graph was captured with
        bool with_restage = false;                  // the graph starts with the restage
        long long replays = 0, captures = 0, fallbacks = 0;
        bool capturing = false;                     // no timer events while a graph is captured
    } g;
    DevBuf gstate, g_hseed, g_cseed, g_over_list, g_over_off, g_sel;
    // box sets (gz_set_boxes): consecutive runs of the particles, each its own
    // periodic box; their index above the Morton bits of the keys
    std::vector<long long> box_counts;
    int box_bits = 0;                // bits of the box index (a multiple of 3: whole octree levels)
    DevBuf box_bid, box_of, root_of; // box of each particle (caller's order, sorted), subtree of each box
    // pipelined transfers (gz_upload_async / gz_download_async): the inputs of
    // the next step land in p_* while a step runs; the outputs of a step leave
    // from dstage while the next one runs
    DevBuf p_stage3, p_vel, p_mass, p_u, p_dt, p_h, p_cond, dstage;
    cudaStream_t cstream = nullptr;  // the copy stream
    cudaEvent_t ev_in_free = nullptr, ev_in_done = nullptr, ev_out_ready = nullptr, ev_out_done = nullptr;
    bool in_pending = false, out_pending = false;
};

namespace {

// Lanes per row of the density and gradient row kernels. Fewer lanes per row
// mean more rows in flight per warp and a shorter cross-lane reduction, but
// fewer threads: the fewest lanes (at least `min_lanes`) with which the rows
// still give about eight waves of resident threads (2048 per multiprocessor),
// at most 16. The density rows keep at least 4 lanes: their pair work is long
// and the lanes of a row share its loads.
int lanes_per_row(const gz_context *c, long long rows, int min_lanes)
{
    const long long want = (long long)c->sms * 2048 * 8;
    int tpt = min_lanes;
    while (tpt < 16 && rows * tpt < want) tpt *= 2;
    return tpt;
}

// The event pair for one launch of timer `id` (null when timing is off, or
// when no event could be had: that launch then goes untimed).
const EventPair *timer_launch(gz_context *c, int id, long long units)
{
    if (!c->timing || c->g.capturing) return nullptr;
    gz_context::Timer &t = c->timers[id];
    if (t.used == t.ev.size()) {
        EventPair e{nullptr, nullptr};
        if (cudaEventCreate(&e.start) != cudaSuccess) return nullptr;
        if (cudaEventCreate(&e.stop) != cudaSuccess) { cudaEventDestroy(e.start); return nullptr; }
        t.ev.push_back(e);
    }
    t.units += units;
    return &t.ev[t.used++];
}

// record the start / stop of a launch timed from here
void ev_start(const EventPair *e, cudaStream_t s) { if (e) cudaEventRecord(e->start, s); }
void ev_stop(const EventPair *e, cudaStream_t s) { if (e) cudaEventRecord(e->stop, s); }

// walk_rows, timed under GZ_TIMER_WALK
void walk_timed(gz_context *c, const Tree &t, const double *x, const double *y, const double *z, const double *reach,
                const double *hsym, int symmetric, const int *targets, int n_targets, long long *counts,
                const long long *off, int *nbr, int cap, DevStatus *st, int *next_group, cudaStream_t s)
{
    const EventPair *ev = n_targets > 0 ? timer_launch(c, GZ_TIMER_WALK, n_targets) : nullptr;
    ev_start(ev, s);
    walk_rows(t, x, y, z, reach, hsym, symmetric, targets, n_targets, counts, off, nbr, cap, st, next_group, s);
    ev_stop(ev, s);
}

int fail(gz_context *c, int code, const char *what)
{
    if (c) {
        if (!c->err) { c->err = code; }
        snprintf(c->msg, sizeof(c->msg), "%s", what);
    }
    return code;
}

#define GZ_CUDA(ctx, call)                                                                \
    do {                                                                                  \
        cudaError_t e_ = (call);                                                          \
        if (e_ != cudaSuccess) {                                                          \
            char b_[200];                                                                 \
            snprintf(b_, sizeof(b_), "%s: %s", #call, cudaGetErrorString(e_));            \
            return fail(ctx, GZ_ERR_CUDA, b_);                                            \
        }                                                                                 \
    } while (0)

template <typename T> T *ptr(DevBuf &b) { return (T *)b.p; }

int ensure(gz_context *c, DevBuf &b, size_t bytes)
{
    if (b.bytes >= bytes && b.p) return 0;
    if (b.p) cudaFree(b.p);
    b.p = nullptr;
    b.bytes = 0;
    size_t want = bytes > 0 ? bytes : 16;
    GZ_CUDA(c, cudaMalloc(&b.p, want));
    b.bytes = want;
    return 0;
}

// like ensure(), but a failed allocation is not an error of the context
bool try_ensure(DevBuf &b, size_t bytes)
{
    if (b.bytes >= bytes && b.p) return true;
    if (b.p) cudaFree(b.p);
    b.p = nullptr;
    b.bytes = 0;
    if (cudaMalloc(&b.p, bytes > 0 ? bytes : 16) != cudaSuccess) {
        cudaGetLastError();  // clear the allocation failure
        b.p = nullptr;
        return false;
    }
    b.bytes = bytes > 0 ? bytes : 16;
    return true;
}

void release(DevBuf &b)
{
    if (b.p) cudaFree(b.p);
    b.p = nullptr;
    b.bytes = 0;
}

PassParams make_pass_params(const gz_params &p)
{
    PassParams q{};
    q.kernel = p.kernel;
    q.method = p.method;
    q.first_step = p.first_step;
    q.selfgravity_off = p.selfgravity_off;
    q.box = p.box_size;
    q.half = 0.5 * p.box_size;
    q.gamma = p.gamma;
    q.des_num_ngb = p.des_num_ngb;
    q.max_num_ngb_dev = p.max_num_ngb_dev;
    q.min_kernel_radius = p.min_kernel_radius;
    q.max_kernel_radius = p.max_kernel_radius;
    return q;
}

int check_params(const gz_params *p)
{
    if (!p) return GZ_ERR_ARG;
    if (p->kernel != GZ_KERNEL_CUBIC && p->kernel != GZ_KERNEL_WENDLAND_C2) return GZ_ERR_ARG;
    if (p->method != GZ_METHOD_MFM && p->method != GZ_METHOD_MFV) return GZ_ERR_ARG;
    if (p->precision != GZ_PRECISION_FP64 && p->precision != GZ_PRECISION_MIXED) return GZ_ERR_ARG;
    if (!(p->box_size > 0) || !(p->gamma > 1.0) || !(p->des_num_ngb > 0)) return GZ_ERR_ARG;
    return GZ_OK;
}

Particles view(gz_context *c)
{
    Particles ps{};
    ps.n = c->n;
    ps.x = ptr<double>(c->x); ps.y = ptr<double>(c->y); ps.z = ptr<double>(c->z);
    ps.vx = ptr<double>(c->vx); ps.vy = ptr<double>(c->vy); ps.vz = ptr<double>(c->vz);
    ps.m = ptr<double>(c->m); ps.u = ptr<double>(c->u); ps.dt = ptr<double>(c->dt);
    ps.h = ptr<double>(c->h); ps.cond = ptr<double>(c->cond);
    ps.num_ngb = ptr<double>(c->num_ngb); ps.drkern = ptr<double>(c->drkern); ps.divvel = ptr<double>(c->divvel);
    ps.rho = ptr<double>(c->rho); ps.pressure = ptr<double>(c->pressure); ps.fce = ptr<double>(c->fce);
    ps.nvt = ptr<double>(c->nvt); ps.pv = ptr<double>(c->pv); ps.grad = ptr<double>(c->grad);
    ps.accel = ptr<double>(c->accel); ps.dudt = ptr<double>(c->dudt); ps.vsig = ptr<double>(c->vsig);
    ps.dtmass = ptr<double>(c->dtmass); ps.dmass = ptr<double>(c->dmass); ps.gw = ptr<double>(c->gw);
    ps.fabs = ptr<double>(c->fabs3);
    ps.iters = ptr<int>(c->iters);
    ps.active = ptr<unsigned char>(c->active);
    if (c->have_bins) {
        ps.timebin = ptr<int>(c->timebin);
        ps.vsig_prev = ptr<double>(c->vsig_prev);
        ps.wakeup = ptr<int>(c->wakeup);
        ps.bin_active = c->binact_on ? ptr<int>(c->binact) : nullptr;
    }
    return ps;
}

std::vector<DevBuf *> all_buffers(gz_context *c)
{
    return {&c->x, &c->y, &c->z, &c->vx, &c->vy, &c->vz, &c->m, &c->u, &c->dt, &c->h, &c->cond, &c->num_ngb,
            &c->drkern, &c->divvel, &c->rho, &c->pressure, &c->fce, &c->nvt, &c->pv, &c->grad, &c->accel,
            &c->dudt, &c->vsig, &c->dtmass, &c->dmass, &c->gw, &c->fabs3, &c->iters, &c->active, &c->stage, &c->stage3,
            &c->perm, &c->inv, &c->keys, &c->keys_sorted, &c->idx, &c->cub_tmp, &c->targets_orig,
            &c->targets, &c->targets_tmp, &c->t_node, &c->t_lo, &c->t_hi, &c->t_parent, &c->t_done, &c->t_nch,
            &c->t_cpos, &c->acc, &c->h_built, &c->scratch, &c->keep, &c->regrow, &c->todo_a, &c->todo_b, &c->grow,
            &c->d_beg, &c->d_end, &c->flag, &c->counts, &c->d_off, &c->d_nbr, &c->n_sel, &c->s_off, &c->s_nbr,
            &c->s_counts, &c->rec, &c->work, &c->hmax, &c->refined, &c->rq, &c->pad_over, &c->pad_list, &c->pad_sum, &c->pad_counts, &c->s_acnt, &c->s_bcnt, &c->s_tmp, &c->pflux, &c->status, &c->o_vel, &c->o_mass, &c->o_u, &c->o_dt, &c->o_h, &c->o_cond, &c->dl, &c->o_timebin,
            &c->o_vsig, &c->timebin, &c->vsig_prev, &c->wakeup, &c->binact, &c->sel_flags, &c->sel_out,
            &c->gstate, &c->g_hseed, &c->g_cseed, &c->g_over_list, &c->g_over_off, &c->g_sel,
            &c->p_stage3, &c->p_vel, &c->p_mass, &c->p_u, &c->p_dt, &c->p_h, &c->p_cond, &c->dstage,
            &c->box_bid, &c->box_of, &c->root_of, &c->t_build};
}

Tree tree_view(gz_context *c)
{
    Tree t{};
    t.box = c->prm.box_size;
    t.n_nodes = c->t_nodes;
    t.n_particles = c->n;
    t.node = ptr<int4>(c->t_node);
    t.lo = ptr<double4>(c->t_lo);
    t.hi = ptr<double4>(c->t_hi);
    if (c->box_bits) {
        t.box_of = ptr<int>(c->box_of);
        t.root_of = ptr<int>(c->root_of);
    }
    return t;
}


// ---------------------------------------------------------------- kernels
// Gathers positions/velocities into sorted order. Positions must lie in
// [0, box) (the periodic domain the octree covers; the search prunes nodes
// by their geometric boxes): others are reported as GZ_ERR_ARG.
__global__ void k_gather_inputs(int n, const int *__restrict__ perm, const double *__restrict__ pos,
                                const double *__restrict__ vel, double *x, double *y, double *z, double *vx,
                                double *vy, double *vz, double box, DevStatus *st)
{
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n) return;
    const size_t o = (size_t)perm[s];
    const double px = pos[3 * o], py = pos[3 * o + 1], pz = pos[3 * o + 2];
    if (!(px >= 0 && px < box && py >= 0 && py < box && pz >= 0 && pz < box)) record_status(st, GZ_ERR_ARG, s);
    x[s] = px; y[s] = py; z[s] = pz;
    vx[s] = vel[3 * o]; vy[s] = vel[3 * o + 1]; vz[s] = vel[3 * o + 2];
}

__global__ void k_gather1(int n, const int *__restrict__ perm, const double *__restrict__ src, double *dst)
{
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s < n) dst[s] = src[perm[s]];
}

__global__ void k_gather_int(int n, const int *__restrict__ perm, const int *__restrict__ src, int *dst)
{
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s < n) dst[s] = src[perm[s]];
}

// flag[i] = 1 for a cell of an active bin with positive mass, original order
// (make_list_of_active_particles, core/run.cc:997-1010)
__global__ void k_active_flags(int n, const int *__restrict__ timebin, const double *__restrict__ mass,
                               const int *__restrict__ bin_active, int *flag)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) flag[i] = (bin_active[timebin[i]] && mass[i] > 0) ? 1 : 0;
}

// process_wake_ups' bin rule (core/timestep.cc:1565-1700), per sorted cell, written in original order
__global__ void k_wakeup_bins(int n, const int *__restrict__ perm, const int *__restrict__ timebin,
                              const int *__restrict__ wakeup, const double *__restrict__ mass,
                              const int *__restrict__ bin_active, int max_active, int lowest, int *out,
                              unsigned long long *moved)
{
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    bool mv = false;
    if (s < n) {
        const int binold = timebin[s];
        int bin = binold;
        if (wakeup[s] && mass[s] > 0 && !bin_active[binold]) {
            int offset = 0;  // the bins WAKEUP spans: the smallest k with 2^k >= WAKEUP
            while ((double)(1ll << offset) < kWakeup) offset++;
            if (wakeup[s] > 0) {
                bin = wakeup[s] - 1 - offset;  // wakeup_timebin_from_flag, core/proto.h:182
                if (bin < 0) bin = 0;
                if (bin < lowest) bin = lowest;
            } else {
                bin = max_active;
            }
            if (bin > max_active) bin = max_active;
            if (bin >= binold) bin = binold;
        }
        out[perm[s]] = bin;
        mv = bin != binold;
    }
    const unsigned b = __ballot_sync(0xffffffffu, mv);
    if ((threadIdx.x & 31) == 0 && b) atomicAdd(moved, (unsigned long long)__popc(b));
}

__global__ void k_inverse(int n, const int *__restrict__ perm, int *inv)
{
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s < n) inv[perm[s]] = s;
}

// sorted field (component-major [k][n]) -> original order row-major [n][k]
__global__ void k_scatter_out(int n, int k, const int *__restrict__ perm, const double *__restrict__ src, double *dst)
{
    const long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (e >= (long long)n * k) return;
    const int s = (int)(e / k), c = (int)(e % k);
    dst[(size_t)perm[s] * k + c] = src[(size_t)c * n + s];
}

__global__ void k_scatter_int(int n, const int *__restrict__ perm, const int *__restrict__ src, int *dst)
{
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s < n) dst[perm[s]] = src[s];
}

__global__ void k_map_targets(int na, const int *__restrict__ orig, const int *__restrict__ inv, int *out, int n,
                              DevStatus *st)
{
    const int a = blockIdx.x * blockDim.x + threadIdx.x;
    if (a >= na) return;
    const int o = orig[a];
    if (o < 0 || o >= n) { record_status(st, GZ_ERR_ARG, o); out[a] = 0; return; }
    out[a] = inv[o];
}

__global__ void k_iota(int n, int *out)
{
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s < n) out[s] = s;
}

__global__ void k_set_active(int na, const int *__restrict__ t, unsigned char *flag)
{
    const int a = blockIdx.x * blockDim.x + threadIdx.x;
    if (a < na) flag[t[a]] = 1;
}

__global__ void k_density_prep(int na, const int *__restrict__ t, double *h, double maxsoft, DensityScratch *sc,
                               unsigned long long *hmax)
{
    const int a = blockIdx.x * blockDim.x + threadIdx.x;
    double hv = 0;
    if (a < na) {
        const int i = t[a];
        hv = h[i];
        if ((hv < 0) || !isfinite(hv) || (hv > 0.99 * maxsoft)) hv = 0.99 * maxsoft;  // density_loop.cc:837-840
        h[i] = hv;
        DensityScratch z{};
        sc[i] = z;
    }
    warp_atomic_max_nonneg(hmax, hv);  // every lane of the (whole) block's warps
}

// search radius of the density rows about to be built for t[0..na)
__global__ void k_row_radius(int na, const int *__restrict__ t, const double *__restrict__ h, double f, double *h_built)
{
    const int a = blockIdx.x * blockDim.x + threadIdx.x;
    if (a < na) h_built[t[a]] = h[t[a]] * f;
}

// rows just built for t[0..na) at nbr + base: record them per particle
__global__ void k_set_rows(int na, const int *__restrict__ t, const long long *__restrict__ off, long long base,
                           long long *beg, long long *end)
{
    const int a = blockIdx.x * blockDim.x + threadIdx.x;
    if (a >= na) return;
    beg[t[a]] = base + off[a];
    end[t[a]] = base + off[a + 1];
}

// ------------------------------------------------------------ host helpers
int sort_targets(gz_context *c, const int *active, int n_active, int *n_out)
{
    const int n = c->n;
    cudaStream_t s = c->stream;
    if (!active) {
        if (ensure(c, c->targets, sizeof(int) * (size_t)std::max(n, 1))) return c->err;
        if (n > 0) { k_iota<<<(n + 255) / 256, 256, 0, s>>>(n, ptr<int>(c->targets)); c->launches++; }
        *n_out = n;
    } else {
        if (n_active < 0 || n_active > n) return fail(c, GZ_ERR_ARG, "n_active out of range");
        const size_t na = (size_t)std::max(n_active, 1);
        if (ensure(c, c->targets_orig, sizeof(int) * na) || ensure(c, c->targets_tmp, sizeof(int) * na) ||
            ensure(c, c->targets, sizeof(int) * na))
            return c->err;
        GZ_CUDA(c, cudaMemcpyAsync(c->targets_orig.p, active, sizeof(int) * (size_t)n_active, cudaMemcpyHostToDevice, s));
        if (n_active > 0) {
            k_map_targets<<<(n_active + 255) / 256, 256, 0, s>>>(n_active, ptr<int>(c->targets_orig), ptr<int>(c->inv),
                                                                 ptr<int>(c->targets_tmp), n, ptr<DevStatus>(c->status));
            c->launches++;
        }
        size_t tmp = 0;
        cub::DeviceRadixSort::SortKeys(nullptr, tmp, ptr<int>(c->targets_tmp), ptr<int>(c->targets), n_active, 0, 32, s);
        if (ensure(c, c->cub_tmp, tmp)) return c->err;
        cub::DeviceRadixSort::SortKeys(c->cub_tmp.p, tmp, ptr<int>(c->targets_tmp), ptr<int>(c->targets), n_active, 0,
                                       32, s);
        *n_out = n_active;
    }
    GZ_CUDA(c, cudaMemsetAsync(c->active.p, 0, (size_t)std::max(n, 1), s));
    if (*n_out > 0) {
        k_set_active<<<(*n_out + 255) / 256, 256, 0, s>>>(*n_out, ptr<int>(c->targets), ptr<unsigned char>(c->active));
        c->launches++;
    }
    return 0;
}

// off[0] = 0, off[r + 1] = counts[0] + ... + counts[r]; counts are 64-bit so
// that the scan accumulates in 64 bits (row totals can pass 2^31).
int exclusive_scan_counts(gz_context *c, int rows, DevBuf &counts, DevBuf &off, long long *total)
{
    cudaStream_t s = c->stream;
    if (ensure(c, off, sizeof(long long) * (size_t)(rows + 1))) return c->err;
    GZ_CUDA(c, cudaMemsetAsync(off.p, 0, sizeof(long long), s));
    if (rows > 0) {
        size_t tmp = 0;
        cub::DeviceScan::InclusiveSum(nullptr, tmp, ptr<long long>(counts), ptr<long long>(off) + 1, rows, s);
        if (ensure(c, c->cub_tmp, tmp)) return c->err;
        cub::DeviceScan::InclusiveSum(c->cub_tmp.p, tmp, ptr<long long>(counts), ptr<long long>(off) + 1, rows, s);
    }
    GZ_CUDA(c, cudaMemcpyAsync(total, ptr<long long>(off) + rows, sizeof(long long), cudaMemcpyDeviceToHost, s));
    GZ_CUDA(c, cudaStreamSynchronize(s));
    return 0;
}

// nbr holds at least `need` ints, its first `keep` kept if it must grow
int grow_keep(gz_context *c, DevBuf &nbr, long long &cap, long long keep, long long need)
{
    if (need <= cap && nbr.p) return 0;
    cudaStream_t s = c->stream;
    const long long want = std::max(need, keep > 0 ? cap + cap / 2 : 0ll);
    DevBuf grown;
    if (ensure(c, grown, sizeof(int) * (size_t)std::max(want, 1ll))) return c->err;
    if (keep > 0) GZ_CUDA(c, cudaMemcpyAsync(grown.p, nbr.p, sizeof(int) * (size_t)keep, cudaMemcpyDeviceToDevice, s));
    GZ_CUDA(c, cudaStreamSynchronize(s));
    release(nbr);
    nbr = grown;
    cap = (long long)(nbr.bytes / sizeof(int));
    return 0;
}

// Exact neighbour rows of `targets` (count walk, scan, fill walk), written
// at nbr + base; the first `base` entries of nbr are kept if it must grow.
int build_rows(gz_context *c, const double *reach, int symmetric, const int *targets, int rows, DevBuf &counts,
               DevBuf &off, DevBuf &nbr, long long &cap, long long *total, long long base = 0)
{
    cudaStream_t s = c->stream;
    Tree t = tree_view(c);
    if (ensure(c, counts, sizeof(long long) * (size_t)std::max(rows, 1)) || ensure(c, c->work, sizeof(int)))
        return c->err;
    walk_timed(c, t, ptr<double>(c->x), ptr<double>(c->y), ptr<double>(c->z), reach, ptr<double>(c->h), symmetric, targets,
              rows, ptr<long long>(counts), nullptr, nullptr, 0, ptr<DevStatus>(c->status), ptr<int>(c->work), s);
    if (rows > 0) c->launches++;
    GZ_CUDA(c, cudaGetLastError());
    if (exclusive_scan_counts(c, rows, counts, off, total)) return c->err;
    if (base + *total > (long long)INT32_MAX * 4) return fail(c, GZ_ERR_CAPACITY, "neighbour rows exceed capacity");
    if (grow_keep(c, nbr, cap, base, base + *total)) return c->err;
    walk_timed(c, t, ptr<double>(c->x), ptr<double>(c->y), ptr<double>(c->z), reach, ptr<double>(c->h), symmetric, targets,
              rows, ptr<long long>(counts), ptr<long long>(off), ptr<int>(nbr) + base, 0, ptr<DevStatus>(c->status),
              ptr<int>(c->work), s);
    if (rows > 0) c->launches++;
    GZ_CUDA(c, cudaGetLastError());
    return 0;
}

// Density rows of `targets` in one walk: cap slots per target at d_nbr + base
// (rows [beg, end) per particle); a row longer than cap is rebuilt by the
// two-pass build behind the padded block. Returns the entries now in use and
// the row entries built.
int build_rows_padded(gz_context *c, const double *reach, const int *targets, int rows, int cap, long long base,
                      long long *used, long long *entries)
{
    cudaStream_t s = c->stream;
    const long long need = base + (long long)rows * cap;
    if (need > (long long)INT32_MAX * 4) return fail(c, GZ_ERR_CAPACITY, "neighbour rows exceed capacity");
    if (grow_keep(c, c->d_nbr, c->d_nbr_cap, base, need)) return c->err;
    const size_t R = (size_t)std::max(rows, 1);
    if (ensure(c, c->counts, sizeof(long long) * R) || ensure(c, c->work, sizeof(int)) ||
        ensure(c, c->pad_over, R) || ensure(c, c->pad_list, sizeof(int) * R) || ensure(c, c->n_sel, sizeof(int) * 2))
        return c->err;
    Tree t = tree_view(c);
    walk_timed(c, t, ptr<double>(c->x), ptr<double>(c->y), ptr<double>(c->z), reach, ptr<double>(c->h), 0, targets, rows,
              ptr<long long>(c->counts), nullptr, ptr<int>(c->d_nbr) + base, cap, ptr<DevStatus>(c->status),
              ptr<int>(c->work), s);
    padded_rows(rows, targets, ptr<long long>(c->counts), cap, base, ptr<long long>(c->d_beg), ptr<long long>(c->d_end),
                ptr<unsigned char>(c->pad_over), s);
    c->launches += 2;
    GZ_CUDA(c, cudaGetLastError());
    // rows built: sum of the counts; rows over their cap: compacted list
    size_t t1 = 0, t2 = 0;
    cub::DeviceReduce::Sum(nullptr, t1, ptr<long long>(c->counts), ptr<long long>(c->pad_sum), rows, s);
    cub::DeviceSelect::Flagged(nullptr, t2, targets, ptr<unsigned char>(c->pad_over), ptr<int>(c->pad_list),
                               ptr<int>(c->n_sel), rows, s);
    if (ensure(c, c->pad_sum, sizeof(long long)) || ensure(c, c->cub_tmp, std::max(t1, t2))) return c->err;
    cub::DeviceReduce::Sum(c->cub_tmp.p, t1, ptr<long long>(c->counts), ptr<long long>(c->pad_sum), rows, s);
    long long built = 0;
    GZ_CUDA(c, cudaMemcpyAsync(&built, c->pad_sum.p, sizeof(long long), cudaMemcpyDeviceToHost, s));
    cub::DeviceSelect::Flagged(c->cub_tmp.p, t2, targets, ptr<unsigned char>(c->pad_over), ptr<int>(c->pad_list),
                               ptr<int>(c->n_sel), rows, s);
    int n_over = 0;
    GZ_CUDA(c, cudaMemcpyAsync(&n_over, c->n_sel.p, sizeof(int), cudaMemcpyDeviceToHost, s));
    GZ_CUDA(c, cudaStreamSynchronize(s));
    long long extra = 0;
    if (n_over > 0) {
        // the padded walk took every row's full count: the longer rows need the
        // fill walk only, at offsets from those counts
        if (ensure(c, c->pad_counts, sizeof(long long) * (size_t)n_over)) return c->err;
        size_t t3 = 0;
        cub::DeviceSelect::Flagged(nullptr, t3, ptr<long long>(c->counts), ptr<unsigned char>(c->pad_over),
                                   ptr<long long>(c->pad_counts), ptr<int>(c->n_sel) + 1, rows, s);
        if (ensure(c, c->cub_tmp, t3)) return c->err;
        cub::DeviceSelect::Flagged(c->cub_tmp.p, t3, ptr<long long>(c->counts), ptr<unsigned char>(c->pad_over),
                                   ptr<long long>(c->pad_counts), ptr<int>(c->n_sel) + 1, rows, s);
        if (exclusive_scan_counts(c, n_over, c->pad_counts, c->d_off, &extra)) return c->err;
        if (need + extra > (long long)INT32_MAX * 4) return fail(c, GZ_ERR_CAPACITY, "neighbour rows exceed capacity");
        if (grow_keep(c, c->d_nbr, c->d_nbr_cap, need, need + extra)) return c->err;
        walk_timed(c, t, ptr<double>(c->x), ptr<double>(c->y), ptr<double>(c->z), reach, ptr<double>(c->h), 0,
                  ptr<int>(c->pad_list), n_over, ptr<long long>(c->pad_counts), ptr<long long>(c->d_off),
                  ptr<int>(c->d_nbr) + need, 0, ptr<DevStatus>(c->status), ptr<int>(c->work), s);
        k_set_rows<<<(n_over + 255) / 256, 256, 0, s>>>(n_over, ptr<int>(c->pad_list), ptr<long long>(c->d_off), need,
                                                        ptr<long long>(c->d_beg), ptr<long long>(c->d_end));
        c->launches += 2;
        GZ_CUDA(c, cudaGetLastError());
    }
    *used = need + extra;
    *entries = built;
    return 0;
}

// the copy stream and events of the pipelined transfers, made on first use
int copy_stream(gz_context *c)
{
    if (c->cstream) return 0;
    GZ_CUDA(c, cudaStreamCreateWithFlags(&c->cstream, cudaStreamNonBlocking));
    cudaEvent_t *ev[] = {&c->ev_in_free, &c->ev_in_done, &c->ev_out_ready, &c->ev_out_done};
    for (cudaEvent_t *e : ev) GZ_CUDA(c, cudaEventCreateWithFlags(e, cudaEventDisableTiming));
    return 0;
}

// inputs of a pipelined upload become the resident ones: the context's stream
// waits for their copies, and the buffers trade places (no copy)
int take_pending_inputs(gz_context *c, bool copy = false)
{
    if (!c->in_pending) return 0;
    GZ_CUDA(c, cudaStreamWaitEvent(c->stream, c->ev_in_done, 0));
    if (copy) {  // into the resident buffers, which keep their addresses
        const size_t N = (size_t)c->n;
        struct { DevBuf *dst, *src; size_t k; } f[] = {
            {&c->stage3, &c->p_stage3, 3}, {&c->o_vel, &c->p_vel, 3}, {&c->o_mass, &c->p_mass, 1},
            {&c->o_u, &c->p_u, 1}, {&c->o_dt, &c->p_dt, 1}, {&c->o_h, &c->p_h, 1}, {&c->o_cond, &c->p_cond, 1}};
        for (auto &e : f)
            GZ_CUDA(c, cudaMemcpyAsync(e.dst->p, e.src->p, sizeof(double) * e.k * N, cudaMemcpyDeviceToDevice,
                                       c->stream));
        c->in_pending = false;
        return 0;
    }
    std::swap(c->stage3, c->p_stage3);
    std::swap(c->o_vel, c->p_vel);
    std::swap(c->o_mass, c->p_mass);
    std::swap(c->o_u, c->p_u);
    std::swap(c->o_dt, c->p_dt);
    std::swap(c->o_h, c->p_h);
    std::swap(c->o_cond, c->p_cond);
    c->in_pending = false;
    return 0;
}

int read_status(gz_context *c)
{
    DevStatus h{};
    GZ_CUDA(c, cudaMemcpyAsync(&h, c->status.p, sizeof(DevStatus), cudaMemcpyDeviceToHost, c->stream));
    GZ_CUDA(c, cudaStreamSynchronize(c->stream));
    if (h.code && !c->err) {
        c->err = h.code;
        c->err_index = h.index;
        snprintf(c->msg, sizeof(c->msg), "device status %d at sorted index %d", h.code, h.index);
    }
    return h.code;
}

int build_grid(gz_context *c)
{
    const int n = c->n;
    cudaStream_t s = c->stream;
    const size_t N = (size_t)std::max(n, 1);
    if (ensure(c, c->keys, sizeof(unsigned long long) * N) || ensure(c, c->keys_sorted, sizeof(unsigned long long) * N) ||
        ensure(c, c->idx, sizeof(int) * N))
        return c->err;
    grid_keys(n, ptr<double>(c->stage3), c->prm.box_size, c->box_bits ? ptr<int>(c->box_bid) : nullptr,
              21 - c->box_bits / 3, ptr<unsigned long long>(c->keys), ptr<int>(c->idx), s);
    size_t tmp = 0;
    cub::DeviceRadixSort::SortPairs(nullptr, tmp, ptr<unsigned long long>(c->keys),
                                    ptr<unsigned long long>(c->keys_sorted), ptr<int>(c->idx), ptr<int>(c->perm), n, 0,
                                    63, s);
    if (ensure(c, c->cub_tmp, tmp)) return c->err;
    cub::DeviceRadixSort::SortPairs(c->cub_tmp.p, tmp, ptr<unsigned long long>(c->keys),
                                    ptr<unsigned long long>(c->keys_sorted), ptr<int>(c->idx), ptr<int>(c->perm), n, 0,
                                    63, s);
    if (n > 0) k_inverse<<<(n + 255) / 256, 256, 0, s>>>(n, ptr<int>(c->perm), ptr<int>(c->inv));
    if (c->box_bits && n > 0) {
        if (ensure(c, c->box_of, sizeof(int) * N) ||
            ensure(c, c->root_of, sizeof(int) * std::max<size_t>(c->box_counts.size(), 1)))
            return c->err;
        k_gather_int<<<(n + 255) / 256, 256, 0, s>>>(n, ptr<int>(c->perm), ptr<int>(c->box_bid), ptr<int>(c->box_of));
        GZ_CUDA(c, cudaMemsetAsync(c->root_of.p, 0xff, sizeof(int) * c->box_counts.size(), s));
        c->launches++;
    }
    GZ_CUDA(c, cudaGetLastError());
    return 0;
}

// Octree over the sorted keys, split top-down one level per step with the size
// of the next level read back each step (the fallback of build_tree).
int build_tree_levels(gz_context *c)
{
    const int n = c->n;
    cudaStream_t s = c->stream;
    c->t_nodes = 0;
    c->t_levels = 0;
    if (n == 0) return 0;
    long long cap = std::max<long long>(1024, n / 4);
    if (c->t_node.bytes >= sizeof(int4) * 1024) cap = std::max<long long>(cap, (long long)(c->t_node.bytes / sizeof(int4)));
    if (ensure(c, c->t_node, sizeof(int4) * (size_t)cap) || ensure(c, c->t_parent, sizeof(int) * (size_t)cap))
        return c->err;
    const int4 root = make_int4(0, n, -1, 0);
    const int no_parent = -1;
    GZ_CUDA(c, cudaMemcpyAsync(c->t_node.p, &root, sizeof(int4), cudaMemcpyHostToDevice, s));
    GZ_CUDA(c, cudaMemcpyAsync(c->t_parent.p, &no_parent, sizeof(int), cudaMemcpyHostToDevice, s));
    int beg = 0, cnt = 1, L = 0;
    const unsigned long long *keys = ptr<unsigned long long>(c->keys_sorted);
    const int split_levels = c->box_bits / 3;
    while (cnt > 0) {
        if (ensure(c, c->t_nch, sizeof(long long) * (size_t)cnt)) return c->err;
        if (c->box_bits && L == split_levels) {  // one node per box
            box_roots(beg, cnt, ptr<int4>(c->t_node), ptr<int>(c->box_of), ptr<int>(c->root_of), s);
            c->launches++;
        }
        tree_count(keys, L, ptr<int4>(c->t_node), beg, cnt, ptr<long long>(c->t_nch), c->leaf_max, split_levels, s);
        c->launches++;
        long long next = 0;
        if (exclusive_scan_counts(c, cnt, c->t_nch, c->t_cpos, &next)) return c->err;
        const long long end = (long long)beg + cnt;
        if (end + next > INT32_MAX) return fail(c, GZ_ERR_CAPACITY, "octree exceeds capacity");
        if (end + next > cap) {
            // grow, keeping the nodes built so far
            const long long want = std::max(end + next, cap * 2);
            DevBuf gn, gp;
            if (ensure(c, gn, sizeof(int4) * (size_t)want) || ensure(c, gp, sizeof(int) * (size_t)want)) return c->err;
            GZ_CUDA(c, cudaMemcpyAsync(gn.p, c->t_node.p, sizeof(int4) * (size_t)end, cudaMemcpyDeviceToDevice, s));
            GZ_CUDA(c, cudaMemcpyAsync(gp.p, c->t_parent.p, sizeof(int) * (size_t)end, cudaMemcpyDeviceToDevice, s));
            GZ_CUDA(c, cudaStreamSynchronize(s));
            release(c->t_node);
            release(c->t_parent);
            c->t_node = gn;
            c->t_parent = gp;
            cap = want;
        }
        tree_write(keys, L, ptr<int4>(c->t_node), ptr<int>(c->t_parent), beg, cnt, ptr<long long>(c->t_cpos), (int)end, s);
        c->launches++;
        GZ_CUDA(c, cudaGetLastError());
        beg = (int)end;
        cnt = (int)next;
        L++;
    }
    c->t_nodes = beg;
    c->t_levels = L;
    if (ensure(c, c->t_lo, sizeof(double4) * (size_t)c->t_nodes) || ensure(c, c->t_hi, sizeof(double4) * (size_t)c->t_nodes) ||
        ensure(c, c->t_done, sizeof(int) * (size_t)c->t_nodes))
        return c->err;
    tree_up(c->t_nodes, ptr<int4>(c->t_node), ptr<int>(c->t_parent), ptr<double>(c->x), ptr<double>(c->y),
            ptr<double>(c->z), ptr<double>(c->h), ptr<double4>(c->t_lo), ptr<double4>(c->t_hi), ptr<int>(c->t_done), 1, s);
    c->launches++;
    GZ_CUDA(c, cudaGetLastError());
    return 0;
}

// nodes held for the octree of c->n particles (and its box sets)
long long tree_cap(const gz_context *c)
{
    return std::max<long long>(4096, c->n / 4) + 2 * (long long)c->box_counts.size() + 64;
}

// Octree over the sorted keys, all levels on the device (tree_build_device)
// with one read-back of the node count at the end, then boxes and h maxima
// bottom-up. A tree larger than the nodes held for it (a few coincident
// particles split down to the deepest level) is built level by level instead.
int build_tree(gz_context *c)
{
    const int n = c->n;
    cudaStream_t s = c->stream;
    c->t_nodes = 0;
    c->t_levels = 0;
    if (n == 0) return 0;
    const long long cap = tree_cap(c);
    if (cap > INT32_MAX) return fail(c, GZ_ERR_CAPACITY, "octree exceeds capacity");
    if (ensure(c, c->t_node, sizeof(int4) * (size_t)cap) || ensure(c, c->t_parent, sizeof(int) * (size_t)cap) ||
        ensure(c, c->t_build, sizeof(TreeBuild)))
        return c->err;
    tree_build_device(ptr<unsigned long long>(c->keys_sorted), n, ptr<int4>(c->t_node), ptr<int>(c->t_parent),
                      ptr<TreeBuild>(c->t_build), (int)cap, c->leaf_max, c->box_bits / 3,
                      c->box_bits ? ptr<int>(c->box_of) : nullptr, c->box_bits ? ptr<int>(c->root_of) : nullptr,
                      c->sms * 8, s);
    c->launches += 1 + 2 * 22;
    TreeBuild tb{};
    GZ_CUDA(c, cudaMemcpyAsync(&tb, c->t_build.p, sizeof(tb), cudaMemcpyDeviceToHost, s));
    GZ_CUDA(c, cudaStreamSynchronize(s));
    if (tb.fail) return build_tree_levels(c);
    c->t_nodes = tb.total;
    c->t_levels = tb.L;
    if (ensure(c, c->t_lo, sizeof(double4) * (size_t)c->t_nodes) || ensure(c, c->t_hi, sizeof(double4) * (size_t)c->t_nodes) ||
        ensure(c, c->t_done, sizeof(int) * (size_t)c->t_nodes))
        return c->err;
    tree_up(c->t_nodes, ptr<int4>(c->t_node), ptr<int>(c->t_parent), ptr<double>(c->x), ptr<double>(c->y),
            ptr<double>(c->z), ptr<double>(c->h), ptr<double4>(c->t_lo), ptr<double4>(c->t_hi), ptr<int>(c->t_done), 1, s);
    c->launches++;
    GZ_CUDA(c, cudaGetLastError());
    return 0;
}

// node maxima of h after the radii changed
int refresh_hmax(gz_context *c)
{
    tree_up(c->t_nodes, ptr<int4>(c->t_node), ptr<int>(c->t_parent), ptr<double>(c->x), ptr<double>(c->y),
            ptr<double>(c->z), ptr<double>(c->h), ptr<double4>(c->t_lo), ptr<double4>(c->t_hi), ptr<int>(c->t_done), 0,
            c->stream);
    if (c->t_nodes > 0) c->launches++;
    GZ_CUDA(c, cudaGetLastError());
    return 0;
}

// Symmetric rows of all particles from the density rows of a pass over all
// particles: A_i (the converged one-way row) plus B_i (the pairs reached only
// from j's side), sorted -- the walk's rows, without a second walk.
int sym_rows_from_density(gz_context *c)
{
    const int n = c->n;
    cudaStream_t s = c->stream;
    const size_t N = (size_t)std::max(n, 1);
    if (ensure(c, c->s_acnt, sizeof(int) * N) || ensure(c, c->s_bcnt, sizeof(int) * N) ||
        ensure(c, c->s_counts, sizeof(long long) * N))
        return c->err;
    GZ_CUDA(c, cudaMemsetAsync(c->s_bcnt.p, 0, sizeof(int) * N, s));
    sym_split(n, ptr<double>(c->x), ptr<double>(c->y), ptr<double>(c->z), ptr<double>(c->h), c->prm.box_size,
              ptr<long long>(c->d_beg), ptr<long long>(c->d_end), ptr<int>(c->d_nbr), ptr<int>(c->s_acnt),
              ptr<int>(c->s_bcnt), s);
    sym_counts(n, ptr<int>(c->s_acnt), ptr<int>(c->s_bcnt), ptr<long long>(c->s_counts), s);
    c->launches += 2;
    GZ_CUDA(c, cudaGetLastError());
    c->dens_all = false;  // the density rows are compacted in place: consumed
    long long total = 0;
    if (exclusive_scan_counts(c, n, c->s_counts, c->s_off, &total)) return c->err;
    if (total > (long long)INT32_MAX * 4) return fail(c, GZ_ERR_CAPACITY, "neighbour rows exceed capacity");
    if (ensure(c, c->s_tmp, sizeof(int) * (size_t)std::max(total, 1ll))) return c->err;
    if (total > c->s_nbr_cap || !c->s_nbr.p) {
        if (ensure(c, c->s_nbr, sizeof(int) * (size_t)std::max(total, 1ll))) return c->err;
        c->s_nbr_cap = (long long)(c->s_nbr.bytes / sizeof(int));
    }
    GZ_CUDA(c, cudaMemsetAsync(c->s_bcnt.p, 0, sizeof(int) * N, s));  // reused as the B cursors
    sym_scatter(n, ptr<long long>(c->d_beg), ptr<int>(c->d_nbr), ptr<int>(c->s_acnt), ptr<long long>(c->s_off),
                ptr<int>(c->s_bcnt), ptr<int>(c->s_tmp), s);
    sym_sort(n, ptr<long long>(c->s_off), ptr<int>(c->s_acnt), ptr<int>(c->s_tmp), ptr<int>(c->s_nbr), s);
    c->launches += 2;
    GZ_CUDA(c, cudaGetLastError());
    c->pairs_symmetric = total;
    return 0;
}

int build_sym_rows(gz_context *c, int rows, bool all)
{
    if (all && c->dens_all && rows == c->n && c->n > 0) {
        if (sym_rows_from_density(c)) return c->err;
    } else {
        if (refresh_hmax(c)) return c->err;
        long long total = 0;
        if (build_rows(c, ptr<double>(c->h), 1, ptr<int>(c->targets), rows, c->s_counts, c->s_off, c->s_nbr,
                       c->s_nbr_cap, &total))
            return c->err;
        c->pairs_symmetric = total;
    }
    c->sym_rows = rows;
    c->sym_valid = true;
    return 0;
}

// The octree built on the device with nothing read back: the bottom-up pass
// covers the nodes held and stops at the count the build left on the device.
int enqueue_tree_device(gz_context *c)
{
    const long long cap = tree_cap(c);
    cudaStream_t s = c->stream;
    tree_build_device(ptr<unsigned long long>(c->keys_sorted), c->n, ptr<int4>(c->t_node), ptr<int>(c->t_parent),
                      ptr<TreeBuild>(c->t_build), (int)cap, c->leaf_max, c->box_bits / 3,
                      c->box_bits ? ptr<int>(c->box_of) : nullptr, c->box_bits ? ptr<int>(c->root_of) : nullptr,
                      c->sms * 8, s);
    tree_up((int)cap, ptr<int4>(c->t_node), ptr<int>(c->t_parent), ptr<double>(c->x), ptr<double>(c->y),
            ptr<double>(c->z), ptr<double>(c->h), ptr<double4>(c->t_lo), ptr<double4>(c->t_hi), ptr<int>(c->t_done), 1, s,
            &ptr<TreeBuild>(c->t_build)->total);
    GZ_CUDA(c, cudaGetLastError());
    return 0;
}

// The restage's device work: status cleared, keys, sort, the sorted mirror
// gathered from the resident inputs, outputs zeroed, the octree. in_graph (a
// restage captured into the pass's graph): the tree is built without its
// read-back (tree_build_device; the node count stays on the device and the
// bottom-up pass runs over the nodes held).
int enqueue_restage(gz_context *c, bool in_graph)
{
    const int n = c->n;
    cudaStream_t s = c->stream;
    GZ_CUDA(c, cudaMemsetAsync(c->status.p, 0, sizeof(DevStatus), s));
    if (n > 0) {
        if (build_grid(c)) return c->err;
        c->launches += 2;  // keys, inverse permutation
        const unsigned blocks = (unsigned)((n + 255) / 256);
        k_gather_inputs<<<blocks, 256, 0, s>>>(n, ptr<int>(c->perm), ptr<double>(c->stage3), ptr<double>(c->o_vel),
                                               ptr<double>(c->x), ptr<double>(c->y), ptr<double>(c->z),
                                               ptr<double>(c->vx), ptr<double>(c->vy), ptr<double>(c->vz),
                                               c->prm.box_size, ptr<DevStatus>(c->status));
        c->launches += 1;
        struct { DevBuf *src; DevBuf *dst; } one_in[] = {
            {&c->o_mass, &c->m}, {&c->o_u, &c->u}, {&c->o_dt, &c->dt}, {&c->o_h, &c->h}, {&c->o_cond, &c->cond}};
        for (auto &f : one_in) {
            k_gather1<<<blocks, 256, 0, s>>>(n, ptr<int>(c->perm), ptr<double>(*f.src), ptr<double>(*f.dst));
            c->launches += 1;
        }
        if (c->have_bins) {
            k_gather_int<<<blocks, 256, 0, s>>>(n, ptr<int>(c->perm), ptr<int>(c->o_timebin), ptr<int>(c->timebin));
            k_gather1<<<blocks, 256, 0, s>>>(n, ptr<int>(c->perm), ptr<double>(c->o_vsig), ptr<double>(c->vsig_prev));
            GZ_CUDA(c, cudaMemsetAsync(c->wakeup.p, 0, sizeof(int) * (size_t)n, s));
            c->launches += 2;
        }
        DevBuf *zero[] = {&c->num_ngb, &c->drkern, &c->divvel, &c->rho, &c->pressure, &c->fce, &c->dudt, &c->vsig,
                          &c->dtmass, &c->dmass};
        for (DevBuf *b : zero) GZ_CUDA(c, cudaMemsetAsync(b->p, 0, sizeof(double) * (size_t)n, s));
        GZ_CUDA(c, cudaMemsetAsync(c->nvt.p, 0, sizeof(double) * 6 * (size_t)n, s));
        GZ_CUDA(c, cudaMemsetAsync(c->pv.p, 0, sizeof(double) * 3 * (size_t)n, s));
        GZ_CUDA(c, cudaMemsetAsync(c->grad.p, 0, sizeof(double) * 15 * (size_t)n, s));
        GZ_CUDA(c, cudaMemsetAsync(c->accel.p, 0, sizeof(double) * 3 * (size_t)n, s));
        GZ_CUDA(c, cudaMemsetAsync(c->gw.p, 0, sizeof(double) * 3 * (size_t)n, s));
        GZ_CUDA(c, cudaMemsetAsync(c->fabs3.p, 0, sizeof(double) * 3 * (size_t)n, s));
        GZ_CUDA(c, cudaMemsetAsync(c->iters.p, 0, sizeof(int) * (size_t)n, s));
        GZ_CUDA(c, cudaGetLastError());
        if (in_graph ? enqueue_tree_device(c) : build_tree(c)) return c->err;
    }
    return 0;
}

// ------------------------------------------------- the pass as one CUDA graph
// gz_hydro_pass over every particle: density (the iteration as a WHILE node
// whose body is one iteration, sized from the device state), then, if every
// target converged, the symmetric rows from the density rows, and, if those
// fit their buffers, gradients and force (two nested IF nodes). The kernels
// are the plain pass's (the density rows, sums, after_iter, symmetric rows,
// gradient and force kernels) or their device-sized forms, which give every
// row the same entries and sums: only the order of the targets in the
// iteration's lists differs, and no result depends on it. A buffer that
// would overflow stops the graph's work (GraphState::fail); the host then
// restores the kernel lengths and condition numbers the graph started from
// and runs the plain pass.

__global__ void k_g_init(GraphState *gs, int n)
{
    GraphState g{};
    g.n_todo = n;
    g.n_grow = n;
    *gs = g;
}

// start of an iteration: this iteration's padded block and density lanes
__global__ void k_g_prep(GraphState *gs, int cap0, int cap1, long long nbr_cap, int n_particles,
                         long long group_warps, int sms)
{
    GraphState &g = *gs;
    g.n_next = 0;
    g.n_regrow = 0;
    g.n_over = 0;
    g.sums_next = 0;
    g.after_next = 0;
    g.extra = 0;
    g.next_group[0] = g.next_group[1] = 0;
    // lanes per density row: lanes_per_row(n_todo, 4)
    const long long want = (long long)sms * 2048 * 8;
    int tpt = 4;
    while (tpt < 16 && (long long)g.n_todo * tpt < want) tpt *= 2;
    g.tpt = tpt;
    g.need = g.base;
    if (g.n_grow > 0) {
        g.cap = g.iter == 0 ? cap0 : cap1;
        g.need = g.base + (long long)g.n_grow * g.cap;
        if (g.need > nbr_cap) g.fail |= kGraphFailRows;
        // the walk mode of walk_rows (both modes write the same rows)
        const bool sparse = (long long)g.n_grow * 4 < n_particles;
        g.walk_solo = (g.n_grow == 1 || (sparse && (g.n_grow + 31) / 32 < group_warps)) ? 1 : 0;
    }
}

__global__ void k_g_row_radius(const GraphState *gs, const int *__restrict__ first, const int *__restrict__ grow,
                               const double *__restrict__ h, double f0, double f1, double *h_built)
{
    if (gs->fail) return;
    const int n = gs->n_grow;
    const int *t = gs->iter == 0 ? first : grow;
    const double f = gs->iter == 0 ? f0 : f1;
    for (int a = blockIdx.x * blockDim.x + threadIdx.x; a < n; a += gridDim.x * blockDim.x) h_built[t[a]] = h[t[a]] * f;
}

// After the padded fill: a row that fit gets [base + a cap, + count), a longer
// one a place behind the block (its fill walk follows); the entries are counted.
__global__ void k_g_padded_rows(GraphState *gs, const int *__restrict__ first, const int *__restrict__ grow,
                                const long long *__restrict__ counts, long long *beg, long long *end, int *over_list,
                                long long *over_off)
{
    if (gs->fail) return;
    const int n = gs->n_grow, cap = gs->cap;
    const long long base = gs->base, need = gs->need;
    const int *t = gs->iter == 0 ? first : grow;
    long long built = 0;
    for (int a0 = blockIdx.x * blockDim.x + (threadIdx.x & ~31); a0 < n; a0 += gridDim.x * blockDim.x) {
        const int a = a0 + (threadIdx.x & 31);
        if (a < n) {
            const long long c = counts[a];
            built += c;
            const int i = t[a];
            if (c <= cap) {
                beg[i] = base + (long long)a * cap;
                end[i] = base + (long long)a * cap + c;
            } else {
                const int k = atomicAdd(&gs->n_over, 1);
                const long long o = (long long)atomicAdd((unsigned long long *)&gs->extra, (unsigned long long)c);
                over_list[k] = i;
                over_off[k] = o;
                beg[i] = need + o;
                end[i] = need + o + c;
            }
        }
    }
    for (int o = 16; o > 0; o >>= 1) built += __shfl_xor_sync(0xffffffffu, built, o);
    if ((threadIdx.x & 31) == 0 && built) atomicAdd((unsigned long long *)&gs->entries, (unsigned long long)built);
}

// the overflow rows' room, then the entries in use after this iteration
__global__ void k_g_over_check(GraphState *gs, long long nbr_cap)
{
    GraphState &g = *gs;
    if (g.fail || g.n_grow == 0) return;
    if (g.need + g.extra > nbr_cap) { g.fail |= kGraphFailRows; return; }
    g.base = g.need + g.extra;
}

// Stable selection of the flagged slots of this iteration's list (count on
// the device), in three steps over chunks of kSelChunk slots: each chunk's
// counts, their exclusive scan (one block), then each chunk's writes at its
// offset in slot order: the order CUB's DeviceSelect::Flagged gives the plain
// pass. Two flag arrays at once: still iterating -> `next`, radius outgrew
// its row -> `grow`.
constexpr int kSelChunk = 1024;
__global__ void __launch_bounds__(kSelChunk) k_sel_count(const GraphState *gs, const unsigned char *__restrict__ fa,
                                                         const unsigned char *__restrict__ fb, int *ca, int *cb)
{
    __shared__ int sa[32], sb[32];
    if (gs->fail) return;
    const int n = gs->n_todo, chunks = (n + kSelChunk - 1) / kSelChunk;
    for (int ch = blockIdx.x; ch < chunks; ch += gridDim.x) {
        const int i = ch * kSelChunk + threadIdx.x;
        const int a = (i < n) ? fa[i] : 0, b = (i < n) ? fb[i] : 0;
        const int wa = __popc(__ballot_sync(0xffffffffu, a)), wb = __popc(__ballot_sync(0xffffffffu, b));
        if ((threadIdx.x & 31) == 0) { sa[threadIdx.x >> 5] = wa; sb[threadIdx.x >> 5] = wb; }
        __syncthreads();
        if (threadIdx.x < 32) {
            int x = sa[threadIdx.x], y = sb[threadIdx.x];
            for (int o = 16; o > 0; o >>= 1) { x += __shfl_xor_sync(0xffffffffu, x, o); y += __shfl_xor_sync(0xffffffffu, y, o); }
            if (threadIdx.x == 0) { ca[ch] = x; cb[ch] = y; }
        }
        __syncthreads();
    }
}

// exclusive scan of the chunk counts in place; the totals into the state
__global__ void __launch_bounds__(kSelChunk) k_sel_scan(GraphState *gs, int *ca, int *cb)
{
    __shared__ int pa[kSelChunk], pb[kSelChunk];
    if (gs->fail) return;
    const int n = gs->n_todo, chunks = (n + kSelChunk - 1) / kSelChunk;
    // each thread scans a contiguous run of chunks, then the run totals are scanned
    const int per = (chunks + kSelChunk - 1) / kSelChunk;
    const int c0 = threadIdx.x * per, c1 = min(chunks, c0 + per);
    int ta = 0, tb = 0;
    for (int c = c0; c < c1; c++) { ta += ca[c]; tb += cb[c]; }
    pa[threadIdx.x] = ta;
    pb[threadIdx.x] = tb;
    __syncthreads();
    for (int o = 1; o < kSelChunk; o <<= 1) {
        const int xa = threadIdx.x >= o ? pa[threadIdx.x - o] : 0, xb = threadIdx.x >= o ? pb[threadIdx.x - o] : 0;
        __syncthreads();
        pa[threadIdx.x] += xa;
        pb[threadIdx.x] += xb;
        __syncthreads();
    }
    int oa = pa[threadIdx.x] - ta, ob = pb[threadIdx.x] - tb;  // exclusive
    for (int c = c0; c < c1; c++) {
        const int xa = ca[c], xb = cb[c];
        ca[c] = oa;
        cb[c] = ob;
        oa += xa;
        ob += xb;
    }
    if (threadIdx.x == kSelChunk - 1) {
        gs->n_next = pa[kSelChunk - 1];
        gs->n_regrow = pb[kSelChunk - 1];
    }
}

__global__ void __launch_bounds__(kSelChunk) k_sel_write(const GraphState *gs, const int *__restrict__ todo,
                                                         const unsigned char *__restrict__ fa,
                                                         const unsigned char *__restrict__ fb,
                                                         const int *__restrict__ ca, const int *__restrict__ cb,
                                                         int *next, int *grow)
{
    __shared__ int sa[32], sb[32];
    if (gs->fail) return;
    const int n = gs->n_todo, chunks = (n + kSelChunk - 1) / kSelChunk;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    for (int ch = blockIdx.x; ch < chunks; ch += gridDim.x) {
        const int i = ch * kSelChunk + threadIdx.x;
        const bool a = (i < n) && fa[i], b = (i < n) && fb[i];
        const unsigned ma = __ballot_sync(0xffffffffu, a), mb = __ballot_sync(0xffffffffu, b);
        if (lane == 0) { sa[w] = __popc(ma); sb[w] = __popc(mb); }
        __syncthreads();
        if (w == 0) {  // exclusive scan of the 32 warp counts
            int x = sa[lane], y = sb[lane];
            for (int o = 1; o < 32; o <<= 1) {
                const int px = __shfl_up_sync(0xffffffffu, x, o), py = __shfl_up_sync(0xffffffffu, y, o);
                if (lane >= o) { x += px; y += py; }
            }
            sa[lane] = x - sa[lane];
            sb[lane] = y - sb[lane];
        }
        __syncthreads();
        const unsigned below = (1u << lane) - 1u;
        if (a) next[ca[ch] + sa[w] + __popc(ma & below)] = todo[i];
        if (b) grow[cb[ch] + sb[w] + __popc(mb & below)] = todo[i];
        __syncthreads();
    }
}

// end of an iteration: the targets still iterating (selected in order into
// `next`) become the list, the next iteration's counts are set, and whether it
// runs (thread 0 of block 0; the others copy)
__global__ void k_g_next(GraphState *gs, const int *__restrict__ next, int *todo, cudaGraphConditionalHandle loop)
{
    const int m = gs->fail ? 0 : gs->n_next;
    for (int a = blockIdx.x * blockDim.x + threadIdx.x; a < m; a += gridDim.x * blockDim.x) todo[a] = next[a];
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        GraphState &g = *gs;
        g.n_todo = m;
        g.n_grow = g.fail ? 0 : g.n_regrow;
        g.iter++;
        g.todo_left = g.n_todo;
        cudaGraphSetConditional(loop, (!g.fail && g.n_todo > 0 && g.iter < kMaxIter) ? 1u : 0u);
    }
}

// after the loop: the symmetric rows follow only if every target converged
__global__ void k_g_if_converged(const GraphState *gs, cudaGraphConditionalHandle h)
{
    cudaGraphSetConditional(h, (!gs->fail && gs->todo_left == 0) ? 1u : 0u);
}

// the symmetric rows' total against their buffers and the pair-flux buffer
__global__ void k_g_sym_check(GraphState *gs, const long long *total, long long cap, cudaGraphConditionalHandle h)
{
    const long long t = *total;
    gs->sym_total = t;
    const bool ok = t <= cap;
    if (!ok) gs->fail |= kGraphFailSym;
    cudaGraphSetConditional(h, ok ? 1u : 0u);
}

// a restage captured into the graph: a tree that would overflow its nodes stops the pass
__global__ void k_g_tree_check(const TreeBuild *tb, GraphState *gs)
{
    if (tb->fail) gs->fail |= kGraphFailTree;
}

int density_caps(const gz_context *c, int *cap0, int *cap1)
{
    const double fs[2] = {kDensityBufferFirst, kDensityBuffer};
    int *out[2] = {cap0, cap1};
    for (int k = 0; k < 2; k++) {
        const double f = fs[k];
        *out[k] = std::max(32, std::min(4096, 32 * (int)std::ceil(c->row_slots * c->prm.des_num_ngb * f * f * f / 32.0)));
    }
    return 0;
}

// Room the graph works in: the plain pass's buffers at their sizes after a
// plain pass, the row buffers with a margin. Symmetric rows, pair fluxes and
// the refine queue take the last pass's count plus a quarter. Returns kNoRoom
// (no error recorded) when the device has no room for them: the pass then
// runs plain.
constexpr int kNoRoom = -1;
int graph_buffers(gz_context *c, long long *sym_cap, long long *rq_cap, bool with_restage)
{
    const int n = c->n;
    const size_t N = (size_t)std::max(n, 1);
    int cap0 = 0, cap1 = 0;
    density_caps(c, &cap0, &cap1);
    const long long nbr_need = (long long)n * cap0 + std::max<long long>(n / 8, 4096) * cap1;
    if (nbr_need > (long long)INT32_MAX * 4) return kNoRoom;
    const long long sc = c->pairs_symmetric + c->pairs_symmetric / 4 + 1024;
    const int mixed = c->prm.precision == GZ_PRECISION_MIXED;
    const long long rq = mixed ? std::max(65536ll, sc / 8) : 0;
    if (ensure(c, c->targets, sizeof(int) * N) || ensure(c, c->todo_a, sizeof(int) * N) ||
        ensure(c, c->todo_b, sizeof(int) * N) || ensure(c, c->grow, sizeof(int) * N) ||
        ensure(c, c->counts, sizeof(long long) * N) || ensure(c, c->hmax, sizeof(unsigned long long)) ||
        ensure(c, c->gstate, sizeof(GraphState)) || ensure(c, c->g_hseed, sizeof(double) * N) ||
        ensure(c, c->g_cseed, sizeof(double) * N) || ensure(c, c->g_over_list, sizeof(int) * N) ||
        ensure(c, c->g_over_off, sizeof(long long) * N) || ensure(c, c->s_acnt, sizeof(int) * N) ||
        ensure(c, c->s_bcnt, sizeof(int) * N) || ensure(c, c->s_counts, sizeof(long long) * N) ||
        ensure(c, c->s_off, sizeof(long long) * (N + 1)) || ensure(c, c->refined, sizeof(unsigned long long)) ||
        ensure(c, c->keep, N) || ensure(c, c->regrow, N) ||
        ensure(c, c->g_sel, sizeof(int) * 2 * (N / kSelChunk + 1)))
        return c->err;
    // the large buffers: without room for them the pass runs plain (which
    // allocates what it needs again)
    if (c->d_nbr_cap < nbr_need || !c->d_nbr.p) {
        if (!try_ensure(c->d_nbr, sizeof(int) * (size_t)nbr_need)) { c->d_nbr_cap = 0; return kNoRoom; }
        c->d_nbr_cap = nbr_need;
    }
    if (!try_ensure(c->s_tmp, sizeof(int) * (size_t)sc)) return kNoRoom;
    if ((long long)(c->s_nbr.bytes / sizeof(int)) < sc || !c->s_nbr.p) {
        if (!try_ensure(c->s_nbr, sizeof(int) * (size_t)sc)) { c->s_nbr_cap = 0; return kNoRoom; }
        c->s_nbr_cap = (long long)(c->s_nbr.bytes / sizeof(int));
    }
    if (!try_ensure(c->pflux, pair_flux_bytes(mixed) * (size_t)sc)) return kNoRoom;
    if (mixed && !try_ensure(c->rq, sizeof(RefineItem) * (size_t)rq)) return kNoRoom;
    size_t tmp = 0, tmp_sort = 0;
    cub::DeviceScan::InclusiveSum(nullptr, tmp, ptr<long long>(c->s_counts), ptr<long long>(c->s_off) + 1, n,
                                  c->stream);
    if (with_restage) {  // the restage's key sort and octree, sized before the capture
        cub::DeviceRadixSort::SortPairs(nullptr, tmp_sort, ptr<unsigned long long>(c->keys),
                                        ptr<unsigned long long>(c->keys_sorted), ptr<int>(c->idx), ptr<int>(c->perm), n,
                                        0, 63, c->stream);
        const size_t cap = (size_t)tree_cap(c);
        if (ensure(c, c->t_node, sizeof(int4) * cap) || ensure(c, c->t_parent, sizeof(int) * cap) ||
            ensure(c, c->t_lo, sizeof(double4) * cap) || ensure(c, c->t_hi, sizeof(double4) * cap) ||
            ensure(c, c->t_done, sizeof(int) * cap) || ensure(c, c->t_build, sizeof(TreeBuild)))
            return c->err;
    }
    if (ensure(c, c->cub_tmp, std::max(tmp, tmp_sort))) return c->err;
    *sym_cap = std::min<long long>({sc, (long long)(c->s_nbr.bytes / sizeof(int)), (long long)(c->s_tmp.bytes / sizeof(int)),
                                    (long long)(c->pflux.bytes / pair_flux_bytes(mixed))});
    *rq_cap = rq;
    return 0;
}

// what a captured graph depends on: every buffer's address and size, the
// particle count, the pass settings
std::vector<unsigned long long> graph_signature(gz_context *c, bool with_restage)
{
    // the pipelined copies of the inputs and the download staging are never
    // read by the graph; the resident inputs only by a restage in it (the
    // pipelined upload swaps them every step when the restage is outside)
    const DevBuf *outside[] = {&c->p_stage3, &c->p_vel, &c->p_mass, &c->p_u, &c->p_dt, &c->p_h, &c->p_cond,
                               &c->dstage, &c->dl};
    const DevBuf *inputs[] = {&c->stage3, &c->o_vel, &c->o_mass, &c->o_u, &c->o_dt, &c->o_h, &c->o_cond};
    std::vector<unsigned long long> v;
    v.push_back(with_restage ? 1 : 0);
    for (DevBuf *b : all_buffers(c)) {
        if (std::find(std::begin(outside), std::end(outside), b) != std::end(outside)) continue;
        if (!with_restage && std::find(std::begin(inputs), std::end(inputs), b) != std::end(inputs)) continue;
        v.push_back((unsigned long long)(uintptr_t)b->p);
        v.push_back(b->bytes);
    }
    v.push_back((unsigned long long)c->n);
    const unsigned char *pp = (const unsigned char *)&c->pp;
    for (size_t k = 0; k < sizeof(PassParams); k++) v.push_back(pp[k]);
    v.push_back((unsigned long long)c->prm.precision);
    v.push_back((unsigned long long)(c->row_slots * 1024));
    v.push_back((unsigned long long)(c->have_bins ? 1 : 0) | (c->binact_on ? 2 : 0));
    v.push_back((unsigned long long)c->d_nbr_cap);
    v.push_back((unsigned long long)c->s_nbr_cap);
    v.push_back((unsigned long long)c->sms);
    return v;
}

void graph_release(gz_context *c)
{
    if (c->g.exec) cudaGraphExecDestroy(c->g.exec);
    if (c->g.graph) cudaGraphDestroy(c->g.graph);
    c->g.exec = nullptr;
    c->g.graph = nullptr;
    c->g.sig.clear();
}

// the runtime's last error, recorded against `where`
int check_last(gz_context *c, const char *where)
{
    const cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) return 0;
    char b[200];
    snprintf(b, sizeof(b), "captured pass, %s: %s", where, cudaGetErrorString(e));
    return fail(c, GZ_ERR_CUDA, b);
}

// A conditional handle of the graph being captured on `s` (reset to
// `default_value` at every launch of the graph).
int make_handle(gz_context *c, cudaStream_t s, cudaGraphConditionalHandle *h, unsigned int default_value)
{
    cudaStreamCaptureStatus st;
    cudaGraph_t g = nullptr;
    GZ_CUDA(c, cudaStreamGetCaptureInfo(s, &st, nullptr, &g, nullptr, nullptr));
    if (st != cudaStreamCaptureStatusActive) return fail(c, GZ_ERR_CUDA, "captured pass: stream not capturing");
    GZ_CUDA(c, cudaGraphConditionalHandleCreate(h, g, default_value, cudaGraphCondAssignDefault));
    return 0;
}

// A conditional node after the work captured so far on `s`; the stream's
// later work depends on it. Returns its body graph.
int add_conditional(gz_context *c, cudaStream_t s, cudaGraphConditionalHandle h, cudaGraphConditionalNodeType type,
                    cudaGraph_t *body)
{
    cudaStreamCaptureStatus st;
    cudaGraph_t g = nullptr;
    const cudaGraphNode_t *deps = nullptr;
    size_t nd = 0;
    GZ_CUDA(c, cudaStreamGetCaptureInfo(s, &st, nullptr, &g, &deps, &nd));
    if (st != cudaStreamCaptureStatusActive) return fail(c, GZ_ERR_CUDA, "captured pass: stream not capturing");
    cudaGraphNodeParams cp{};
    cp.type = cudaGraphNodeTypeConditional;
    cp.conditional.handle = h;
    cp.conditional.type = type;
    cp.conditional.size = 1;
    cudaGraphNode_t node;
    GZ_CUDA(c, cudaGraphAddNode(&node, g, deps, nd, &cp));
    *body = cp.conditional.phGraph_out[0];
    GZ_CUDA(c, cudaStreamUpdateCaptureDependencies(s, &node, 1, cudaStreamSetCaptureDependencies));
    return 0;
}

// The work of the three bodies, captured on `s` (a body stream).
int capture_density_iteration(gz_context *c, cudaStream_t s, cudaGraphConditionalHandle loop)
{
    const int n = c->n;
    int cap0 = 0, cap1 = 0;
    density_caps(c, &cap0, &cap1);
    GraphState *gs = ptr<GraphState>(c->gstate);
    Particles ps = view(c);
    Tree t = tree_view(c);
    const int blocks = c->sms * 8;
    k_g_prep<<<1, 1, 0, s>>>(gs, cap0, cap1, c->d_nbr_cap, n, walk_group_warps(), c->sms);
    k_g_row_radius<<<blocks, 256, 0, s>>>(gs, ptr<int>(c->targets), ptr<int>(c->grow), ptr<double>(c->h),
                                          kDensityBufferFirst, kDensityBuffer, ptr<double>(c->h_built));
    walk_rows_graph(t, ptr<double>(c->x), ptr<double>(c->y), ptr<double>(c->z), ptr<double>(c->h_built),
                    ptr<int>(c->targets), ptr<int>(c->grow), gs, ptr<long long>(c->counts), ptr<int>(c->d_nbr),
                    ptr<DevStatus>(c->status), s);
    k_g_padded_rows<<<blocks, 256, 0, s>>>(gs, ptr<int>(c->targets), ptr<int>(c->grow), ptr<long long>(c->counts),
                                           ptr<long long>(c->d_beg), ptr<long long>(c->d_end), ptr<int>(c->g_over_list),
                                           ptr<long long>(c->g_over_off));
    k_g_over_check<<<1, 1, 0, s>>>(gs, c->d_nbr_cap);
    walk_over_graph(t, ptr<double>(c->x), ptr<double>(c->y), ptr<double>(c->z), ptr<double>(c->h_built),
                    ptr<int>(c->g_over_list), ptr<long long>(c->g_over_off), gs, ptr<int>(c->d_nbr),
                    ptr<DevStatus>(c->status), c->sms * 4, s);
    DensityWork w{};
    w.beg = ptr<long long>(c->d_beg);
    w.end = ptr<long long>(c->d_end);
    w.nbr = ptr<int>(c->d_nbr);
    w.rec = ptr<DensRec>(c->rec);
    w.acc = ptr<double>(c->acc);
    w.h_built = ptr<double>(c->h_built);
    w.scratch = ptr<DensityScratch>(c->scratch);
    w.h_iter_max = ptr<unsigned long long>(c->hmax);
    w.keep = ptr<unsigned char>(c->keep);
    w.regrow = ptr<unsigned char>(c->regrow);
    density_sums_graph(c->pp, ps, w, gs, ptr<int>(c->todo_a), c->sms * 6, s);
    density_after_iter_graph(c->pp, ps, w, ptr<DevStatus>(c->status), gs, ptr<int>(c->todo_a), c->sms * 16, s);
    int *ca = ptr<int>(c->g_sel), *cb = ca + (n + kSelChunk - 1) / kSelChunk;
    k_sel_count<<<c->sms * 2, kSelChunk, 0, s>>>(gs, ptr<unsigned char>(c->keep), ptr<unsigned char>(c->regrow), ca, cb);
    k_sel_scan<<<1, kSelChunk, 0, s>>>(gs, ca, cb);
    k_sel_write<<<c->sms * 2, kSelChunk, 0, s>>>(gs, ptr<int>(c->todo_a), ptr<unsigned char>(c->keep),
                                                 ptr<unsigned char>(c->regrow), ca, cb, ptr<int>(c->todo_b),
                                                 ptr<int>(c->grow));
    k_g_next<<<c->sms * 4, 256, 0, s>>>(gs, ptr<int>(c->todo_b), ptr<int>(c->todo_a), loop);
    GZ_CUDA(c, cudaGetLastError());
    return 0;
}

// The symmetric rows' counts and offsets, then (if they fit) the body that
// builds them and runs gradients and force, returned in *body_gf.
int capture_sym_rows(gz_context *c, cudaStream_t s, long long sym_cap, cudaGraph_t *body_gf)
{
    const int n = c->n;
    const size_t N = (size_t)std::max(n, 1);
    GZ_CUDA(c, cudaMemsetAsync(c->s_bcnt.p, 0, sizeof(int) * N, s));
    sym_split(n, ptr<double>(c->x), ptr<double>(c->y), ptr<double>(c->z), ptr<double>(c->h), c->prm.box_size,
              ptr<long long>(c->d_beg), ptr<long long>(c->d_end), ptr<int>(c->d_nbr), ptr<int>(c->s_acnt),
              ptr<int>(c->s_bcnt), s);
    sym_counts(n, ptr<int>(c->s_acnt), ptr<int>(c->s_bcnt), ptr<long long>(c->s_counts), s);
    GZ_CUDA(c, cudaMemsetAsync(c->s_off.p, 0, sizeof(long long), s));
    size_t tmp = c->cub_tmp.bytes;
    cub::DeviceScan::InclusiveSum(c->cub_tmp.p, tmp, ptr<long long>(c->s_counts), ptr<long long>(c->s_off) + 1, n, s);
    GZ_CUDA(c, cudaGetLastError());
    cudaGraphConditionalHandle h;
    if (make_handle(c, s, &h, 0)) return c->err;
    k_g_sym_check<<<1, 1, 0, s>>>(ptr<GraphState>(c->gstate), ptr<long long>(c->s_off) + n, sym_cap, h);
    GZ_CUDA(c, cudaGetLastError());
    return add_conditional(c, s, h, cudaGraphCondTypeIf, body_gf);
}

int capture_gradients_force(gz_context *c, cudaStream_t s, long long rq_cap)
{
    const int n = c->n;
    const size_t N = (size_t)std::max(n, 1);
    GZ_CUDA(c, cudaMemsetAsync(c->s_bcnt.p, 0, sizeof(int) * N, s));  // reused as the B cursors
    sym_scatter(n, ptr<long long>(c->d_beg), ptr<int>(c->d_nbr), ptr<int>(c->s_acnt), ptr<long long>(c->s_off),
                ptr<int>(c->s_bcnt), ptr<int>(c->s_tmp), s);
    sym_sort(n, ptr<long long>(c->s_off), ptr<int>(c->s_acnt), ptr<int>(c->s_tmp), ptr<int>(c->s_nbr), s);
    Csr rows{ptr<long long>(c->s_off), ptr<int>(c->s_nbr)};
    Particles ps = view(c);
    gradients_fp64(c->pp, ps, ptr<int>(c->targets), n, rows, lanes_per_row(c, n, 1), c->rec.p, nullptr, s);
    if (c->have_bins) GZ_CUDA(c, cudaMemsetAsync(c->wakeup.p, 0, sizeof(int) * N, s));
    force_preloop(c->pp, ps, ptr<int>(c->targets), n, s);
    if (c->prm.precision == GZ_PRECISION_MIXED) {
        GZ_CUDA(c, cudaMemsetAsync(c->refined.p, 0, sizeof(unsigned long long), s));
        const RefineQueue q{ptr<RefineItem>(c->rq), ptr<unsigned long long>(c->refined), rq_cap};
        force_mixed(c->pp, ps, ptr<int>(c->targets), n, rows, c->tpt_force, ptr<DevStatus>(c->status), c->rec.p,
                    c->pflux.p, true, q, ptr<double>(c->acc), nullptr, s);
    } else {
        force_fp64(c->pp, ps, ptr<int>(c->targets), n, rows, c->tpt_force, ptr<DevStatus>(c->status), c->rec.p,
                   c->pflux.p, true, ptr<double>(c->acc), nullptr, s);
    }
    GZ_CUDA(c, cudaGetLastError());
    return 0;
}

// Captures the pass into c->g (graph_buffers has sized everything it uses).
int graph_capture(gz_context *c, long long sym_cap, long long rq_cap, bool with_restage)
{
    graph_release(c);
    for (auto &b : c->g.body)
        if (!b) GZ_CUDA(c, cudaStreamCreateWithFlags(&b, cudaStreamNonBlocking));
    const int n = c->n;
    const size_t N = (size_t)n;
    cudaStream_t s = c->stream;
    cudaStream_t s1 = c->g.body[0], s2 = c->g.body[1];
    Particles ps = view(c);
    walk_group_warps();  // its occupancy query runs before the capture
    GZ_CUDA(c, cudaGetLastError());
    const long long launches0 = c->launches;
    cudaGraph_t body_loop = nullptr, body_sym = nullptr, body_gf = nullptr;
    cudaGraphConditionalHandle h_loop, h_conv;
    int rc = 0;
    cudaGraph_t g = nullptr;
    GZ_CUDA(c, cudaStreamBeginCapture(s, cudaStreamCaptureModeRelaxed));
    c->g.capturing = true;
    // the bodies are captured on their own streams into the nodes' graphs
    auto body = [&](cudaStream_t bs, cudaGraph_t bg, auto &&fill) -> int {
        if (cudaStreamBeginCaptureToGraph(bs, bg, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed) != cudaSuccess)
            return fail(c, GZ_ERR_CUDA, "captured pass: cannot capture a body");
        const int r = fill();
        cudaGraph_t out = bg;
        const cudaError_t e = cudaStreamEndCapture(bs, &out);
        if (r) return r;
        if (e != cudaSuccess) return fail(c, GZ_ERR_CUDA, cudaGetErrorString(e));
        return 0;
    };
    long long restage_kernels = 0;
    do {
        k_g_init<<<1, 1, 0, s>>>(ptr<GraphState>(c->gstate), n);
        if (with_restage) {  // the restage first, its tree with nothing read back
            const long long l0 = c->launches;
            if ((rc = enqueue_restage(c, true))) break;
            k_g_tree_check<<<1, 1, 0, s>>>(ptr<TreeBuild>(c->t_build), ptr<GraphState>(c->gstate));
            restage_kernels = c->launches - l0 + 1 + 2 * 22 + 1 + 1;  // + tree build, bottom-up pass, check
            if ((rc = check_last(c, "restage"))) break;
        }
        // the inputs a plain pass would restart from
        cudaMemcpyAsync(c->g_hseed.p, c->h.p, sizeof(double) * N, cudaMemcpyDeviceToDevice, s);
        cudaMemcpyAsync(c->g_cseed.p, c->cond.p, sizeof(double) * N, cudaMemcpyDeviceToDevice, s);
        int na = 0;
        if ((rc = sort_targets(c, nullptr, 0, &na))) break;
        cudaMemsetAsync(c->hmax.p, 0, sizeof(unsigned long long), s);
        k_density_prep<<<(n + 255) / 256, 256, 0, s>>>(n, ptr<int>(c->targets), ptr<double>(c->h),
                                                       c->prm.max_kernel_radius, ptr<DensityScratch>(c->scratch),
                                                       ptr<unsigned long long>(c->hmax));
        cudaMemcpyAsync(c->todo_a.p, c->targets.p, sizeof(int) * N, cudaMemcpyDeviceToDevice, s);
        density_pack(ps, ptr<DensRec>(c->rec), s);
        if ((rc = check_last(c, "density setup"))) break;
        if ((rc = make_handle(c, s, &h_loop, 1))) break;
        if ((rc = add_conditional(c, s, h_loop, cudaGraphCondTypeWhile, &body_loop))) break;
        if ((rc = body(s1, body_loop, [&] { return capture_density_iteration(c, s1, h_loop); }))) break;
        if ((rc = check_last(c, "density iteration"))) break;
        density_finalize(c->pp, ps, ptr<double>(c->acc), ptr<int>(c->targets), n, s);
        if ((rc = make_handle(c, s, &h_conv, 0))) break;
        k_g_if_converged<<<1, 1, 0, s>>>(ptr<GraphState>(c->gstate), h_conv);
        if ((rc = add_conditional(c, s, h_conv, cudaGraphCondTypeIf, &body_sym))) break;
        rc = body(s1, body_sym, [&] {
            int r = capture_sym_rows(c, s1, sym_cap, &body_gf);
            if (!r) r = check_last(c, "symmetric rows");
            if (r) return r;
            r = body(s2, body_gf, [&] { return capture_gradients_force(c, s2, rq_cap); });
            if (!r) r = check_last(c, "gradients and force");
            return r;
        });
        if (rc) break;
        if (cudaGetLastError() != cudaSuccess) { rc = fail(c, GZ_ERR_CUDA, "captured pass: a launch failed"); break; }
    } while (0);
    const cudaError_t e = cudaStreamEndCapture(s, &g);
    c->g.capturing = false;
    c->launches = launches0;
    if (!rc && e != cudaSuccess) rc = fail(c, GZ_ERR_CUDA, cudaGetErrorString(e));
    if (rc) {
        if (g) cudaGraphDestroy(g);
        cudaGetLastError();
        return rc;
    }
    c->g.graph = g;
    if (check_last(c, "end of capture")) { graph_release(c); return c->err; }
    // this library's kernels in each part (the key sort and scans are CUB's):
    // setup (targets, active flags, prep, pack, state) + finalize + the
    // convergence test; per iteration prep, radii, two walk modes, padded
    // rows, overflow check, overflow walk, three sums instances, after_iter,
    // the selection's three steps, next; the rows' split, counts and check;
    // scatter, sort, the gradient pack and rows, the force preloop, pack,
    // pairs, (refine,) gather, finish
    c->g.kernels_top = 7 + restage_kernels;
    c->g.kernels_loop = 15;
    c->g.kernels_sym = 3;
    c->g.kernels_tail = c->prm.precision == GZ_PRECISION_MIXED ? 10 : 9;
    const cudaError_t ie = cudaGraphInstantiate(&c->g.exec, g, 0);
    if (ie != cudaSuccess) {
        char b[200];
        snprintf(b, sizeof(b), "captured pass: cannot instantiate the graph: %s", cudaGetErrorString(ie));
        cudaGetLastError();
        graph_release(c);
        return fail(c, GZ_ERR_CUDA, b);
    }
    if (check_last(c, "instantiation")) { graph_release(c); return c->err; }
    c->g.rq_cap = rq_cap;
    c->g.with_restage = with_restage;
    c->g.captures++;
    return 0;
}

// One replay of the captured pass; a buffer overflow (or more fragile pairs
// than the refine queue holds) is answered by the plain pass from the
// graph's starting kernel lengths and condition numbers.
int graph_pass(gz_context *c, bool with_restage)
{
    cudaStream_t s = c->stream;
    const int n = c->n;
    auto plain = [&]() -> int {
        int rc = with_restage ? gz_restage(c) : 0;
        if (!rc) rc = gz_hydro_density(c, nullptr, 0);
        if (!rc) rc = gz_hydro_gradients(c, nullptr, 0);
        if (!rc) rc = gz_hydro_force(c, nullptr, 0);
        return rc;
    };
    long long sym_cap = 0, rq_cap = 0;
    const int room = graph_buffers(c, &sym_cap, &rq_cap, with_restage);
    if (room == kNoRoom) return plain();  // no room for the graph's buffers
    if (room) return room;
    if (with_restage) {
        // the graph reads the resident inputs at their addresses: inputs of a
        // pipelined upload are copied into them rather than swapped in
        if (take_pending_inputs(c, true)) return c->err;
        c->fabs_valid = false;
        c->err = 0;
        c->err_index = -1;
        c->msg[0] = 0;
    }
    std::vector<unsigned long long> sig = graph_signature(c, with_restage);
    if (!c->g.exec || sig != c->g.sig) {
        if (graph_capture(c, sym_cap, rq_cap, with_restage)) return c->err;
        c->g.sig = sig;
    }
    if (check_last(c, "before the launch")) return c->err;
    GZ_CUDA(c, cudaGraphLaunch(c->g.exec, s));
    GraphState gs{};
    TreeBuild tb{};
    unsigned long long refined = 0, hbits = 0;
    const int mixed = c->prm.precision == GZ_PRECISION_MIXED;
    GZ_CUDA(c, cudaMemcpyAsync(&gs, c->gstate.p, sizeof(gs), cudaMemcpyDeviceToHost, s));
    GZ_CUDA(c, cudaMemcpyAsync(&hbits, c->hmax.p, sizeof(hbits), cudaMemcpyDeviceToHost, s));
    if (mixed) GZ_CUDA(c, cudaMemcpyAsync(&refined, c->refined.p, sizeof(refined), cudaMemcpyDeviceToHost, s));
    if (with_restage) GZ_CUDA(c, cudaMemcpyAsync(&tb, c->t_build.p, sizeof(tb), cudaMemcpyDeviceToHost, s));
    GZ_CUDA(c, cudaStreamSynchronize(s));
    if (check_last(c, "graph launch")) return c->err;
    c->g.replays++;
    if (with_restage) {
        c->t_nodes = tb.total;
        c->t_levels = tb.L;
        c->grid_valid = true;
        c->have_density = c->have_gradients = false;
        c->sym_valid = false;
        c->dens_all = false;
    }
    const bool converged = gs.todo_left == 0 && !gs.fail;
    c->launches += c->g.kernels_top + c->g.kernels_loop * gs.iter + (converged ? c->g.kernels_sym : 0) +
                   ((converged && !(gs.fail & kGraphFailSym)) ? c->g.kernels_tail : 0);
    if (gs.fail || (long long)refined > c->g.rq_cap) {
        c->g.fallbacks++;
        if (with_restage) return plain();  // the restage starts again from the resident inputs
        GZ_CUDA(c, cudaMemcpyAsync(c->h.p, c->g_hseed.p, sizeof(double) * (size_t)n, cudaMemcpyDeviceToDevice, s));
        GZ_CUDA(c, cudaMemcpyAsync(c->cond.p, c->g_cseed.p, sizeof(double) * (size_t)n, cudaMemcpyDeviceToDevice, s));
        return plain();
    }
    c->last_iters = gs.iter;
    c->d_used = gs.base;
    memcpy(&c->h_iter_max, &hbits, sizeof(double));
    c->pairs_density = gs.entries;
    if (read_status(c)) return c->err;
    if (gs.todo_left > 0) return fail(c, GZ_ERR_DENSITY_MAXITER, "density did not converge in MAXITER iterations");
    c->have_density = true;
    c->dens_all = false;  // the symmetric rows consumed the density rows
    c->pairs_symmetric = gs.sym_total;
    c->sym_rows = n;
    c->sym_valid = true;
    c->sym_all = true;
    c->sym_active.clear();
    c->have_gradients = true;
    c->fabs_valid = c->pp.diag_flux_abs != 0;
    c->pairs_refined = (long long)refined;
    return GZ_OK;
}

}  // namespace

// ===================================================================== ABI
extern "C" {

int gz_create(const gz_params *params, int device, gz_context **out)
{
    if (!out) return GZ_ERR_ARG;
    *out = nullptr;
    if (check_params(params)) return GZ_ERR_ARG;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= 0) return GZ_ERR_NO_DEVICE;
    if (device < 0 || device >= ndev) return GZ_ERR_ARG;
    if (cudaSetDevice(device) != cudaSuccess) return GZ_ERR_CUDA;
    gz_context *c = new (std::nothrow) gz_context();
    if (!c) return GZ_ERR_CAPACITY;
    c->prm = *params;
    c->pp = make_pass_params(*params);
    c->device = device;
    int sms = 0;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device) == cudaSuccess && sms > 0) c->sms = sms;
    if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess) { delete c; return GZ_ERR_CUDA; }
    if (ensure(c, c->status, sizeof(DevStatus))) { cudaStreamDestroy(c->stream); delete c; return GZ_ERR_CUDA; }
    cudaMemsetAsync(c->status.p, 0, sizeof(DevStatus), c->stream);
    *out = c;
    return GZ_OK;
}

int gz_destroy(gz_context *c)
{
    if (!c) return GZ_ERR_ARG;
    cudaSetDevice(c->device);
    cudaStreamSynchronize(c->stream);
    graph_release(c);
    for (auto &b : c->g.body)
        if (b) cudaStreamDestroy(b);
    if (c->cstream) {
        cudaStreamSynchronize(c->cstream);
        cudaStreamDestroy(c->cstream);
        for (cudaEvent_t e : {c->ev_in_free, c->ev_in_done, c->ev_out_ready, c->ev_out_done}) cudaEventDestroy(e);
    }
    for (DevBuf *b : all_buffers(c)) release(*b);
    for (auto &t : c->timers)
        for (auto &e : t.ev) { cudaEventDestroy(e.start); cudaEventDestroy(e.stop); }
    cudaStreamDestroy(c->stream);
    delete c;
    return GZ_OK;
}

int gz_set_params(gz_context *c, const gz_params *params)
{
    if (!c || check_params(params)) return GZ_ERR_ARG;
    const bool box_changed = params->box_size != c->prm.box_size;
    c->prm = *params;
    c->pp = make_pass_params(*params);
    c->pp.diag_flux_abs = (c->diag & GZ_DIAG_FLUX_ABS) != 0;
    if (box_changed) c->grid_valid = false;
    return GZ_OK;
}

int gz_set_diagnostics(gz_context *c, int flags)
{
    if (!c || (flags & ~GZ_DIAG_FLUX_ABS)) return GZ_ERR_ARG;
    c->diag = flags;
    c->pp.diag_flux_abs = (flags & GZ_DIAG_FLUX_ABS) != 0;
    return GZ_OK;
}

void *gz_stream(gz_context *c) { return c ? (void *)c->stream : nullptr; }

int gz_kernel_timing(gz_context *c, int enable)
{
    if (!c) return GZ_ERR_ARG;
    c->timing = enable != 0;
    for (auto &t : c->timers) { t.used = 0; t.units = 0; }
    return GZ_OK;
}

int gz_kernel_time(gz_context *c, int timer, double *ms, int64_t *launches, int64_t *units)
{
    if (!c || timer < 0 || timer >= GZ_TIMERS) return GZ_ERR_ARG;
    cudaSetDevice(c->device);
    GZ_CUDA(c, cudaStreamSynchronize(c->stream));
    gz_context::Timer &t = c->timers[timer];
    double total = 0;
    for (size_t k = 0; k < t.used; k++) {
        float m = 0;
        GZ_CUDA(c, cudaEventElapsedTime(&m, t.ev[k].start, t.ev[k].stop));
        total += m;
    }
    if (ms) *ms = total;
    if (launches) *launches = (int64_t)t.used;
    if (units) *units = t.units;
    t.used = 0;
    t.units = 0;
    return GZ_OK;
}

// Rebuild the sorted mirror and the octree from the resident inputs (the
// state a pass starts from): Morton keys, radix sort, gathers, zeroed
// outputs, tree.
static int stage_inputs(gz_context *c)
{
    c->fabs_valid = false;
    c->err = 0;
    c->err_index = -1;
    c->msg[0] = 0;
    if (enqueue_restage(c, false)) return c->err;
    c->grid_valid = true;
    c->have_density = c->have_gradients = false;
    c->sym_valid = false;
    c->dens_all = false;
    return 0;
}

// gz_upload from host arrays (kind = kind) or from the
// caller's device arrays (cudaMemcpyDeviceToDevice, gz_upload_device).
static int upload_from(gz_context *c, const gz_particles *in, cudaMemcpyKind kind)
{
    if (!c || !in || in->n < 0 || in->n > INT32_MAX / 16) return GZ_ERR_ARG;
    if (in->n > 0 && (!in->pos || !in->vel || !in->mass || !in->u || !in->dt || !in->h)) return GZ_ERR_ARG;
    cudaSetDevice(c->device);
    c->in_pending = false;  // a pipelined upload not yet restaged is superseded
    const int n = (int)in->n;
    c->n = n;
    cudaStream_t s = c->stream;
    const size_t N = (size_t)std::max(n, 1);
    DevBuf *one[] = {&c->x, &c->y, &c->z, &c->vx, &c->vy, &c->vz, &c->m, &c->u, &c->dt, &c->h, &c->cond, &c->num_ngb,
                     &c->drkern, &c->divvel, &c->rho, &c->pressure, &c->fce, &c->dudt, &c->vsig, &c->dtmass,
                     &c->dmass, &c->h_built, &c->o_mass, &c->o_u, &c->o_dt, &c->o_h, &c->o_cond, &c->dl};
    for (DevBuf *b : one)
        if (ensure(c, *b, sizeof(double) * N)) return c->err;
    if (ensure(c, c->nvt, sizeof(double) * 6 * N) || ensure(c, c->pv, sizeof(double) * 3 * N) ||
        ensure(c, c->grad, sizeof(double) * 15 * N) || ensure(c, c->accel, sizeof(double) * 3 * N) ||
        ensure(c, c->gw, sizeof(double) * 3 * N) || ensure(c, c->fabs3, sizeof(double) * 3 * N) ||
        ensure(c, c->iters, sizeof(int) * N) ||
        ensure(c, c->active, N) || ensure(c, c->stage, sizeof(double) * 3 * N) ||
        ensure(c, c->stage3, sizeof(double) * 3 * N) || ensure(c, c->o_vel, sizeof(double) * 3 * N) ||
        ensure(c, c->perm, sizeof(int) * N) || ensure(c, c->inv, sizeof(int) * N) ||
        ensure(c, c->acc, sizeof(double) * 17 * N) || ensure(c, c->scratch, sizeof(DensityScratch) * N) ||
        ensure(c, c->d_beg, sizeof(long long) * N) || ensure(c, c->d_end, sizeof(long long) * N) ||
        ensure(c, c->rec, std::max({sizeof(DensRec), gradient_record_bytes(0), gradient_record_bytes(1),
                                    force_record_bytes(0), force_record_bytes(1)}) * N))
        return c->err;
    if (n > 0) {
        GZ_CUDA(c, cudaMemcpyAsync(c->stage3.p, in->pos, sizeof(double) * 3 * (size_t)n, kind, s));
        GZ_CUDA(c, cudaMemcpyAsync(c->o_vel.p, in->vel, sizeof(double) * 3 * (size_t)n, kind, s));
        struct { const double *src; DevBuf *dst; } f1[] = {
            {in->mass, &c->o_mass}, {in->u, &c->o_u}, {in->dt, &c->o_dt}, {in->h, &c->o_h}, {in->cond, &c->o_cond}};
        for (auto &f : f1) {
            if (f.src) GZ_CUDA(c, cudaMemcpyAsync(f.dst->p, f.src, sizeof(double) * (size_t)n, kind, s));
            else GZ_CUDA(c, cudaMemsetAsync(f.dst->p, 0, sizeof(double) * (size_t)n, s));
        }
    }
    c->have_bins = in->timebin != nullptr;
    if (c->have_bins) {
        if (ensure(c, c->o_timebin, sizeof(int) * N) || ensure(c, c->o_vsig, sizeof(double) * N) ||
            ensure(c, c->timebin, sizeof(int) * N) || ensure(c, c->vsig_prev, sizeof(double) * N) ||
            ensure(c, c->wakeup, sizeof(int) * N))
            return c->err;
        if (kind == cudaMemcpyHostToDevice)
            for (int k = 0; k < n; k++)
                if (in->timebin[k] < 0 || in->timebin[k] >= GZ_TIMEBINS)
                    return fail(c, GZ_ERR_ARG, "timebin out of range");
        if (n > 0) {
            GZ_CUDA(c, cudaMemcpyAsync(c->o_timebin.p, in->timebin, sizeof(int) * (size_t)n, kind, s));
            if (in->vsig)
                GZ_CUDA(c, cudaMemcpyAsync(c->o_vsig.p, in->vsig, sizeof(double) * (size_t)n, kind, s));
            else
                GZ_CUDA(c, cudaMemsetAsync(c->o_vsig.p, 0, sizeof(double) * (size_t)n, s));
        }
    }
    if (!c->box_counts.empty()) {
        long long total = 0;
        for (long long k : c->box_counts) total += k;
        if (total != n) return fail(c, GZ_ERR_ARG, "box counts do not add up to the particle count");
        std::vector<int> bid((size_t)std::max(n, 1));
        size_t at = 0;
        for (size_t b = 0; b < c->box_counts.size(); b++)
            for (long long k = 0; k < c->box_counts[b]; k++) bid[at++] = (int)b;
        if (ensure(c, c->box_bid, sizeof(int) * N)) return c->err;
        GZ_CUDA(c, cudaMemcpyAsync(c->box_bid.p, bid.data(), sizeof(int) * (size_t)n, cudaMemcpyHostToDevice, s));
        GZ_CUDA(c, cudaStreamSynchronize(s));  // (bid is freed on return)
    }
    if (stage_inputs(c)) return c->err;
    GZ_CUDA(c, cudaStreamSynchronize(s));
    return c->err;
}

int gz_upload(gz_context *c, const gz_particles *in) { return upload_from(c, in, cudaMemcpyHostToDevice); }

int gz_upload_device(gz_context *c, const gz_particles *in) { return upload_from(c, in, cudaMemcpyDeviceToDevice); }

int gz_restage(gz_context *c)
{
    if (!c) return GZ_ERR_ARG;
    cudaSetDevice(c->device);
    if (!c->grid_valid && c->n > 0) return fail(c, GZ_ERR_ORDER, "restage before upload");
    if (take_pending_inputs(c)) return c->err;
    if (stage_inputs(c)) return c->err;
    return GZ_OK;
}

int gz_upload_async(gz_context *c, const gz_particles *in)
{
    if (!c || !in) return GZ_ERR_ARG;
    cudaSetDevice(c->device);
    // a new size, timebins, or no set yet: the synchronous upload
    if (!c->grid_valid || in->n != c->n || in->timebin || c->n == 0) return upload_from(c, in, cudaMemcpyHostToDevice);
    if (!in->pos || !in->vel || !in->mass || !in->u || !in->dt || !in->h) return GZ_ERR_ARG;
    if (copy_stream(c)) return c->err;
    if (take_pending_inputs(c)) return c->err;  // an upload not yet restaged is taken now
    const size_t N = (size_t)c->n;
    if (ensure(c, c->p_stage3, sizeof(double) * 3 * N) || ensure(c, c->p_vel, sizeof(double) * 3 * N) ||
        ensure(c, c->p_mass, sizeof(double) * N) || ensure(c, c->p_u, sizeof(double) * N) ||
        ensure(c, c->p_dt, sizeof(double) * N) || ensure(c, c->p_h, sizeof(double) * N) ||
        ensure(c, c->p_cond, sizeof(double) * N))
        return c->err;
    // the copies wait for the work queued so far (it may read these buffers'
    // previous contents), then run beside the next pass
    GZ_CUDA(c, cudaEventRecord(c->ev_in_free, c->stream));
    GZ_CUDA(c, cudaStreamWaitEvent(c->cstream, c->ev_in_free, 0));
    const cudaMemcpyKind k = cudaMemcpyHostToDevice;
    GZ_CUDA(c, cudaMemcpyAsync(c->p_stage3.p, in->pos, sizeof(double) * 3 * N, k, c->cstream));
    GZ_CUDA(c, cudaMemcpyAsync(c->p_vel.p, in->vel, sizeof(double) * 3 * N, k, c->cstream));
    struct { const double *src; DevBuf *dst; } f1[] = {
        {in->mass, &c->p_mass}, {in->u, &c->p_u}, {in->dt, &c->p_dt}, {in->h, &c->p_h}, {in->cond, &c->p_cond}};
    for (auto &f : f1) {
        if (f.src) GZ_CUDA(c, cudaMemcpyAsync(f.dst->p, f.src, sizeof(double) * N, k, c->cstream));
        else GZ_CUDA(c, cudaMemsetAsync(f.dst->p, 0, sizeof(double) * N, c->cstream));
    }
    GZ_CUDA(c, cudaEventRecord(c->ev_in_done, c->cstream));
    c->in_pending = true;
    return GZ_OK;
}

int gz_wait(gz_context *c)
{
    if (!c) return GZ_ERR_ARG;
    cudaSetDevice(c->device);
    if (c->out_pending) {
        // the context's stream is ordered after the copies too (a caller's event
        // recorded on it then covers them)
        GZ_CUDA(c, cudaStreamWaitEvent(c->stream, c->ev_out_done, 0));
        GZ_CUDA(c, cudaEventSynchronize(c->ev_out_done));
        c->out_pending = false;
    }
    return GZ_OK;
}

int gz_hydro_density(gz_context *c, const int *active, int n_active)
{
    if (!c) return GZ_ERR_ARG;
    cudaSetDevice(c->device);
    if (!c->grid_valid) return fail(c, GZ_ERR_ORDER, "density before upload");
    c->dens_all = false;  // set again only when this pass completes over every particle
    cudaStream_t s = c->stream;
    int na = 0;
    if (sort_targets(c, active, n_active, &na)) return c->err;
    if (na == 0) {  // no target (an empty set or active list): nothing runs, no output changes
        c->last_iters = 0;
        c->h_iter_max = 0;
        c->have_density = true;
        c->sym_valid = false;
        c->dens_all = (active == nullptr);
        return GZ_OK;
    }
    Particles ps = view(c);
    const int n = c->n;
    if (ensure(c, c->todo_a, sizeof(int) * (size_t)std::max(na, 1)) ||
        ensure(c, c->todo_b, sizeof(int) * (size_t)std::max(na, 1)) ||
        ensure(c, c->grow, sizeof(int) * (size_t)std::max(na, 1)) || ensure(c, c->keep, (size_t)std::max(na, 1)) ||
        ensure(c, c->regrow, (size_t)std::max(na, 1)) || ensure(c, c->flag, sizeof(int)) ||
        ensure(c, c->n_sel, sizeof(int) * 2) || ensure(c, c->hmax, sizeof(unsigned long long)))
        return c->err;
    GZ_CUDA(c, cudaMemsetAsync(c->hmax.p, 0, sizeof(unsigned long long), s));
    if (na > 0) {
        k_density_prep<<<(na + 255) / 256, 256, 0, s>>>(na, ptr<int>(c->targets), ptr<double>(c->h),
                                                         c->prm.max_kernel_radius, ptr<DensityScratch>(c->scratch),
                                                         ptr<unsigned long long>(c->hmax));
        c->launches++;
    }
    GZ_CUDA(c, cudaMemcpyAsync(c->todo_a.p, c->targets.p, sizeof(int) * (size_t)na, cudaMemcpyDeviceToDevice, s));
    density_pack(ps, ptr<DensRec>(c->rec), s);
    c->launches++;
    int n_todo = na;
    int *todo = ptr<int>(c->todo_a), *todo_next = ptr<int>(c->todo_b);
    // Rows at the buffered radius (DensitySpec's CSR buffer factor) are built
    // for every target first; afterwards only the particles whose radius
    // outgrew their row get a new row, appended behind the others.
    const int *grow = todo;
    int n_grow = n_todo;
    long long base = 0;
    c->pairs_density = 0;
    int iter = 0;
    for (iter = 0; iter < kMaxIter && n_todo > 0; iter++) {
        if (n_grow > 0) {
            k_row_radius<<<(n_grow + 255) / 256, 256, 0, s>>>(n_grow, grow, ptr<double>(c->h),
                                                               iter == 0 ? kDensityBufferFirst : kDensityBuffer,
                                                               ptr<double>(c->h_built));
            c->launches++;
            // slots per padded row: row_slots (2.5 by default) x the expected row length, in multiples of 32
            const double f = iter == 0 ? kDensityBufferFirst : kDensityBuffer;
            const int cap = std::max(
                32, std::min(4096, 32 * (int)std::ceil(c->row_slots * c->prm.des_num_ngb * f * f * f / 32.0)));
            long long used = 0, entries = 0;
            if (build_rows_padded(c, ptr<double>(c->h_built), grow, n_grow, cap, base, &used, &entries)) return c->err;
            base = used;
            c->pairs_density += entries;
        }
        DensityWork w{};
        w.todo = todo;
        w.n_todo = n_todo;
        w.beg = ptr<long long>(c->d_beg);
        w.end = ptr<long long>(c->d_end);
        w.nbr = ptr<int>(c->d_nbr);
        w.rec = ptr<DensRec>(c->rec);
        w.acc = ptr<double>(c->acc);
        w.h_built = ptr<double>(c->h_built);
        w.scratch = ptr<DensityScratch>(c->scratch);
        w.keep = ptr<unsigned char>(c->keep);
        w.regrow = ptr<unsigned char>(c->regrow);
        w.rebuild = ptr<int>(c->flag);
        w.h_iter_max = ptr<unsigned long long>(c->hmax);
        w.iter = iter;
        GZ_CUDA(c, cudaMemsetAsync(c->flag.p, 0, sizeof(int), s));
        const EventPair *ev = timer_launch(c, GZ_TIMER_DENSITY_SUMS, w.n_todo);
        ev_start(ev, s);
        if (c->prm.precision == GZ_PRECISION_MIXED) density_sums_mixed(c->pp, ps, w, lanes_per_row(c, w.n_todo, 4), s);
        else density_sums_fp64(c->pp, ps, w, lanes_per_row(c, w.n_todo, 4), s);
        ev_stop(ev, s);
        density_after_iter(c->pp, ps, w, ptr<DevStatus>(c->status), s);
        c->launches += 2;
        GZ_CUDA(c, cudaGetLastError());
        size_t tmp = 0;
        cub::DeviceSelect::Flagged(nullptr, tmp, todo, ptr<unsigned char>(c->keep), todo_next, ptr<int>(c->n_sel), n_todo, s);
        size_t tmp2 = 0;
        cub::DeviceSelect::Flagged(nullptr, tmp2, todo, ptr<unsigned char>(c->regrow), ptr<int>(c->grow),
                                   ptr<int>(c->n_sel) + 1, n_todo, s);
        if (ensure(c, c->cub_tmp, std::max(tmp, tmp2))) return c->err;
        cub::DeviceSelect::Flagged(c->cub_tmp.p, tmp, todo, ptr<unsigned char>(c->keep), todo_next, ptr<int>(c->n_sel),
                                   n_todo, s);
        int hv[3] = {0, 0, 0};
        GZ_CUDA(c, cudaMemcpyAsync(&hv[2], c->flag.p, sizeof(int), cudaMemcpyDeviceToHost, s));
        GZ_CUDA(c, cudaMemcpyAsync(&hv[0], c->n_sel.p, sizeof(int), cudaMemcpyDeviceToHost, s));
        GZ_CUDA(c, cudaStreamSynchronize(s));
        n_grow = 0;
        if (hv[2]) {
            cub::DeviceSelect::Flagged(c->cub_tmp.p, tmp2, todo, ptr<unsigned char>(c->regrow), ptr<int>(c->grow),
                                       ptr<int>(c->n_sel) + 1, n_todo, s);
            GZ_CUDA(c, cudaMemcpyAsync(&hv[1], ptr<int>(c->n_sel) + 1, sizeof(int), cudaMemcpyDeviceToHost, s));
            GZ_CUDA(c, cudaStreamSynchronize(s));
            n_grow = hv[1];
            grow = ptr<int>(c->grow);
        }
        n_todo = hv[0];
        std::swap(todo, todo_next);
    }
    c->last_iters = iter;
    c->d_used = base;
    density_finalize(c->pp, ps, ptr<double>(c->acc), ptr<int>(c->targets), na, s);
    if (na > 0) c->launches++;
    GZ_CUDA(c, cudaGetLastError());
    (void)n;
    unsigned long long hbits = 0;
    GZ_CUDA(c, cudaMemcpyAsync(&hbits, c->hmax.p, sizeof(hbits), cudaMemcpyDeviceToHost, s));
    if (read_status(c)) return c->err;
    memcpy(&c->h_iter_max, &hbits, sizeof(double));
    if (n_todo > 0) return fail(c, GZ_ERR_DENSITY_MAXITER, "density did not converge in MAXITER iterations");
    c->have_density = true;
    c->sym_valid = false;
    c->dens_all = (active == nullptr);
    return GZ_OK;
}

int gz_hydro_gradients(gz_context *c, const int *active, int n_active)
{
    if (!c) return GZ_ERR_ARG;
    cudaSetDevice(c->device);
    if (!c->have_density) return fail(c, GZ_ERR_ORDER, "gradients before density");
    int na = 0;
    if (sort_targets(c, active, n_active, &na)) return c->err;
    if (na == 0) {  // no target: nothing runs, no output changes
        c->sym_valid = false;
        c->have_gradients = true;
        return GZ_OK;
    }
    if (build_sym_rows(c, na, active == nullptr)) return c->err;
    c->sym_all = (active == nullptr);
    c->sym_active.assign(active ? active : (const int *)nullptr, active ? active + n_active : (const int *)nullptr);
    Csr rows{ptr<long long>(c->s_off), ptr<int>(c->s_nbr)};
    Particles ps = view(c);
    const EventPair *ev = na > 0 ? timer_launch(c, GZ_TIMER_GRADIENTS, na) : nullptr;
    // Both forms take the gradient pair terms in FP64: the pass is bound by its
    // record gathers, not by arithmetic (FP32 terms saved 0.6 of 26 ms per step
    // at 256^3), and FP64 gradients make the mixed form's force inputs the FP64
    // form's exactly (FP32 terms left 9 of 16.8M particles above 1e-5).
    gradients_fp64(c->pp, ps, ptr<int>(c->targets), na, rows, lanes_per_row(c, na, 1), c->rec.p, ev, c->stream);
    if (na > 0) c->launches += 2;  // the record pack and the rows
    GZ_CUDA(c, cudaGetLastError());
    if (read_status(c)) return c->err;
    c->have_gradients = true;
    return GZ_OK;
}

int gz_hydro_force(gz_context *c, const int *active, int n_active)
{
    if (!c) return GZ_ERR_ARG;
    cudaSetDevice(c->device);
    if (!c->have_gradients) return fail(c, GZ_ERR_ORDER, "force before gradients");
    int na = 0;
    if (sort_targets(c, active, n_active, &na)) return c->err;
    if (na == 0) {  // no target: nothing runs, no output changes
        c->pairs_refined = 0;
        return GZ_OK;
    }
    // the gradient pass's symmetric rows are reused when the active set is
    // the same (the corridor list shared by both loops, hydro_corridor.cc:195-255)
    const bool same = c->sym_valid && c->sym_rows == na &&
                      ((active == nullptr && c->sym_all) ||
                       (active != nullptr && !c->sym_all && c->sym_active.size() == (size_t)n_active &&
                        std::equal(c->sym_active.begin(), c->sym_active.end(), active)));
    if (!same) {
        if (build_sym_rows(c, na, active == nullptr)) return c->err;
        c->sym_all = (active == nullptr);
        c->sym_active.assign(active ? active : (const int *)nullptr, active ? active + n_active : (const int *)nullptr);
    }
    Csr rows{ptr<long long>(c->s_off), ptr<int>(c->s_nbr)};
    Particles ps = view(c);
    if (c->have_bins && c->n > 0) GZ_CUDA(c, cudaMemsetAsync(c->wakeup.p, 0, sizeof(int) * (size_t)c->n, c->stream));
    force_preloop(c->pp, ps, ptr<int>(c->targets), na, c->stream);
    c->fabs_valid = c->pp.diag_flux_abs != 0;
    // The pairs go through a flux per row entry when that scratch can be had:
    // every particle a target -> each pair evaluated once; an active subset ->
    // each row entry. The mixed form needs it (its fragile pairs are evaluated
    // again in FP64 there); the FP64 form otherwise evaluates the rows in place.
    const int mixed = c->prm.precision == GZ_PRECISION_MIXED;
    const bool all = active == nullptr && na == c->n && c->n > 0;
    void *flux = nullptr;
    if (na > 0 && try_ensure(c->pflux, pair_flux_bytes(mixed) * (size_t)std::max(c->pairs_symmetric, 1ll)))
        flux = c->pflux.p;
    if (mixed && na > 0 && !flux) return fail(c, GZ_ERR_CAPACITY, "mixed-form force pass: no room for the pair fluxes");
    // Mixed form: queue room for one pair in 8 of the pass (about one in 700 is
    // queued on the Plummer mixture, one in 130 on the log-normal field). A pass
    // over every particle that queued more runs again with room for all of
    // them; an active subset cannot (its j-side mass writes would count twice).
    long long cap = mixed ? std::max(65536ll, c->pairs_symmetric / 8) : 0;
    unsigned long long refined = 0;
    for (int attempt = 0;; attempt++) {
        RefineQueue q{nullptr, nullptr, 0};
        if (mixed) {
            if (ensure(c, c->refined, sizeof(unsigned long long)) || ensure(c, c->rq, sizeof(RefineItem) * (size_t)cap))
                return c->err;
            GZ_CUDA(c, cudaMemsetAsync(c->refined.p, 0, sizeof(unsigned long long), c->stream));
            q = RefineQueue{ptr<RefineItem>(c->rq), ptr<unsigned long long>(c->refined), cap};
        }
        // the rows' sums before the writeback go to the density accumulators
        // (17 x n doubles, unused between density passes)
        const EventPair *ev =
            na > 0 ? timer_launch(c, GZ_TIMER_FORCE, (flux && all) ? c->pairs_symmetric / 2 : c->pairs_symmetric)
                   : nullptr;
        if (mixed)
            force_mixed(c->pp, ps, ptr<int>(c->targets), na, rows, c->tpt_force, ptr<DevStatus>(c->status), c->rec.p,
                        flux, all, q, ptr<double>(c->acc), ev, c->stream);
        else
            force_fp64(c->pp, ps, ptr<int>(c->targets), na, rows, c->tpt_force, ptr<DevStatus>(c->status), c->rec.p,
                       flux, all, ptr<double>(c->acc), ev, c->stream);
        if (na > 0) c->launches += flux ? (mixed ? 5 : 4) : 3;
        GZ_CUDA(c, cudaGetLastError());
        if (!q.item) break;
        GZ_CUDA(c, cudaMemcpyAsync(&refined, c->refined.p, sizeof(refined), cudaMemcpyDeviceToHost, c->stream));
        GZ_CUDA(c, cudaStreamSynchronize(c->stream));
        if ((long long)refined <= cap) break;
        if (!all || attempt > 0)
            return fail(c, GZ_ERR_CAPACITY, "mixed-form force pass: more fragile pairs than the refine queue holds");
        cap = (long long)refined;
        force_preloop(c->pp, ps, ptr<int>(c->targets), na, c->stream);
    }
    if (read_status(c)) return c->err;
    c->pairs_refined = (long long)refined;
    return GZ_OK;
}

int gz_hydro_pass(gz_context *c, int flags)
{
    if (!c || (flags & ~(GZ_PASS_GRAPH | GZ_PASS_RESTAGE))) return GZ_ERR_ARG;
    cudaSetDevice(c->device);
    if (!c->grid_valid) return fail(c, GZ_ERR_ORDER, "pass before upload");
    const bool restage = (flags & GZ_PASS_RESTAGE) != 0;
    // the graph needs the counts of a plain pass to size its buffers, and the
    // kernel timers need plain launches
    const bool graph = (flags & GZ_PASS_GRAPH) && c->n > 0 && c->pairs_symmetric > 0 && !c->timing;
    if (graph) return graph_pass(c, restage);
    int rc = restage ? gz_restage(c) : 0;
    if (!rc) rc = gz_hydro_density(c, nullptr, 0);
    if (!rc) rc = gz_hydro_gradients(c, nullptr, 0);
    if (!rc) rc = gz_hydro_force(c, nullptr, 0);
    return rc;
}

int gz_set_boxes(gz_context *c, int n_boxes, const int64_t *counts)
{
    if (!c || n_boxes < 0 || n_boxes > (1 << 15) || (n_boxes > 1 && !counts)) return GZ_ERR_ARG;
    if (n_boxes <= 1) {
        c->box_counts.clear();
        c->box_bits = 0;
    } else {
        for (int b = 0; b < n_boxes; b++)
            if (counts[b] < 0) return GZ_ERR_ARG;
        int bits = 0;
        while ((1 << bits) < n_boxes) bits++;
        c->box_counts.assign(counts, counts + n_boxes);
        c->box_bits = 3 * ((bits + 2) / 3);  // whole octree levels
    }
    c->grid_valid = false;  // the next upload builds the grid of the boxes
    return GZ_OK;
}

int gz_graph_stats(gz_context *c, gz_graph_info *out)
{
    if (!c || !out) return GZ_ERR_ARG;
    memset(out, 0, sizeof(*out));
    out->captures = c->g.captures;
    out->replays = c->g.replays;
    out->fallbacks = c->g.fallbacks;
    out->kernels_top = c->g.kernels_top;
    out->kernels_per_iteration = c->g.kernels_loop;
    out->kernels_after = c->g.kernels_sym + c->g.kernels_tail;
    return GZ_OK;
}

// The requested output fields, each as (destination, sorted source, values per
// particle, element size).
struct OutField {
    void *dst;
    const void *src;
    int k;
    int bytes;  // 8 (double) or 4 (int)
};

static int output_fields(gz_context *c, const gz_outputs *o, std::vector<OutField> &f)
{
    const size_t n = (size_t)c->n;
    struct { double *dst; DevBuf *src; int k; } d[] = {
        {o->h, &c->h, 1}, {o->num_ngb, &c->num_ngb, 1}, {o->drkern, &c->drkern, 1}, {o->divvel, &c->divvel, 1},
        {o->rho, &c->rho, 1}, {o->pressure, &c->pressure, 1}, {o->nvt, &c->nvt, 6}, {o->cond, &c->cond, 1},
        {o->fce, &c->fce, 1}, {o->pvel, &c->pv, 3}, {o->accel, &c->accel, 3}, {o->dudt, &c->dudt, 1},
        {o->vsig, &c->vsig, 1}, {o->dtmass, &c->dtmass, 1}, {o->dmass, &c->dmass, 1}, {o->gravwork, &c->gw, 3},
        {o->flux_abs, &c->fabs3, 3}};
    for (auto &e : d)
        if (e.dst) {
            if ((size_t)e.k * n * sizeof(double) > e.src->bytes) return fail(c, GZ_ERR_CAPACITY, "output field");
            f.push_back({e.dst, e.src->p, e.k, 8});
        }
    struct { double *dst; int off; int k; } g[] = {{o->grad_rho, 0, 3}, {o->grad_p, 3, 3}, {o->grad_v, 6, 9}};
    for (auto &e : g)
        if (e.dst) f.push_back({e.dst, ptr<double>(c->grad) + (size_t)e.off * n, e.k, 8});
    if (o->iters) f.push_back({o->iters, c->iters.p, 1, 4});
    if (o->wakeup) {
        if (!c->have_bins) return fail(c, GZ_ERR_ORDER, "wakeup: no timebins were uploaded");
        f.push_back({o->wakeup, c->wakeup.p, 1, 4});
    }
    return 0;
}

// one field from sorted to the caller's order, at `to` (device memory)
static void scatter_field(gz_context *c, const OutField &e, void *to, cudaStream_t s)
{
    const int n = c->n;
    const long long cnt = (long long)n * e.k;
    if (e.bytes == 8)
        k_scatter_out<<<(unsigned)((cnt + 255) / 256), 256, 0, s>>>(n, e.k, ptr<int>(c->perm), (const double *)e.src,
                                                                      (double *)to);
    else
        k_scatter_int<<<(n + 255) / 256, 256, 0, s>>>(n, ptr<int>(c->perm), (const int *)e.src, (int *)to);
    c->launches++;
}

// gz_download into host arrays through the staging buffer, or (to_device)
// straight into the caller's device arrays (gz_download_device). The host
// form scatters as many fields as the staging holds (up to 16 doubles per
// particle), copies them out and waits once per such group.
static int download_to(gz_context *c, const gz_outputs *o, bool to_device)
{
    if (!c || !o) return GZ_ERR_ARG;
    if (o->flux_abs && !c->fabs_valid)
        return fail(c, GZ_ERR_ORDER, "flux_abs: the last force pass ran without GZ_DIAG_FLUX_ABS");
    cudaSetDevice(c->device);
    const int n = c->n;
    if (n == 0) return GZ_OK;
    cudaStream_t s = c->stream;
    std::vector<OutField> f;
    if (output_fields(c, o, f)) return c->err;
    if (to_device) {
        for (auto &e : f) scatter_field(c, e, e.dst, s);
        GZ_CUDA(c, cudaGetLastError());
        GZ_CUDA(c, cudaStreamSynchronize(s));
        return GZ_OK;
    }
    const size_t cap = sizeof(double) * 16 * (size_t)n;
    if (ensure(c, c->dl, cap)) return c->err;
    size_t used = 0;
    std::vector<const OutField *> group;
    auto flush = [&]() -> int {
        size_t at = 0;
        for (const OutField *e : group) {
            const size_t nb = (size_t)e->bytes * e->k * n;
            GZ_CUDA(c, cudaMemcpyAsync(e->dst, (char *)c->dl.p + at, nb, cudaMemcpyDeviceToHost, s));
            at += nb;
        }
        GZ_CUDA(c, cudaStreamSynchronize(s));
        group.clear();
        used = 0;
        return 0;
    };
    for (auto &e : f) {
        const size_t nb = (size_t)e.bytes * e.k * n;
        if (used + nb > cap && flush()) return c->err;
        scatter_field(c, e, (char *)c->dl.p + used, s);
        group.push_back(&e);
        used += nb;
    }
    GZ_CUDA(c, cudaGetLastError());
    if (!group.empty() && flush()) return c->err;
    return GZ_OK;
}

// gz_download_async: every requested field is scattered into its own staging
// slot on the context's stream, then copied out on the copy stream, which the
// next pass does not wait for. A second call waits (on the device) until the
// staging is free again; gz_wait waits for the copies.
static int download_async(gz_context *c, const gz_outputs *o)
{
    if (!c || !o) return GZ_ERR_ARG;
    if (o->flux_abs && !c->fabs_valid)
        return fail(c, GZ_ERR_ORDER, "flux_abs: the last force pass ran without GZ_DIAG_FLUX_ABS");
    cudaSetDevice(c->device);
    const int n = c->n;
    if (n == 0) return GZ_OK;
    std::vector<OutField> f;
    if (output_fields(c, o, f)) return c->err;
    size_t total = 0;
    for (auto &e : f) total += (size_t)e.bytes * e.k * n;
    if (copy_stream(c)) return c->err;
    if (c->out_pending) GZ_CUDA(c, cudaStreamWaitEvent(c->stream, c->ev_out_done, 0));
    if (!c->dstage.p || c->dstage.bytes < total) {
        if (c->out_pending) GZ_CUDA(c, cudaEventSynchronize(c->ev_out_done));
        if (!try_ensure(c->dstage, total)) return download_to(c, o, false);  // no room: the plain download
    }
    cudaStream_t s = c->stream;
    size_t at = 0;
    for (auto &e : f) {
        scatter_field(c, e, (char *)c->dstage.p + at, s);
        at += (size_t)e.bytes * e.k * n;
    }
    GZ_CUDA(c, cudaGetLastError());
    GZ_CUDA(c, cudaEventRecord(c->ev_out_ready, s));
    GZ_CUDA(c, cudaStreamWaitEvent(c->cstream, c->ev_out_ready, 0));
    at = 0;
    for (auto &e : f) {
        const size_t nb = (size_t)e.bytes * e.k * n;
        GZ_CUDA(c, cudaMemcpyAsync(e.dst, (char *)c->dstage.p + at, nb, cudaMemcpyDeviceToHost, c->cstream));
        at += nb;
    }
    GZ_CUDA(c, cudaEventRecord(c->ev_out_done, c->cstream));
    c->out_pending = true;
    return GZ_OK;
}

int gz_download(gz_context *c, const gz_outputs *o) { return download_to(c, o, false); }

int gz_download_async(gz_context *c, const gz_outputs *o) { return download_async(c, o); }

int gz_download_device(gz_context *c, const gz_outputs *o) { return download_to(c, o, true); }


// Host-side reorder of rows built for the sorted targets into the caller's
// active order with original indices, each row ascending.
static int rows_to_host(gz_context *c, const int *active, int n_active, int na, DevBuf &off, DevBuf &nbr,
                        std::vector<long long> &h_off, std::vector<int> &h_nbr, std::vector<int> &order)
{
    const int n = c->n;
    cudaStream_t s = c->stream;
    std::vector<long long> o((size_t)na + 1);
    std::vector<int> tg((size_t)std::max(na, 1)), perm((size_t)std::max(n, 1));
    // the rows were written on the context's (non-blocking) stream: copy back on it
    GZ_CUDA(c, cudaMemcpyAsync(o.data(), off.p, sizeof(long long) * ((size_t)na + 1), cudaMemcpyDeviceToHost, s));
    GZ_CUDA(c, cudaStreamSynchronize(s));
    std::vector<int> e((size_t)std::max(o[(size_t)na], 1ll));
    if (o[(size_t)na] > 0)
        GZ_CUDA(c, cudaMemcpyAsync(e.data(), nbr.p, sizeof(int) * (size_t)o[(size_t)na], cudaMemcpyDeviceToHost, s));
    if (na > 0) GZ_CUDA(c, cudaMemcpyAsync(tg.data(), c->targets.p, sizeof(int) * (size_t)na, cudaMemcpyDeviceToHost, s));
    if (n > 0) GZ_CUDA(c, cudaMemcpyAsync(perm.data(), c->perm.p, sizeof(int) * (size_t)n, cudaMemcpyDeviceToHost, s));
    GZ_CUDA(c, cudaStreamSynchronize(s));
    std::vector<int> slot_of_orig((size_t)std::max(n, 1), -1);
    for (int a = 0; a < na; a++) slot_of_orig[(size_t)perm[(size_t)tg[(size_t)a]]] = a;
    const int rows = active ? n_active : n;
    order.assign((size_t)rows, -1);
    for (int r = 0; r < rows; r++) order[(size_t)r] = slot_of_orig[(size_t)(active ? active[r] : r)];
    h_off.assign((size_t)rows + 1, 0);
    for (int r = 0; r < rows; r++) {
        const int a = order[(size_t)r];
        h_off[(size_t)r + 1] = h_off[(size_t)r] + (a >= 0 ? (o[(size_t)a + 1] - o[(size_t)a]) : 0);
    }
    h_nbr.assign((size_t)std::max(h_off[(size_t)rows], 1ll), 0);
    for (int r = 0; r < rows; r++) {
        const int a = order[(size_t)r];
        if (a < 0) continue;
        long long w = h_off[(size_t)r];
        for (long long k = o[(size_t)a]; k < o[(size_t)a + 1]; k++) h_nbr[(size_t)w++] = perm[(size_t)e[(size_t)k]];
        std::sort(h_nbr.begin() + h_off[(size_t)r], h_nbr.begin() + h_off[(size_t)r + 1]);
    }
    return 0;
}

int gz_neighbors(gz_context *c, const int *active, int n_active, int mode, int64_t *offsets, int *nbrs)
{
    if (!c || !offsets || mode < 0 || mode > 2) return GZ_ERR_ARG;
    cudaSetDevice(c->device);
    if (!c->grid_valid) return fail(c, GZ_ERR_ORDER, "neighbours before upload");
    if (mode == 2) {
        // the rows the last gradient/force pass over all particles used
        if (!c->sym_valid || !c->sym_all) return fail(c, GZ_ERR_ORDER, "no symmetric rows of a pass over all particles");
        int na_all = 0;
        if (sort_targets(c, nullptr, 0, &na_all)) return c->err;
        std::vector<long long> h_off;
        std::vector<int> h_nbr, order;
        const int rc = rows_to_host(c, active, n_active, na_all, c->s_off, c->s_nbr, h_off, h_nbr, order);
        if (rc) return rc;
        const size_t rows = order.size();
        for (size_t r = 0; r <= rows; r++) offsets[r] = (int64_t)h_off[r];
        if (nbrs && h_off[rows] > 0) memcpy(nbrs, h_nbr.data(), sizeof(int) * (size_t)h_off[rows]);
        return GZ_OK;
    }
    int na = 0;
    if (sort_targets(c, active, n_active, &na)) return c->err;
    if (mode == 1 && refresh_hmax(c)) return c->err;
    long long total = 0, cap = 0;
    DevBuf cnt, off, nbr;
    int rc = build_rows(c, ptr<double>(c->h), mode, ptr<int>(c->targets), na, cnt, off, nbr, cap, &total);
    std::vector<long long> h_off;
    std::vector<int> h_nbr, order;
    if (!rc) rc = rows_to_host(c, active, n_active, na, off, nbr, h_off, h_nbr, order);
    release(cnt); release(off); release(nbr);
    if (rc) return rc;
    if (read_status(c)) return c->err;
    const size_t rows = order.size();
    for (size_t r = 0; r <= rows; r++) offsets[r] = (int64_t)h_off[r];
    if (nbrs && h_off[rows] > 0) memcpy(nbrs, h_nbr.data(), sizeof(int) * (size_t)h_off[rows]);
    return GZ_OK;
}

int gz_density_sums(gz_context *c, const int *active, int n_active, double *acc, double *pv)
{
    if (!c || !acc) return GZ_ERR_ARG;
    cudaSetDevice(c->device);
    if (!c->grid_valid) return fail(c, GZ_ERR_ORDER, "density sums before upload");
    c->dens_all = false;  // the density rows are about to be replaced
    cudaStream_t s = c->stream;
    int na = 0;
    if (sort_targets(c, active, n_active, &na)) return c->err;
    if (na > 0)
        k_row_radius<<<(na + 255) / 256, 256, 0, s>>>(na, ptr<int>(c->targets), ptr<double>(c->h), 1.0,
                                                       ptr<double>(c->h_built));
    long long total = 0;
    if (build_rows(c, ptr<double>(c->h_built), 0, ptr<int>(c->targets), na, c->counts, c->d_off, c->d_nbr,
                   c->d_nbr_cap, &total))
        return c->err;
    if (na > 0)
        k_set_rows<<<(na + 255) / 256, 256, 0, s>>>(na, ptr<int>(c->targets), ptr<long long>(c->d_off), 0,
                                                    ptr<long long>(c->d_beg), ptr<long long>(c->d_end));
    Particles ps = view(c);
    DensityWork w{};
    w.todo = ptr<int>(c->targets);
    w.n_todo = na;
    w.beg = ptr<long long>(c->d_beg);
    w.end = ptr<long long>(c->d_end);
    w.nbr = ptr<int>(c->d_nbr);
    w.rec = ptr<DensRec>(c->rec);
    density_pack(ps, ptr<DensRec>(c->rec), s);
    w.acc = ptr<double>(c->acc);
    const EventPair *ev = timer_launch(c, GZ_TIMER_DENSITY_SUMS, w.n_todo);
    ev_start(ev, s);
    if (c->prm.precision == GZ_PRECISION_MIXED) density_sums_mixed(c->pp, ps, w, lanes_per_row(c, w.n_todo, 4), s);
    else density_sums_fp64(c->pp, ps, w, lanes_per_row(c, w.n_todo, 4), s);
    ev_stop(ev, s);
    GZ_CUDA(c, cudaGetLastError());
    const int n = c->n;
    std::vector<double> a17((size_t)17 * (size_t)std::max(n, 1));
    std::vector<int> perm((size_t)std::max(n, 1)), tg((size_t)std::max(na, 1));
    GZ_CUDA(c, cudaMemcpyAsync(a17.data(), c->acc.p, sizeof(double) * 17 * (size_t)n, cudaMemcpyDeviceToHost, s));
    GZ_CUDA(c, cudaMemcpyAsync(perm.data(), c->perm.p, sizeof(int) * (size_t)n, cudaMemcpyDeviceToHost, s));
    GZ_CUDA(c, cudaMemcpyAsync(tg.data(), c->targets.p, sizeof(int) * (size_t)na, cudaMemcpyDeviceToHost, s));
    GZ_CUDA(c, cudaStreamSynchronize(s));
    std::vector<int> sorted_of_orig((size_t)std::max(n, 1), -1);
    for (int a = 0; a < na; a++) sorted_of_orig[(size_t)perm[(size_t)tg[(size_t)a]]] = tg[(size_t)a];
    const int rows = active ? n_active : n;
    for (int r = 0; r < rows; r++) {
        const int t = sorted_of_orig[(size_t)(active ? active[r] : r)];
        for (int k = 0; k < 14; k++) acc[(size_t)r * 14 + k] = (t >= 0 && k < 13) ? a17[(size_t)k * n + t] : 0.0;
        if (pv)
            for (int k = 0; k < 3; k++) pv[(size_t)r * 3 + k] = t >= 0 ? a17[(size_t)(14 + k) * n + t] : 0.0;
    }
    return read_status(c) ? c->err : GZ_OK;
}

int gz_get_tuning(gz_context *c, gz_tuning *t)
{
    if (!c || !t) return GZ_ERR_ARG;
    t->leaf_max = c->leaf_max;
    t->reserved = 0;
    t->row_slots = c->row_slots;
    return GZ_OK;
}

int gz_set_tuning(gz_context *c, const gz_tuning *t)
{
    if (!c || !t || t->leaf_max < 8 || t->leaf_max > 1024 || !(t->row_slots >= 1.0 && t->row_slots <= 16.0))
        return GZ_ERR_ARG;
    c->leaf_max = t->leaf_max;
    c->row_slots = t->row_slots;
    return GZ_OK;
}

namespace {
// Tuned walk settings per device, particle count (rounded to a power of two)
// and neighbour count: a context that meets a key already tuned in this
// process takes the result without timing again.
struct TuneKey {
    int device, log2n, ngb, kernel;
    bool operator<(const TuneKey &o) const
    {
        return std::tie(device, log2n, ngb, kernel) < std::tie(o.device, o.log2n, o.ngb, o.kernel);
    }
};
std::mutex g_tune_mutex;
std::map<TuneKey, gz_tuning> g_tuned;
}  // namespace

int gz_autotune(gz_context *c, gz_tuning *chosen)
{
    if (!c) return GZ_ERR_ARG;
    cudaSetDevice(c->device);
    if (!c->grid_valid) return fail(c, GZ_ERR_ORDER, "autotune before upload");
    int log2n = 0;
    while ((1ll << log2n) < (long long)std::max(c->n, 1)) log2n++;
    const TuneKey key{c->device, log2n, (int)std::lround(c->prm.des_num_ngb), c->prm.kernel};
    {
        std::lock_guard<std::mutex> lock(g_tune_mutex);
        auto it = g_tuned.find(key);
        if (it != g_tuned.end()) {
            c->leaf_max = it->second.leaf_max;
            c->row_slots = it->second.row_slots;
            if (chosen) *chosen = it->second;
            return gz_restage(c);
        }
    }
    // Each candidate: rebuild the grid (gz_restage: the uploaded h again) and
    // run a density pass over every particle, timed on the context's stream.
    // The rows, and so every result, are the same for every candidate.
    cudaEvent_t e0, e1;
    GZ_CUDA(c, cudaEventCreate(&e0));
    GZ_CUDA(c, cudaEventCreate(&e1));
    auto trial = [&](int leaf, double slots, float &ms) -> int {
        c->leaf_max = leaf;
        c->row_slots = slots;
        GZ_CUDA(c, cudaEventRecord(e0, c->stream));
        if (gz_restage(c) || gz_hydro_density(c, nullptr, 0)) return c->err;
        GZ_CUDA(c, cudaEventRecord(e1, c->stream));
        GZ_CUDA(c, cudaEventSynchronize(e1));
        GZ_CUDA(c, cudaEventElapsedTime(&ms, e0, e1));
        return 0;
    };
    gz_tuning best{c->leaf_max, 0, c->row_slots};
    float best_ms = 1e30f, ms = 0;
    int rc = 0;
    for (int leaf : {32, 64, 96, 128}) {
        if ((rc = trial(leaf, best.row_slots, ms))) break;
        if (ms < best_ms) { best_ms = ms; best.leaf_max = leaf; }
    }
    for (double slots : {1.5, 2.0, 3.0}) {
        if (rc || (rc = trial(best.leaf_max, slots, ms))) break;
        if (ms < best_ms) { best_ms = ms; best.row_slots = slots; }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (rc) return rc;
    c->leaf_max = best.leaf_max;
    c->row_slots = best.row_slots;
    {
        std::lock_guard<std::mutex> lock(g_tune_mutex);
        g_tuned[key] = best;
    }
    if (chosen) *chosen = best;
    return gz_restage(c);
}

int gz_set_bin_active(gz_context *c, const int *bin_active)
{
    if (!c) return GZ_ERR_ARG;
    cudaSetDevice(c->device);
    if (!bin_active) { c->binact_on = false; return GZ_OK; }
    if (ensure(c, c->binact, sizeof(int) * GZ_TIMEBINS)) return c->err;
    GZ_CUDA(c, cudaMemcpyAsync(c->binact.p, bin_active, sizeof(int) * GZ_TIMEBINS, cudaMemcpyHostToDevice, c->stream));
    GZ_CUDA(c, cudaStreamSynchronize(c->stream));
    c->binact_on = true;
    return GZ_OK;
}

int gz_active_list(gz_context *c, const int *bin_active, int *out, int *n_out)
{
    if (!c || !bin_active || !n_out) return GZ_ERR_ARG;
    cudaSetDevice(c->device);
    if (!c->grid_valid || !c->have_bins) return fail(c, GZ_ERR_ORDER, "active list: no timebins were uploaded");
    const int n = c->n;
    cudaStream_t s = c->stream;
    const size_t N = (size_t)std::max(n, 1);
    DevBuf tab;  // this call's table; the wake-up keeps the one gz_set_bin_active gave
    if (ensure(c, tab, sizeof(int) * GZ_TIMEBINS) || ensure(c, c->sel_flags, sizeof(int) * N) ||
        ensure(c, c->sel_out, sizeof(int) * N) || ensure(c, c->n_sel, sizeof(int) * 2) ||
        ensure(c, c->targets_tmp, sizeof(int) * N))
        return c->err;
    GZ_CUDA(c, cudaMemcpyAsync(tab.p, bin_active, sizeof(int) * GZ_TIMEBINS, cudaMemcpyHostToDevice, s));
    *n_out = 0;
    if (n > 0) {
        k_iota<<<(n + 255) / 256, 256, 0, s>>>(n, ptr<int>(c->targets_tmp));
        k_active_flags<<<(n + 255) / 256, 256, 0, s>>>(n, ptr<int>(c->o_timebin), ptr<double>(c->o_mass), ptr<int>(tab),
                                                       ptr<int>(c->sel_flags));
        c->launches += 2;
        size_t tmp = 0;
        cub::DeviceSelect::Flagged(nullptr, tmp, ptr<int>(c->targets_tmp), ptr<int>(c->sel_flags), ptr<int>(c->sel_out),
                                   ptr<int>(c->n_sel), n, s);
        if (ensure(c, c->cub_tmp, tmp)) { release(tab); return c->err; }
        cub::DeviceSelect::Flagged(c->cub_tmp.p, tmp, ptr<int>(c->targets_tmp), ptr<int>(c->sel_flags),
                                   ptr<int>(c->sel_out), ptr<int>(c->n_sel), n, s);
        int k = 0;
        GZ_CUDA(c, cudaMemcpyAsync(&k, c->n_sel.p, sizeof(int), cudaMemcpyDeviceToHost, s));
        GZ_CUDA(c, cudaStreamSynchronize(s));
        *n_out = k;
        if (out && k > 0) {
            GZ_CUDA(c, cudaMemcpyAsync(out, c->sel_out.p, sizeof(int) * (size_t)k, cudaMemcpyDeviceToHost, s));
            GZ_CUDA(c, cudaStreamSynchronize(s));
        }
    }
    release(tab);
    GZ_CUDA(c, cudaGetLastError());
    return GZ_OK;
}

int gz_wakeup_bins(gz_context *c, const int *bin_active, int max_time_bin_active, int lowest_occupied_active_bin,
                   int *timebin_out, int *n_moved)
{
    if (!c || !bin_active || !timebin_out) return GZ_ERR_ARG;
    if (max_time_bin_active < 0 || max_time_bin_active >= GZ_TIMEBINS) return GZ_ERR_ARG;
    cudaSetDevice(c->device);
    if (!c->grid_valid || !c->have_bins) return fail(c, GZ_ERR_ORDER, "wakeup bins: no timebins were uploaded");
    const int n = c->n;
    cudaStream_t s = c->stream;
    DevBuf tab, moved;
    if (ensure(c, tab, sizeof(int) * GZ_TIMEBINS) || ensure(c, moved, sizeof(unsigned long long)) ||
        ensure(c, c->dl, sizeof(double) * 9 * (size_t)std::max(n, 1)))
        return c->err;
    GZ_CUDA(c, cudaMemcpyAsync(tab.p, bin_active, sizeof(int) * GZ_TIMEBINS, cudaMemcpyHostToDevice, s));
    GZ_CUDA(c, cudaMemsetAsync(moved.p, 0, sizeof(unsigned long long), s));
    unsigned long long m = 0;
    if (n > 0) {
        k_wakeup_bins<<<(n + 255) / 256, 256, 0, s>>>(n, ptr<int>(c->perm), ptr<int>(c->timebin), ptr<int>(c->wakeup),
                                                      ptr<double>(c->m), ptr<int>(tab), max_time_bin_active,
                                                      lowest_occupied_active_bin, ptr<int>(c->dl),
                                                      ptr<unsigned long long>(moved));
        c->launches++;
        GZ_CUDA(c, cudaMemcpyAsync(timebin_out, c->dl.p, sizeof(int) * (size_t)n, cudaMemcpyDeviceToHost, s));
        GZ_CUDA(c, cudaMemcpyAsync(&m, moved.p, sizeof(m), cudaMemcpyDeviceToHost, s));
    }
    GZ_CUDA(c, cudaStreamSynchronize(s));
    release(tab);
    release(moved);
    if (n_moved) *n_moved = (int)m;
    return GZ_OK;
}

int gz_status(gz_context *c, gz_status_info *info)
{
    if (!c || !info) return GZ_ERR_ARG;
    memset(info, 0, sizeof(*info));
    cudaSetDevice(c->device);
    read_status(c);
    info->code = c->err;
    info->index = -1;
    if (c->err_index >= 0 && c->err_index < c->n && c->perm.p) {
        int orig = -1;
        if (cudaMemcpyAsync(&orig, ptr<int>(c->perm) + c->err_index, sizeof(int), cudaMemcpyDeviceToHost, c->stream) ==
                cudaSuccess &&
            cudaStreamSynchronize(c->stream) == cudaSuccess)
            info->index = orig;
    }
    info->density_iterations = c->last_iters;
    info->h_iter_max = c->h_iter_max;
    info->pairs_refined = c->pairs_refined;
    info->kernel_launches = c->launches;
    info->pairs_density = c->pairs_density;
    info->pairs_symmetric = c->pairs_symmetric;
    size_t bytes = 0;
    for (DevBuf *b : all_buffers(c)) bytes += b->bytes;
    info->device_bytes = (int64_t)bytes;
    snprintf(info->message, sizeof(info->message), "%s", c->msg);
    return GZ_OK;
}

}  // extern "C"

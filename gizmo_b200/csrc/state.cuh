// gizmo_b200/csrc/state.cuh -- device-resident structure-of-arrays particle mirror.
//
// All arrays are in Morton-sorted order (the order of the neighbour grid),
// component-major ([k][n]) so a warp reading one field of consecutive
// particles issues one coalesced transaction per component. The host
// original order is recovered through `perm` (sorted -> original).
#pragma once

#include "common.cuh"
#include "physics.cuh"

namespace gz {

struct Particles {
    int n;
    const double *x, *y, *z;        // P.Pos
    const double *vx, *vy, *vz;     // CellP.VelPred
    const double *m;                // P.Mass
    const double *u;                // CellP.InternalEnergyPred
    const double *dt;               // physical timestep
    double *h;                      // P.KernelRadius
    double *cond;                   // CellP.ConditionNumber (in: previous step, out: new)
    double *num_ngb, *drkern, *divvel, *rho, *pressure, *fce;
    double *nvt;                    // [6][n] inverse NV_T, xx yy zz xy yz xz
    double *pv;                     // [3][n] CellP.ParticleVel (MFV)
    double *grad;                   // [15][n] d rho (3), d P (3), d v_k (3 x 3)
    double *accel;                  // [3][n]
    double *dudt, *vsig, *dtmass, *dmass;
    double *gw;                     // [3][n] GravWorkTerm
    double *fabs;                   // [3][n] sums of |mass|, |momentum|, |energy| pair fluxes (diagnostic)
    int *iters;
    const unsigned char *active;    // 1 for particles of the current active set
    // wake-up of inactive neighbours (hydro_functions.h:534-544); bin_active null: off
    const int *timebin;             // P.TimeBin
    const double *vsig_prev;        // CellP.MaxSignalVel from each cell's last force pass
    int *wakeup;                    // out: largest waker bin + 1 (0: none)
    const int *bin_active;          // TimeBinActive[60]
};

constexpr double kWakeup = 4.1;  // WAKEUP (declarations/constants.h:11-13; no GR, slope-limiter tolerance > 0)

// The wake-up test of one evaluated pair: `t` the active row owner, `j` its
// neighbour, vsig_ts the pair's timestep signal speed (hydro_functions.h:534-544).
GZ_DEV void wakeup_test(const Particles &ps, int t, int j, double vsig_ts)
{
    if (ps.bin_active && !ps.bin_active[ps.timebin[j]] && vsig_ts > kWakeup * ps.vsig_prev[j])
        atomicMax(ps.wakeup + j, ps.timebin[t] + 1);  // wakeup_flag_from_timebin, core/proto.h:181
}

// Octree over the Morton-sorted particles (63-bit keys, 21 levels): node i
// owns the sorted run [first, first + count); an internal node's children
// are the nodes [child, child + nchild); a leaf (child = -1) has at most
// leaf_max particles unless it is at the deepest level (coincident keys).
// Leaves are tested 32 particles at a time; leaves of up to 96 particles
// (measured against 8 to 128) cost the walk fewer node openings than the extra
// candidate tests they bring.
constexpr int kLeafMax = 96;  // the default leaf size (gz_tuning.leaf_max)

struct Tree {
    double box;
    int n_nodes;
    int n_particles;
    const int4 *node;               // {first, count, child or -1, nchild}
    const double4 *lo;              // tight box minimum xyz; w = maximum h in the node
    const double4 *hi;              // tight box maximum xyz
    // box sets (null for one box): each particle's box (sorted order) and the
    // node of each box's subtree, where the walk of its particles starts
    const int *box_of;
    const int *root_of;
};

// Device state of the octree build (tree_build_device).
struct TreeBuild {
    int level_beg, level_cnt, next_cnt, total, fail, L;
};

// What a density row reads of each neighbour, in one 64-byte record (sorted
// order), packed once per pass: the pair loop then issues two 32-byte reads
// per neighbour instead of seven scattered ones.
struct __align__(16) DensRec {
    double x, y, z, m, vx, vy, vz, pad;
};

// Compressed neighbour rows: row r of `slot_of` targets.
// CUDA events recorded around one kernel of a pass, for the caller's timing
// (null: not timed).
struct EventPair {
    cudaEvent_t start, stop;
};

// Mixed-form force pairs whose FP32 branch decisions were too close to call
// (Guard<float>): each names the flux entries it was stored at (row i's and,
// for a pair evaluated once, row j's; -1 if none) and the pair in canonical
// orientation (i the lower sorted index). force_refine evaluates them again in
// FP64 and overwrites those entries before the rows are accumulated.
struct RefineItem {
    long long e, a;
    int i, j;
    int t;      // the active row owner for the wake-up test (-1: none; every particle active)
    int pad;
};
struct RefineQueue {
    RefineItem *item;            // null: nothing is queued (the FP64 form)
    unsigned long long *count;   // items pushed (may pass cap: the pass then runs again with room for all)
    long long cap;
};

struct Csr {
    const long long *off;           // [rows + 1]
    const int *nbr;                 // sorted particle indices
};

// The density iteration's control state on the device, for a pass captured as
// one CUDA graph (no host round trip between iterations). Each iteration takes
// its targets from one list and selects, in list order, the ones still
// iterating into the next and those whose radius outgrew their row into the
// regrow list; the rows rebuilt are those of every target in the first
// iteration and of the regrow list afterwards. `fail` stops the graph's work
// where a device-sized buffer would overflow (the host then runs the pass
// without the graph).
struct GraphState {
    int n_todo, n_grow, iter, fail;
    int n_next, n_regrow, n_over, tpt;  // this iteration's selections, padded-row overflows, density lanes
    int cap, walk_solo, next_group[2];  // padded slots, walk mode, walk work counters
    long long base, need, extra;        // padded entries in use, after this iteration's block, overflow room
    long long entries;                  // density row entries built (the pass's pairs_density)
    long long sym_total;                // symmetric row entries
    int todo_left;                      // after the loop: targets still iterating (MAXITER reached)
    int sums_next, after_next;          // the density sums' and after_iter's next chunk of the list
    int pad;
};

// Fail reasons (GraphState::fail, bit flags).
constexpr int kGraphFailRows = 1;   // padded density rows beyond the row buffer
constexpr int kGraphFailSym = 2;    // symmetric rows beyond their buffers or the pair-flux buffer
constexpr int kGraphFailTree = 4;   // a restage in the graph: the octree beyond its nodes

}  // namespace gz

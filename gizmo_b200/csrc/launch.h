// gizmo_b200/csrc/launch.h -- host launchers shared by the C-ABI layer.
#pragma once

#include <cuda_runtime.h>
#include <cstdint>

#include "state.cuh"

namespace gz {

// grid.cu
// keys of axis_bits per axis, with the box index above them for box sets (bid non-null)
void grid_keys(int n, const double *pos, double box, const int *bid, int axis_bits, unsigned long long *keys, int *idx,
               cudaStream_t s);
void tree_count(const unsigned long long *keys, int L, const int4 *node, int beg, int cnt, long long *nch,
                int leaf_max, int split_levels, cudaStream_t s);
// the subtree of each box from the nodes of the level below the box bits
void box_roots(int beg, int cnt, const int4 *node, const int *box_of, int *root_of, cudaStream_t s);
void tree_write(const unsigned long long *keys, int L, int4 *node, int *parent, int beg, int cnt,
                const long long *cpos, int next, cudaStream_t s);
// boxes and h maxima bottom-up over the first n_nodes nodes (or *n_nodes_dev of them, when given)
void tree_up(int n_nodes, const int4 *node, const int *parent, const double *x, const double *y, const double *z,
             const double *h, double4 *lo, double4 *hi, int *done, int boxes, cudaStream_t s,
             const int *n_nodes_dev = nullptr);
// the octree of n sorted keys built level by level on the device (TreeBuild on
// the device: total nodes, fail when cap would be passed)
void tree_build_device(const unsigned long long *keys, int n, int4 *node, int *parent, TreeBuild *tb, int cap,
                       int leaf_max, int split_levels, const int *box_of, int *root_of, int blocks, cudaStream_t s);
void walk_rows(const Tree &t, const double *x, const double *y, const double *z, const double *reach,
               const double *hsym, int symmetric, const int *targets, int n_targets, long long *counts,
               const long long *off, int *nbr, int cap, DevStatus *st, int *next_group, cudaStream_t s);
// The padded density-row fill of a captured pass (both walk modes launched;
// the state names the one that runs) and the fill of its overflow rows.
void walk_rows_graph(const Tree &t, const double *x, const double *y, const double *z, const double *reach,
                     const int *first, const int *grow, GraphState *gs, long long *counts, int *nbr, DevStatus *st,
                     cudaStream_t s);
// warps the group-mode walk holds resident (the walk takes one warp per
// target when a sparse list's groups would not fill them)
long long walk_group_warps();
void walk_over_graph(const Tree &t, const double *x, const double *y, const double *z, const double *reach,
                     const int *list, const long long *off, GraphState *gs, int *nbr, DevStatus *st, int blocks,
                     cudaStream_t s);
// rows of a padded fill (cap > 0 above): [beg, end) for the rows that fit, over[a] = 1 for the others
void padded_rows(int na, const int *t, const long long *counts, int cap, long long base, long long *beg,
                 long long *end, unsigned char *over, cudaStream_t s);

// symmetric rows derived from the density rows of a pass over all particles
void sym_split(int n, const double *x, const double *y, const double *z, const double *h, double box,
               const long long *beg, const long long *end, int *nbr, int *acnt, int *bcnt, cudaStream_t s);
void sym_counts(int n, const int *acnt, const int *bcnt, long long *cnt, cudaStream_t s);
void sym_scatter(int n, const long long *beg, const int *nbr, const int *acnt, const long long *s_off, int *bcur,
                 int *rows, cudaStream_t s);
void sym_sort(int n, const long long *s_off, const int *acnt, const int *rows, int *out, cudaStream_t s);

// Work description of the density iteration.
struct DensityWork {
    const int *todo;        // sorted indices still iterating
    int n_todo;
    const long long *beg;   // sorted index -> its density row [beg, end) in nbr
    const long long *end;
    const int *nbr;
    const DensRec *rec;     // packed neighbour records (sorted index)
    double *acc;            // [17][n] per-particle accumulator (sorted index)
    double *h_built;        // search radius each row was built with
    DensityScratch *scratch;
    unsigned char *keep;    // per todo slot: still iterating
    unsigned char *regrow;  // per todo slot: its radius outgrew its row
    int *rebuild;           // set when any radius outgrows its row
    unsigned long long *h_iter_max;  // atomic maximum of every radius the iteration moves to (double bits)
    int iter;
};

// passes_fp64.cu / passes_mixed.cu (same kernels, pair arithmetic double / float)
struct PassLaunch {
    int tpt_density, tpt_gradient, tpt_force;
};

void density_pack(const Particles &ps, DensRec *rec, cudaStream_t s);
void density_sums_fp64(const PassParams &p, const Particles &ps, const DensityWork &w, int tpt, cudaStream_t s);
void density_sums_mixed(const PassParams &p, const Particles &ps, const DensityWork &w, int tpt, cudaStream_t s);
void density_after_iter(const PassParams &p, const Particles &ps, const DensityWork &w, DevStatus *st, cudaStream_t s);
// Captured-pass forms (GraphState): every TPT instance is launched with `blocks`
// blocks and the one the device state names runs; after_iter writes the
// per-slot flags of w.keep and w.regrow for the iteration's target count.
void density_sums_graph(const PassParams &p, const Particles &ps, const DensityWork &w, GraphState *gs,
                        const int *todo, int blocks, cudaStream_t s);
void density_after_iter_graph(const PassParams &p, const Particles &ps, const DensityWork &w, DevStatus *st,
                              GraphState *gs, const int *todo, int blocks, cudaStream_t s);
void density_finalize(const PassParams &p, const Particles &ps, const double *acc, const int *targets, int n_targets,
                      cudaStream_t s);
// `rec` is scratch for the packed neighbour records: at least n x
// record_bytes(pass) bytes, 16-byte aligned.
size_t gradient_record_bytes(int mixed);
size_t force_record_bytes(int mixed);  // the force record and the gather record of a particle
size_t pair_flux_bytes(int mixed);  // per symmetric row entry, for a force pass evaluating each pair once
void gradients_fp64(const PassParams &p, const Particles &ps, const int *targets, int n_targets, Csr rows, int tpt,
                    void *rec, const EventPair *ev, cudaStream_t s);
// flux: NULL, or (every particle a target, targets[s] = s) scratch for one
// evaluation per pair: n_entries x pair_flux_bytes. sums: 13 x n doubles of
// scratch (the row sums before the writeback).
// `all`: every particle is a target (flux then holds each pair once). The
// mixed form needs flux; q receives its fragile pairs (cap >= 1).
void force_fp64(const PassParams &p, const Particles &ps, const int *targets, int n_targets, Csr rows, int tpt,
                DevStatus *st, void *rec, void *flux, bool all, double *sums, const EventPair *ev, cudaStream_t s);
void force_mixed(const PassParams &p, const Particles &ps, const int *targets, int n_targets, Csr rows, int tpt,
                 DevStatus *st, void *rec, void *flux, bool all, const RefineQueue &q, double *sums,
                 const EventPair *ev, cudaStream_t s);
// The queued pairs of a mixed-form pass evaluated in FP64 from the FP64 mirror
// (the FP64 form's arithmetic bit for bit), their fluxes stored over the FP32
// ones at both entries; the queue's count stays on the device.
void force_refine(const PassParams &p, const Particles &ps, const RefineQueue &q, PairFlux<float> *flux,
                  DevStatus *st, cudaStream_t s);
void force_preloop(const PassParams &p, const Particles &ps, const int *targets, int n_targets, cudaStream_t s);

}  // namespace gz

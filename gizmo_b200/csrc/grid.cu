// gizmo_b200/csrc/grid.cu -- Morton-sorted octree and exact neighbour rows.
//
// Replaces the reference's SIDX spatial index + BVH walk + two-pass CSR
// (src/mesh/gpu_neighbor_list.cc:1134-1169, 1736-1816;
// src/mesh/gpu_neighbor_list.h:207-264). Particles are sorted by a 63-bit
// Morton key (21 bits per axis); every octree node is then one contiguous
// run of the sorted arrays. The tree is explicit: it is split top-down one
// level per launch (a node with more than leaf_max particles gets its
// non-empty children, stored contiguously), then a single bottom-up launch
// gives every node the tight bounding box of its particles and the maximum
// of their h. A 1e5 density contrast only adds levels where the particles
// are, and the walk never searches: a node's children are one index range.
//
// Neighbour rows come from a warp-cooperative walk: one warp takes 32
// consecutive sorted targets and descends the tree once for the group. A node
// is opened when the search sphere of at least one lane reaches its box (each
// lane tests its own target), so 32 targets on both sides of a jump of the
// Morton curve cost two small searches, not one search of their joint
// bounding box. Leaf particles are staged through shared memory, and every
// lane whose sphere reached the leaf tests them. Box and candidate tests run
// in FP32 with outward margins that bound the FP32 rounding; only a candidate
// within that margin of its sphere takes the FP64 test. Membership is thus the
// reference predicates on FP64 minimum-image separations rounded exactly as
// the CPU does, so the rows are bit-identical to an exact CPU search:
//   one-way   r2 < R_i^2                                (density, R = buffered h)
//   symmetric r2 > 0 and !(r2 >= h_i^2 and r2 >= h_j^2) (gradients, force)
#include <cub/cub.cuh>

#include <atomic>

#include "launch.h"

namespace gz {

constexpr int kBits = 21;  // Morton levels

GZ_DEV unsigned long long spread21(unsigned long long x)
{
    x &= 0x1fffffull;
    x = (x | (x << 32)) & 0x1f00000000ffffull;
    x = (x | (x << 16)) & 0x1f0000ff0000ffull;
    x = (x | (x << 8)) & 0x100f00f00f00f00full;
    x = (x | (x << 4)) & 0x10c30c30c30c30c3ull;
    x = (x | (x << 2)) & 0x1249249249249249ull;
    return x;
}

// Morton key of `axis_bits` bits per axis; with box sets (bid non-null) the
// particle's box index above them, so every box is one run of the sorted keys
// and one subtree of the octree (its top levels split the box bits).
__global__ void k_keys(int n, const double *__restrict__ pos, double box, const int *__restrict__ bid, int axis_bits,
                       unsigned long long *keys, int *idx)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const long long G = 1ll << axis_bits;
    unsigned long long c[3];
    for (int k = 0; k < 3; k++) {
        long long v = (long long)(pos[3 * (size_t)i + k] / box * (double)G);
        v = v < 0 ? 0 : (v >= G ? G - 1 : v);
        c[k] = (unsigned long long)v;
    }
    unsigned long long key = spread21(c[0]) | (spread21(c[1]) << 1) | (spread21(c[2]) << 2);
    if (bid) key |= (unsigned long long)bid[i] << (3 * axis_bits);
    keys[i] = key;
    idx[i] = i;
}

// The subtree of each box: the nodes of the level below the box bits, each one
// box's particles.
__global__ void k_box_roots(int beg, int cnt, const int4 *__restrict__ node, const int *__restrict__ box_of,
                            int *root_of)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= cnt) return;
    root_of[box_of[node[beg + i].x]] = beg + i;
}

// first position in [a, b) whose key is >= key
GZ_DEV int lower_bound_key(const unsigned long long *__restrict__ keys, int a, int b, unsigned long long key)
{
    while (a < b) {
        const int mid = a + ((b - a) >> 1);
        if (keys[mid] < key) a = mid + 1; else b = mid;
    }
    return a;
}

// The run [a, b) of a level-L node split into its 8 children (level L+1):
// child d is [bound[d], bound[d+1]).
GZ_DEV void child_bounds(const unsigned long long *__restrict__ keys, int a, int b, int L, int bound[9])
{
    const int shift = 3 * (kBits - L - 1);
    const unsigned long long prefix = keys[a] >> (shift + 3);
    bound[0] = a;
    int lo = a;
    for (int d = 0; d < 7; d++) {
        lo = lower_bound_key(keys, lo, b, ((prefix << 3) + (unsigned long long)(d + 1)) << shift);
        bound[d + 1] = lo;
    }
    bound[8] = b;
}

// number of non-empty children of every node of one level
// (levels above split_levels split whatever their size: the box bits of box sets)
__global__ void k_tree_count(const unsigned long long *__restrict__ keys, int L, const int4 *__restrict__ node,
                             int beg, int cnt, long long *nch, int leaf_max, int split_levels)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= cnt) return;
    const int4 nd = node[beg + i];
    int c = 0;
    if ((nd.y > leaf_max || L < split_levels) && L < kBits) {
        int bound[9];
        child_bounds(keys, nd.x, nd.x + nd.y, L, bound);
        for (int d = 0; d < 8; d++) c += bound[d + 1] > bound[d];
    }
    nch[i] = c;
}

// ---------------------------------------------- the octree built on the device
// All levels in one stream of launches with no host round trip: each level's
// nodes take their children's places from a counter (a node's children are
// contiguous and in octant order; the order of the nodes of a level depends on
// the atomics, and nothing downstream depends on it: the walks follow child
// ranges, the boxes are reduced bottom-up). A level that would pass the node
// capacity sets `fail` and the host builds the tree level by level instead.
__global__ void k_tree_init(TreeBuild *tb, int4 *node, int *parent, int n)
{
    node[0] = make_int4(0, n, -1, 0);
    parent[0] = -1;
    TreeBuild t{};
    t.level_cnt = n > 0 ? 1 : 0;
    t.total = t.level_cnt;
    *tb = t;
}

__global__ void k_tree_level(const unsigned long long *__restrict__ keys, int4 *node, int *parent, TreeBuild *tb,
                             int cap, int leaf_max, int split_levels, const int *__restrict__ box_of, int *root_of)
{
    if (tb->fail) return;
    const int L = tb->L, beg = tb->level_beg, cnt = tb->level_cnt, end = tb->total;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < cnt; i += gridDim.x * blockDim.x) {
        int4 nd = node[beg + i];
        if (box_of && L == split_levels) root_of[box_of[nd.x]] = beg + i;  // one node per box
        int bound[9];
        int c = 0;
        if ((nd.y > leaf_max || L < split_levels) && L < kBits) {
            child_bounds(keys, nd.x, nd.x + nd.y, L, bound);
            for (int d = 0; d < 8; d++) c += bound[d + 1] > bound[d];
        }
        nd.z = -1;
        nd.w = 0;
        if (c > 0) {
            const int first = end + atomicAdd(&tb->next_cnt, c);
            if ((long long)first + c > cap) {
                atomicOr(&tb->fail, 1);
            } else {
                int k = 0;
                for (int d = 0; d < 8; d++) {
                    if (bound[d + 1] > bound[d]) {
                        node[first + k] = make_int4(bound[d], bound[d + 1] - bound[d], -1, 0);
                        parent[first + k] = beg + i;
                        k++;
                    }
                }
                nd.z = first;
                nd.w = c;
            }
        }
        node[beg + i] = nd;
    }
}

__global__ void k_tree_next(TreeBuild *tb)
{
    TreeBuild &t = *tb;
    t.level_beg = t.total;
    t.level_cnt = t.fail ? 0 : t.next_cnt;
    t.total += t.level_cnt;
    t.next_cnt = 0;
    t.L++;
}

// children of one level written at next + cpos[i] (cpos: inclusive scan of nch)
__global__ void k_tree_write(const unsigned long long *__restrict__ keys, int L, int4 *node, int *parent, int beg,
                             int cnt, const long long *__restrict__ cpos, int next)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= cnt) return;
    int4 nd = node[beg + i];
    const int first_child = next + (int)cpos[i];
    const int c = (int)(cpos[i + 1] - cpos[i]);
    if (c == 0) {
        nd.z = -1;
        nd.w = 0;
    } else {
        int bound[9];
        child_bounds(keys, nd.x, nd.x + nd.y, L, bound);
        int k = 0;
        for (int d = 0; d < 8; d++) {
            if (bound[d + 1] > bound[d]) {
                node[first_child + k] = make_int4(bound[d], bound[d + 1] - bound[d], -1, 0);
                parent[first_child + k] = beg + i;
                k++;
            }
        }
        nd.z = first_child;
        nd.w = c;
    }
    node[beg + i] = nd;
}

// L2-coherent 32-byte load/store (values written by other blocks of this launch)
GZ_DEV double4 ld_cg4(const double4 *p)
{
    const double2 a = __ldcg((const double2 *)p), b = __ldcg((const double2 *)p + 1);
    return make_double4(a.x, a.y, b.x, b.y);
}
GZ_DEV void st_cg4(double4 *p, double4 v)
{
    __stcg((double2 *)p, make_double2(v.x, v.y));
    __stcg((double2 *)p + 1, make_double2(v.z, v.w));
}

// Bottom-up bounding boxes and h maxima in one launch: a leaf reduces its
// particles, and the last child to finish (atomic count per parent) reduces
// the parent's children, and so on to the root. With boxes == 0 only the h
// maxima (lo.w) are refreshed.
__global__ void k_tree_up(int n_nodes, const int *__restrict__ n_nodes_dev, const int4 *__restrict__ node,
                          const int *__restrict__ parent, const double *__restrict__ x, const double *__restrict__ y,
                          const double *__restrict__ z, const double *__restrict__ h, double4 *lo, double4 *hi,
                          int *done, int boxes)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (n_nodes_dev ? *n_nodes_dev : n_nodes)) return;
    const int4 nd = node[i];
    if (nd.z >= 0) return;  // internal: reduced by its last child
    double4 l = make_double4(1e300, 1e300, 1e300, 0.0), u = make_double4(-1e300, -1e300, -1e300, 0.0);
    for (int j = nd.x; j < nd.x + nd.y; j++) {
        if (boxes) {
            const double px = x[j], py = y[j], pz = z[j];
            l.x = fmin(l.x, px); l.y = fmin(l.y, py); l.z = fmin(l.z, pz);
            u.x = fmax(u.x, px); u.y = fmax(u.y, py); u.z = fmax(u.z, pz);
        }
        const double hv = h[j];
        if (hv > l.w) l.w = hv;
    }
    if (boxes) { lo[i] = l; hi[i] = u; } else { lo[i].w = l.w; }
    int p = parent[i];
    while (p >= 0) {
        __threadfence();
        const int4 pn = node[p];
        if (atomicAdd(done + p, 1) != pn.w - 1) return;
        __threadfence();
        l = make_double4(1e300, 1e300, 1e300, 0.0);
        u = make_double4(-1e300, -1e300, -1e300, 0.0);
        for (int c = pn.z; c < pn.z + pn.w; c++) {
            const double4 cl = ld_cg4(lo + c);
            if (boxes) {
                const double4 cu = ld_cg4(hi + c);
                l.x = fmin(l.x, cl.x); l.y = fmin(l.y, cl.y); l.z = fmin(l.z, cl.z);
                u.x = fmax(u.x, cu.x); u.y = fmax(u.y, cu.y); u.z = fmax(u.z, cu.z);
            }
            l.w = fmax(l.w, cl.w);
        }
        if (boxes) { st_cg4(lo + p, l); st_cg4(hi + p, u); } else { __stcg(&lo[p].w, l.w); }
        p = parent[p];
    }
}

// Periodic gap between a point and a box [l, u] on one axis (both inside
// [0, box)) in FP32, minus an allowance `eps` that covers the FP32 rounding of
// the point, the box (rounded outward) and the subtractions: never larger than
// the FP64 gap.
GZ_DEV float axis_gap_f(float x, float l, float u, float box, float eps)
{
    float g;
    if (x < l) g = fminf(l - x, x + box - u);
    else if (x > u) g = fminf(x - u, l + box - x);
    else return 0.0f;
    g -= eps;
    return g > 0.0f ? g : 0.0f;
}

GZ_DEV float wrap1f(float d, float box, float half)
{
    return (d > half) ? d - box : ((d < -half) ? d + box : d);
}

constexpr int kStack = 160;  // >= 7 x 22 levels + 8
constexpr int kMaxWalkDevices = 64;  // devices whose launch shapes are cached
constexpr int kWarps = 8;    // warps per block of the walks

// A node waiting on a warp's stack: its run, its children and the lanes whose
// search sphere reached its box (tested when its parent was opened).
struct StackNode {
    int first, count, child, nchild;
    unsigned lanes;
};

// FP32 screening of a candidate at FP32 separation r2f from a target whose
// search radius is R (FP32, rounded up): 0 = outside, 1 = inside, 2 = too close
// to the boundary to tell (the FP64 test decides). `scr` bounds the difference
// between an FP32 separation and the FP64 one: positions lie in [0, box), so
// each rounding to FP32 and each FP32 subtraction is within 2^-24 box, and
// three axes of three roundings each stay below 6 x 2^-24 box; scr = 8 x
// 2^-24 box. With `positive` the pair also needs r > 0 (symmetric rows).
GZ_DEV int screen(float r2f, float R, float scr, bool positive)
{
    const float hi = R + scr;
    if (r2f > hi * hi) return 0;
    const float lo = R - scr;
    if (lo > 0.0f && r2f < lo * lo && (!positive || r2f > 4.0f * scr * scr)) return 1;
    return 2;
}

// Warp-cooperative tree walk. FILL=false counts rows; FILL=true writes them.
//   SOLO=false: the warp's 32 lanes hold 32 consecutive targets; a node is
//     opened if any lane's sphere reaches it and a leaf particle is tested by
//     every lane that reached the leaf.
//   SOLO=true: the warp walks one target (for sparse target lists, whose
//     targets are far apart); the lanes test 32 leaf particles at once and a
//     ballot compacts the accepted ones, so the row (content and order) is the
//     one the other mode writes.
// Opening a node loads its children's records in one coalesced access
// (children are contiguous) and tests them there, so only reached children
// are pushed and a pop costs no memory round trip. Box tests and candidate
// tests run in FP32 with outward margins; a candidate within the margin of
// its sphere is decided by the exact FP64 predicate, so the rows are those of
// the FP64 predicates alone.
template <bool SYM, bool FILL, bool SOLO>
__device__ __forceinline__ void walk_group(const int group, const Tree &t, const double *__restrict__ x,
                                           const double *__restrict__ y, const double *__restrict__ z,
                                           const double *__restrict__ reach, const double *__restrict__ hsym,
                                           const int *__restrict__ targets, int n_targets, long long *counts,
                                           const long long *__restrict__ off, int *nbr, int cap, DevStatus *st,
                                           StackNode (*s_stack)[kStack], double4 (*s_c)[32], float4 (*s_cf)[32],
                                           float4 (*s_lo)[8], float4 (*s_hi)[8], int4 (*s_nd)[8])
{
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    const unsigned full = 0xffffffffu;
    const int slot = SOLO ? group : group * 32 + lane;
    const bool valid = slot < n_targets;
    const int tg = valid ? targets[slot] : -1;
    const double box = t.box, half = 0.5 * box;
    const float boxf = (float)box, halff = 0.5f * boxf;
    const float scr = 4.77e-7f * boxf;  // 8 x 2^-24 box
    double xi = 0, yi = 0, zi = 0, ri = 0;
    if (valid) { xi = x[tg]; yi = y[tg]; zi = z[tg]; ri = reach[tg]; }
    const double ri2 = ri * ri;
    const float xf = __double2float_rn(xi), yf = __double2float_rn(yi), zf = __double2float_rn(zi);
    const float rf = __double2float_ru(ri);
    // a row starts at off[slot] (exact counts known), or, with cap > 0, at
    // slot * cap in a padded layout whose rows keep at most cap entries (the
    // count is still taken in full: a longer row is rebuilt elsewhere)
    long long base = 0;
    if (FILL && valid) base = cap ? (long long)slot * cap : off[slot];
    long long cnt = 0;  // SOLO: the row length so far (uniform); else this lane's
    // does this lane's sphere reach box [l, u] holding h up to l.w?
    auto reaches = [&](const float4 &l, const float4 &u) -> bool {
        const float R = (SYM ? fmaxf(rf, l.w) : rf) + scr;
        const float gx = axis_gap_f(xf, l.x, u.x, boxf, scr);
        const float gy = axis_gap_f(yf, l.y, u.y, boxf, scr);
        const float gz = axis_gap_f(zf, l.z, u.z, boxf, scr);
        return valid && (gx * gx + gy * gy + gz * gz <= R * R * 1.00001f);
    };
    auto outward = [](const double4 &l, const double4 &u, float4 &fl, float4 &fu) {
        fl = make_float4(__double2float_rd(l.x), __double2float_rd(l.y), __double2float_rd(l.z), __double2float_ru(l.w));
        fu = make_float4(__double2float_ru(u.x), __double2float_ru(u.y), __double2float_ru(u.z), 0.0f);
    };
    // The tree is walked from its root; with box sets from each lane's box
    // subtree, one box at a time (the lanes of a group of consecutive targets
    // span one box or a few)
    const int my_root = (t.root_of && valid) ? t.root_of[t.box_of[tg]] : 0;
    unsigned roots_left = __ballot_sync(full, valid);
    int sp = 0;
    while (roots_left) {
    const int root = __shfl_sync(full, my_root, __ffs(roots_left) - 1);
    const bool in_root = valid && my_root == root;
    roots_left &= ~__ballot_sync(full, in_root);
    {
        float4 l, u;
        outward(t.lo[root], t.hi[root], l, u);
        const unsigned m = __ballot_sync(full, in_root && reaches(l, u));
        if (m) {
            if (lane == 0) {
                const int4 nd = t.node[root];
                s_stack[wib][0] = StackNode{nd.x, nd.y, nd.z, nd.w, m};
            }
            sp = 1;
        }
    }
    __syncwarp();
    while (sp > 0) {
        sp--;
        const StackNode e = s_stack[wib][sp];
        __syncwarp();
        const bool mine = (e.lanes >> lane) & 1u;
        if (e.child < 0) {
            // leaf: its particles, 32 at a time
            const int a = e.first, b = e.first + e.count;
            for (int c0 = a; c0 < b; c0 += 32) {
                const int jl = c0 + lane;
                if (SOLO) {
                    double cx = 0, cy = 0, cz = 0, hj = 0;
                    int sc = 0;
                    if (jl < b) {
                        cx = x[jl]; cy = y[jl]; cz = z[jl];
                        if (SYM) hj = hsym[jl];
                        const float dx = wrap1f(xf - __double2float_rn(cx), boxf, halff);
                        const float dy = wrap1f(yf - __double2float_rn(cy), boxf, halff);
                        const float dz = wrap1f(zf - __double2float_rn(cz), boxf, halff);
                        sc = screen(dx * dx + dy * dy + dz * dz, SYM ? fmaxf(rf, __double2float_ru(hj)) : rf, scr, SYM);
                    }
                    bool acc = sc == 1;
                    if (sc == 2) {
                        double dx, dy, dz;
                        const double r2 = sep2(xi, yi, zi, cx, cy, cz, box, half, dx, dy, dz);
                        acc = SYM ? ((r2 > 0) && !((r2 >= ri2) && (r2 >= __dmul_rn(hj, hj)))) : (r2 < ri2);
                    }
                    const unsigned bal = __ballot_sync(full, acc);
                    if (FILL && acc) {
                        const long long k = cnt + __popc(bal & ((1u << lane) - 1u));
                        if (!cap || k < cap) nbr[base + k] = jl;
                    }
                    cnt += __popc(bal);
                } else if (__popc(e.lanes) * 7 < min(32, b - c0) * 5) {
                    // few of the warp's targets reached this leaf: the lanes hold
                    // the candidates and the warp loops over the reaching targets
                    // (each target's row gets its hits in candidate order, as below)
                    double cx = 0, cy = 0, cz = 0, hj = 0;
                    float cxf = 0, cyf = 0, czf = 0, hjf = 0;
                    if (jl < b) {
                        cx = x[jl]; cy = y[jl]; cz = z[jl];
                        cxf = __double2float_rn(cx); cyf = __double2float_rn(cy); czf = __double2float_rn(cz);
                        if (SYM) { hj = hsym[jl]; hjf = __double2float_ru(hj); }
                    }
                    unsigned rem = e.lanes;
                    while (rem) {
                        const int tl = __ffs(rem) - 1;
                        rem &= rem - 1u;
                        const float txf = __shfl_sync(full, xf, tl), tyf = __shfl_sync(full, yf, tl);
                        const float tzf = __shfl_sync(full, zf, tl), trf = __shfl_sync(full, rf, tl);
                        int sc = 0;
                        if (jl < b) {
                            const float dx = wrap1f(txf - cxf, boxf, halff);
                            const float dy = wrap1f(tyf - cyf, boxf, halff);
                            const float dz = wrap1f(tzf - czf, boxf, halff);
                            sc = screen(dx * dx + dy * dy + dz * dz, SYM ? fmaxf(trf, hjf) : trf, scr, SYM);
                        }
                        bool acc = sc == 1;
                        if (__any_sync(full, sc == 2)) {
                            const double tx = __shfl_sync(full, xi, tl), ty = __shfl_sync(full, yi, tl);
                            const double tz = __shfl_sync(full, zi, tl), tr2 = __shfl_sync(full, ri2, tl);
                            if (sc == 2) {
                                double dx, dy, dz;
                                const double r2 = sep2(tx, ty, tz, cx, cy, cz, box, half, dx, dy, dz);
                                acc = SYM ? ((r2 > 0) && !((r2 >= tr2) && (r2 >= __dmul_rn(hj, hj)))) : (r2 < tr2);
                            }
                        }
                        const unsigned bal = __ballot_sync(full, acc);
                        if (FILL) {
                            const long long tc = __shfl_sync(full, cnt, tl);
                            const long long at = __shfl_sync(full, base, tl);
                            const long long k = tc + __popc(bal & ((1u << lane) - 1u));
                            if (acc && (!cap || k < cap)) nbr[at + k] = jl;
                        }
                        if (lane == tl) cnt += __popc(bal);
                    }
                } else {
                    if (jl < b) {
                        const double cx = x[jl], cy = y[jl], cz = z[jl], hj = SYM ? hsym[jl] : 0.0;
                        s_c[wib][lane] = make_double4(cx, cy, cz, hj);
                        s_cf[wib][lane] = make_float4(__double2float_rn(cx), __double2float_rn(cy), __double2float_rn(cz),
                                                      SYM ? __double2float_ru(hj) : 0.0f);
                    }
                    __syncwarp();
                    const int nk = min(32, b - c0);
                    if (mine) {
#pragma unroll 4
                        for (int k = 0; k < nk; k++) {
                            const float4 cf = s_cf[wib][k];
                            const float dx = wrap1f(xf - cf.x, boxf, halff);
                            const float dy = wrap1f(yf - cf.y, boxf, halff);
                            const float dz = wrap1f(zf - cf.z, boxf, halff);
                            const int sc = screen(dx * dx + dy * dy + dz * dz, SYM ? fmaxf(rf, cf.w) : rf, scr, SYM);
                            bool acc = sc == 1;
                            if (sc == 2) {
                                const double4 cj = s_c[wib][k];
                                double ddx, ddy, ddz;
                                const double r2 = sep2(xi, yi, zi, cj.x, cj.y, cj.z, box, half, ddx, ddy, ddz);
                                if (SYM) acc = (r2 > 0) && !((r2 >= ri2) && (r2 >= __dmul_rn(cj.w, cj.w)));
                                else acc = r2 < ri2;
                            }
                            if (acc) {
                                if (FILL && (!cap || cnt < cap)) nbr[base + cnt] = c0 + k;
                                cnt++;
                            }
                        }
                    }
                    __syncwarp();
                }
            }
            continue;
        }
        // open the node: its children's records in one access, tested here
        const int nc = e.nchild;
        if (lane < nc) {
            s_nd[wib][lane] = t.node[e.child + lane];
            float4 l, u;
            outward(t.lo[e.child + lane], t.hi[e.child + lane], l, u);
            s_lo[wib][lane] = l;
            s_hi[wib][lane] = u;
        }
        __syncwarp();
        unsigned need[8];
#pragma unroll
        for (int c = 0; c < 8; c++) need[c] = (c < nc) ? __ballot_sync(full, mine && reaches(s_lo[wib][c], s_hi[wib][c])) : 0u;
        int npush = 0;
#pragma unroll
        for (int c = 0; c < 8; c++) npush += need[c] != 0u;
        if (sp + npush > kStack) {
            if (lane == 0) record_status(st, 5 /* GZ_ERR_CAPACITY */, tg);
            break;
        }
        // push the reached children so that the first child is popped first
        if (lane == 0) {
            int pos = sp + npush - 1;
#pragma unroll
            for (int c = 0; c < 8; c++) {
                if (need[c]) {
                    const int4 nd = s_nd[wib][c];
                    s_stack[wib][pos--] = StackNode{nd.x, nd.y, nd.z, nd.w, need[c]};
                }
            }
        }
        sp += npush;
        __syncwarp();
    }
    if (sp > 0) break;  // the stack overflowed (recorded): no further box
    }  // the roots
    if (!FILL || cap) {
        if (SOLO) { if (lane == 0) counts[slot] = cnt; }
        else if (valid) counts[slot] = cnt;
    }
}

// Persistent form: every warp takes the next group (32 consecutive targets,
// or one target in SOLO mode) from a counter until none is left, so warps
// that draw a group on both sides of a Morton jump do not hold up a wave.
template <bool SYM, bool FILL, bool SOLO>
__device__ __forceinline__ void walk_groups(const Tree &t, const double *__restrict__ x, const double *__restrict__ y,
                                            const double *__restrict__ z, const double *__restrict__ reach,
                                            const double *__restrict__ hsym, const int *__restrict__ targets,
                                            int n_targets, long long *counts, const long long *__restrict__ off,
                                            int *nbr, int cap, DevStatus *st, int *next_group)
{
    __shared__ StackNode s_stack[kWarps][kStack];
    __shared__ double4 s_c[kWarps][32];
    __shared__ float4 s_cf[kWarps][32];
    __shared__ float4 s_lo[kWarps][8], s_hi[kWarps][8];
    __shared__ int4 s_nd[kWarps][8];
    const int lane = threadIdx.x & 31;
    const int n_groups = SOLO ? n_targets : (n_targets + 31) / 32;
    for (;;) {
        int g = 0;
        if (lane == 0) g = atomicAdd(next_group, 1);
        g = __shfl_sync(0xffffffffu, g, 0);
        if (g >= n_groups) break;
        walk_group<SYM, FILL, SOLO>(g, t, x, y, z, reach, hsym, targets, n_targets, counts, off, nbr, cap, st, s_stack,
                                    s_c, s_cf, s_lo, s_hi, s_nd);
        __syncwarp();
    }
}

template <bool SYM, bool FILL, bool SOLO>
__global__ void __launch_bounds__(256) k_walk(Tree t, const double *__restrict__ x, const double *__restrict__ y,
                                              const double *__restrict__ z, const double *__restrict__ reach,
                                              const double *__restrict__ hsym, const int *__restrict__ targets,
                                              int n_targets, long long *counts, const long long *__restrict__ off,
                                              int *nbr, int cap, DevStatus *st, int *next_group)
{
    walk_groups<SYM, FILL, SOLO>(t, x, y, z, reach, hsym, targets, n_targets, counts, off, nbr, cap, st, next_group);
}

// The padded density-row fill of a captured pass: the rows of this iteration
// (every target at iteration 0, the regrow list afterwards), their number,
// slots and place in the row buffer come from the device state; the instance
// of the state's walk mode runs (both modes write the same rows).
template <bool SOLO>
__global__ void __launch_bounds__(256) k_walk_graph(Tree t, const double *__restrict__ x, const double *__restrict__ y,
                                                    const double *__restrict__ z, const double *__restrict__ reach,
                                                    const int *__restrict__ first, const int *__restrict__ grow,
                                                    GraphState *gs, long long *counts, int *nbr, DevStatus *st)
{
    if (gs->fail || gs->walk_solo != (int)SOLO || gs->n_grow == 0) return;
    walk_groups<false, true, SOLO>(t, x, y, z, reach, reach, gs->iter == 0 ? first : grow, gs->n_grow, counts,
                                   nullptr, nbr + gs->base, gs->cap, st, &gs->next_group[0]);
}

// The rows longer than their slots, at their exact offsets behind the block.
__global__ void __launch_bounds__(256) k_walk_graph_over(Tree t, const double *__restrict__ x,
                                                         const double *__restrict__ y, const double *__restrict__ z,
                                                         const double *__restrict__ reach, const int *__restrict__ list,
                                                         const long long *__restrict__ off, GraphState *gs, int *nbr,
                                                         DevStatus *st)
{
    if (gs->fail || gs->n_over == 0) return;
    walk_groups<false, true, true>(t, x, y, z, reach, reach, list, gs->n_over, nullptr, off, nbr + gs->need, 0, st,
                                   &gs->next_group[1]);
}

// ------------------------------------------------ symmetric rows from density rows
// When the density pass covered every particle, each particle's density row
// holds every j with r < (row radius) >= its converged h, so the symmetric
// rows follow without another tree walk:
//   S_i = A_i u B_i,  A_i = {j : 0 < r2 < h_i^2},  B_i = {j : i in A_j, r2 >= h_i^2}
// (r2 is bitwise symmetric: the minimum image of -d is the negation of that of
// d), which is exactly the walk's predicate 0 < r2 and !(r2 >= h_i^2 and
// r2 >= h_j^2). The rows are sorted at the end, so they equal the walk's.

// Compacts density row i in place to A_i (order kept), marks an entry whose
// pair is one-sided (r2 >= h_j^2: i belongs in B_j) by storing ~j, and counts
// |A_i| and |B_j|.
// (eight 256-thread blocks per multiprocessor, at most 32 registers: the
// split waits on its position gathers, and full occupancy hides more of
// them; 25.8 vs 26.1 ms for the 256^3 gradients stage at six blocks)
template <int TPT>
__global__ void __launch_bounds__(256, 8) k_sym_split(int n, const double *__restrict__ x, const double *__restrict__ y,
                                                   const double *__restrict__ z, const double *__restrict__ h,
                                                   double box, const long long *__restrict__ beg,
                                                   const long long *__restrict__ end, int *nbr, int *acnt, int *bcnt)
{
    const int gtid = blockIdx.x * blockDim.x + threadIdx.x;
    const int i = gtid / TPT, lane = gtid % TPT;
    if (i >= n) return;
    const int gshift = (threadIdx.x & 31) & ~(TPT - 1);
    const unsigned mask = (TPT == 32) ? 0xffffffffu : (((1u << TPT) - 1u) << gshift);
    const double half = 0.5 * box;
    const double xi = x[i], yi = y[i], zi = z[i], hi = h[i];
    const double hi2 = __dmul_rn(hi, hi);
    const long long b0 = beg[i], b1 = end[i];
    long long wpos = b0;
    for (long long e0 = b0; e0 < b1; e0 += TPT) {
        const long long e = e0 + lane;
        int j = 0;
        bool in_a = false, one_sided = false;
        if (e < b1) {
            j = nbr[e];
            double dx, dy, dz;
            const double r2 = sep2(xi, yi, zi, x[j], y[j], z[j], box, half, dx, dy, dz);
            in_a = (r2 > 0) && (r2 < hi2);
            if (in_a) {
                const double hj = h[j];
                one_sided = !(r2 < __dmul_rn(hj, hj));
                if (one_sided) atomicAdd(bcnt + j, 1);
            }
        }
        const unsigned gb = (__ballot_sync(mask, in_a) >> gshift) & (TPT == 32 ? 0xffffffffu : ((1u << TPT) - 1u));
        __syncwarp(mask);  // every lane has read its entry before any is overwritten
        if (in_a) nbr[wpos + __popc(gb & ((1u << lane) - 1u))] = one_sided ? ~j : j;
        wpos += __popc(gb);
    }
    if (lane == 0) acnt[i] = (int)(wpos - b0);
}

__global__ void k_sym_counts(int n, const int *__restrict__ acnt, const int *__restrict__ bcnt, long long *cnt)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) cnt[i] = (long long)acnt[i] + bcnt[i];
}

// A_i into row i; each marked entry also puts i into row j's B part
template <int TPT>
__global__ void __launch_bounds__(256) k_sym_scatter(int n, const long long *__restrict__ beg,
                                                     const int *__restrict__ nbr, const int *__restrict__ acnt,
                                                     const long long *__restrict__ s_off, int *bcur, int *rows)
{
    const int gtid = blockIdx.x * blockDim.x + threadIdx.x;
    const int i = gtid / TPT, lane = gtid % TPT;
    if (i >= n) return;
    const long long b0 = beg[i], o = s_off[i];
    const int a = acnt[i];
    for (int k = lane; k < a; k += TPT) {
        const int v = nbr[b0 + k];
        const int j = v < 0 ? ~v : v;
        rows[o + k] = j;
        if (v < 0) rows[s_off[j] + acnt[j] + atomicAdd(bcur + j, 1)] = i;
    }
}

// Each row sorted ascending (its entries are distinct), TPT lanes per row. A
// row is A_i (the compacted density row: ascending, as the walk visits leaves
// and their particles in index order) followed by B_i (unordered, appended by
// the scatter). An A entry's rank is its index plus the B entries below it; a
// B entry's rank is the A entries below it (binary search) plus the B entries
// below it. A row whose A part is not ascending is ranked by comparing every
// pair.
template <int TPT>
__global__ void __launch_bounds__(256) k_sym_sort(int n, const long long *__restrict__ s_off,
                                                  const int *__restrict__ acnt, const int *__restrict__ rows, int *out)
{
    const int gtid = blockIdx.x * blockDim.x + threadIdx.x;
    const int i = gtid / TPT, lane = gtid % TPT;
    if (i >= n) return;  // the row's lanes leave together
    const unsigned mask = (TPT == 32) ? 0xffffffffu : (((1u << TPT) - 1u) << ((threadIdx.x & 31) & ~(TPT - 1)));
    const long long b0 = s_off[i], b1 = s_off[i + 1];
    const int len = (int)(b1 - b0), a = acnt[i];
    const int *r = rows + b0;
    bool asc = true;
    for (int k = lane + 1; k < a; k += TPT) asc &= r[k - 1] < r[k];
    asc = __all_sync(mask, asc);
    for (int k = lane; k < len; k += TPT) {
        const int v = r[k];
        int rank = 0;
        if (asc) {
            for (int m = a; m < len; m++) rank += r[m] < v;
            if (k < a) {
                rank += k;
            } else {
                int lo = 0, hi = a;
                while (lo < hi) {
                    const int mid = (lo + hi) >> 1;
                    if (r[mid] < v) lo = mid + 1; else hi = mid;
                }
                rank += lo;
            }
        } else {
            for (int m = 0; m < len; m++) rank += r[m] < v;
        }
        out[b0 + rank] = v;
    }
}

void sym_split(int n, const double *x, const double *y, const double *z, const double *h, double box,
               const long long *beg, const long long *end, int *nbr, int *acnt, int *bcnt, cudaStream_t s)
{
    if (n > 0) k_sym_split<8><<<(unsigned)(((long long)n * 8 + 255) / 256), 256, 0, s>>>(n, x, y, z, h, box, beg, end, nbr, acnt, bcnt);
}

void sym_counts(int n, const int *acnt, const int *bcnt, long long *cnt, cudaStream_t s)
{
    if (n > 0) k_sym_counts<<<(n + 255) / 256, 256, 0, s>>>(n, acnt, bcnt, cnt);
}

void sym_scatter(int n, const long long *beg, const int *nbr, const int *acnt, const long long *s_off, int *bcur,
                 int *rows, cudaStream_t s)
{
    if (n > 0) k_sym_scatter<8><<<(unsigned)(((long long)n * 8 + 255) / 256), 256, 0, s>>>(n, beg, nbr, acnt, s_off, bcur, rows);
}

void sym_sort(int n, const long long *s_off, const int *acnt, const int *rows, int *out, cudaStream_t s)
{
    if (n > 0) k_sym_sort<8><<<(unsigned)(((long long)n * 8 + 255) / 256), 256, 0, s>>>(n, s_off, acnt, rows, out);
}

// After a padded fill: a row that fit its cap slots gets [slot*cap, +count);
// a longer one is flagged for a rebuild.
__global__ void k_padded_rows(int na, const int *__restrict__ t, const long long *__restrict__ counts, int cap,
                              long long base, long long *beg, long long *end, unsigned char *over)
{
    const int a = blockIdx.x * blockDim.x + threadIdx.x;
    if (a >= na) return;
    const long long c = counts[a];
    over[a] = c > cap;
    if (c <= cap) {
        beg[t[a]] = base + (long long)a * cap;
        end[t[a]] = base + (long long)a * cap + c;
    }
}

void padded_rows(int na, const int *t, const long long *counts, int cap, long long base, long long *beg,
                 long long *end, unsigned char *over, cudaStream_t s)
{
    if (na > 0) k_padded_rows<<<(na + 255) / 256, 256, 0, s>>>(na, t, counts, cap, base, beg, end, over);
}

void grid_keys(int n, const double *pos, double box, const int *bid, int axis_bits, unsigned long long *keys, int *idx,
               cudaStream_t s)
{
    if (n > 0) k_keys<<<(n + 255) / 256, 256, 0, s>>>(n, pos, box, bid, axis_bits, keys, idx);
}

void tree_count(const unsigned long long *keys, int L, const int4 *node, int beg, int cnt, long long *nch,
                int leaf_max, int split_levels, cudaStream_t s)
{
    if (cnt > 0) k_tree_count<<<(cnt + 127) / 128, 128, 0, s>>>(keys, L, node, beg, cnt, nch, leaf_max, split_levels);
}

void box_roots(int beg, int cnt, const int4 *node, const int *box_of, int *root_of, cudaStream_t s)
{
    if (cnt > 0) k_box_roots<<<(cnt + 127) / 128, 128, 0, s>>>(beg, cnt, node, box_of, root_of);
}

void tree_write(const unsigned long long *keys, int L, int4 *node, int *parent, int beg, int cnt,
                const long long *cpos, int next, cudaStream_t s)
{
    if (cnt > 0) k_tree_write<<<(cnt + 127) / 128, 128, 0, s>>>(keys, L, node, parent, beg, cnt, cpos, next);
}

void tree_up(int n_nodes, const int4 *node, const int *parent, const double *x, const double *y, const double *z,
             const double *h, double4 *lo, double4 *hi, int *done, int boxes, cudaStream_t s, const int *n_nodes_dev)
{
    if (n_nodes <= 0) return;
    cudaMemsetAsync(done, 0, sizeof(int) * (size_t)n_nodes, s);
    k_tree_up<<<(n_nodes + 127) / 128, 128, 0, s>>>(n_nodes, n_nodes_dev, node, parent, x, y, z, h, lo, hi, done,
                                                     boxes);
}

void tree_build_device(const unsigned long long *keys, int n, int4 *node, int *parent, TreeBuild *tb, int cap,
                       int leaf_max, int split_levels, const int *box_of, int *root_of, int blocks, cudaStream_t s)
{
    k_tree_init<<<1, 1, 0, s>>>(tb, node, parent, n);
    for (int L = 0; L <= kBits; L++) {
        k_tree_level<<<blocks, 128, 0, s>>>(keys, node, parent, tb, cap, leaf_max, split_levels, box_of, root_of);
        k_tree_next<<<1, 1, 0, s>>>(tb);
    }
}

template <bool SYM, bool FILL, bool SOLO>
static void launch_walk(const Tree &t, const double *x, const double *y, const double *z, const double *reach,
                        const double *hsym, const int *targets, int n_targets, long long *counts, const long long *off,
                        int *nbr, int cap, DevStatus *st, int *next_group, cudaStream_t s)
{
    // blocks of this instance resident on the current device (multiprocessors
    // x blocks per multiprocessor), looked up once per device; concurrent
    // first calls store the same value
    static std::atomic<int> resident_of[kMaxWalkDevices];
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 0 || dev >= kMaxWalkDevices) dev = 0;
    int resident = resident_of[dev].load(std::memory_order_relaxed);
    if (resident == 0) {
        int sms = 0, per_sm = 0;
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_walk<SYM, FILL, SOLO>, 32 * kWarps, 0);
        resident = (sms > 0 ? sms : 148) * (per_sm > 0 ? per_sm : 1);
        resident_of[dev].store(resident, std::memory_order_relaxed);
    }
    const long long groups = SOLO ? n_targets : (n_targets + 31) / 32;
    const long long need = (groups + kWarps - 1) / kWarps;
    const unsigned blocks = (unsigned)(need < resident ? need : resident);
    cudaMemsetAsync(next_group, 0, sizeof(int), s);
    k_walk<SYM, FILL, SOLO><<<blocks, 32 * kWarps, 0, s>>>(t, x, y, z, reach, hsym, targets, n_targets, counts, off,
                                                            nbr, cap, st, next_group);
}

// Warps the group-mode walk holds resident on the current device (looked up
// once per device; concurrent first calls store the same value).
long long walk_group_warps()
{
    static std::atomic<long long> group_warps_of[kMaxWalkDevices];
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 0 || dev >= kMaxWalkDevices) dev = 0;
    long long group_warps = group_warps_of[dev].load(std::memory_order_relaxed);
    if (group_warps == 0) {
        int sms = 0, per_sm = 0;
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_walk<false, true, false>, 32 * kWarps, 0);
        group_warps = (long long)(sms > 0 ? sms : 148) * (per_sm > 0 ? per_sm : 1) * kWarps;
        group_warps_of[dev].store(group_warps, std::memory_order_relaxed);
    }
    return group_warps;
}

void walk_rows(const Tree &t, const double *x, const double *y, const double *z, const double *reach,
               const double *hsym, int symmetric, const int *targets, int n_targets, long long *counts,
               const long long *off, int *nbr, int cap, DevStatus *st, int *next_group, cudaStream_t s)
{
    if (n_targets <= 0) return;
    // Group mode (32 targets per warp) for dense lists and for lists whose
    // groups fill the warps the GPU holds resident: its traversal tests 32
    // targets per ballot where the one-target mode tests one. A short sparse
    // list (the rows rebuilt after an h regrowth, scattered through the box)
    // gets one warp per target instead: as groups it would run on a few
    // warps, each walking 32 unrelated regions one after another.
    const long long group_warps = walk_group_warps();
    const bool sparse = (long long)n_targets * 4 < (long long)t.n_particles;
    const bool solo = n_targets == 1 || (sparse && (n_targets + 31) / 32 < group_warps);
#define GZ_WALK(S, F, O) launch_walk<S, F, O>(t, x, y, z, reach, hsym, targets, n_targets, counts, off, nbr, cap, st, next_group, s)
    if (symmetric) {
        if (solo) { if (nbr) GZ_WALK(true, true, true); else GZ_WALK(true, false, true); }
        else { if (nbr) GZ_WALK(true, true, false); else GZ_WALK(true, false, false); }
    } else {
        if (solo) { if (nbr) GZ_WALK(false, true, true); else GZ_WALK(false, false, true); }
        else { if (nbr) GZ_WALK(false, true, false); else GZ_WALK(false, false, false); }
    }
#undef GZ_WALK
}

void walk_rows_graph(const Tree &t, const double *x, const double *y, const double *z, const double *reach,
                     const int *first, const int *grow, GraphState *gs, long long *counts, int *nbr, DevStatus *st,
                     cudaStream_t s)
{
    static std::atomic<int> resident_of[kMaxWalkDevices][2];
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 0 || dev >= kMaxWalkDevices) dev = 0;
    int res[2];
    for (int m = 0; m < 2; m++) {
        res[m] = resident_of[dev][m].load(std::memory_order_relaxed);
        if (res[m] == 0) {
            int sms = 0, per_sm = 0;
            cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
            if (m == 0) cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_walk_graph<false>, 32 * kWarps, 0);
            else cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_walk_graph<true>, 32 * kWarps, 0);
            res[m] = (sms > 0 ? sms : 148) * (per_sm > 0 ? per_sm : 1);
            resident_of[dev][m].store(res[m], std::memory_order_relaxed);
        }
    }
    k_walk_graph<false><<<res[0], 32 * kWarps, 0, s>>>(t, x, y, z, reach, first, grow, gs, counts, nbr, st);
    k_walk_graph<true><<<res[1], 32 * kWarps, 0, s>>>(t, x, y, z, reach, first, grow, gs, counts, nbr, st);
}

void walk_over_graph(const Tree &t, const double *x, const double *y, const double *z, const double *reach,
                     const int *list, const long long *off, GraphState *gs, int *nbr, DevStatus *st, int blocks,
                     cudaStream_t s)
{
    k_walk_graph_over<<<blocks, 32 * kWarps, 0, s>>>(t, x, y, z, reach, list, off, gs, nbr, st);
}

}  // namespace gz

// gizmo_b200/csrc/grid.cu -- Morton neighbour grid and exact neighbour rows.
//
// Replaces the reference's SIDX spatial index + BVH walk + two-pass CSR
// (src/mesh/gpu_neighbor_list.cc:1134-1169, 1736-1816;
// src/mesh/gpu_neighbor_list.h:207-264). Particles are sorted by a 63-bit
// Morton key (21 bits per axis), which makes an implicit octree of 21 levels
// in which every node is one contiguous run of the sorted arrays. The top D
// levels have a dense table of node starts and node maxima of h; a deeper
// node's children are found by binary search inside the parent's run, so a
// 1e5 density contrast costs a few extra levels, not a finer table. Maxima
// of h below level D come from per-32-particle block maxima.
//
// Neighbour rows are produced by a warp-cooperative walk: one warp takes 32
// consecutive sorted targets, descends the octree once for the whole group
// (a node survives when any lane's search sphere reaches it), and streams
// each surviving leaf through the warp 32 candidates at a time, every lane
// testing its own target. Membership uses the reference
// predicates on FP64 minimum-image separations rounded exactly as the CPU
// does, so the rows are bit-identical to an exact CPU search:
//   one-way   r2 < R_i^2                                (density, R = buffered h)
//   symmetric r2 > 0 and !(r2 >= h_i^2 and r2 >= h_j^2) (gradients, force)
#include <cub/cub.cuh>

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

GZ_DEV unsigned long long compact21(unsigned long long x)
{
    x &= 0x1249249249249249ull;
    x = (x | (x >> 2)) & 0x10c30c30c30c30c3ull;
    x = (x | (x >> 4)) & 0x100f00f00f00f00full;
    x = (x | (x >> 8)) & 0x1f0000ff0000ffull;
    x = (x | (x >> 16)) & 0x1f00000000ffffull;
    x = (x | (x >> 32)) & 0x1fffffull;
    return x;
}

__global__ void k_keys(int n, const double *__restrict__ pos, double box, unsigned long long *keys, int *idx)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const long long G = 1ll << kBits;
    unsigned long long c[3];
    for (int k = 0; k < 3; k++) {
        long long v = (long long)(pos[3 * (size_t)i + k] / box * (double)G);
        v = v < 0 ? 0 : (v >= G ? G - 1 : v);
        c[k] = (unsigned long long)v;
    }
    keys[i] = spread21(c[0]) | (spread21(c[1]) << 1) | (spread21(c[2]) << 2);
    idx[i] = i;
}

// first sorted position of every level-D node (lower bound of the key prefixes)
__global__ void k_cell_start(int n, const unsigned long long *__restrict__ skeys, int shift, long long ncell, int *start)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const long long k = (long long)(skeys[i] >> shift);
    const long long kp = (i == 0) ? -1 : (long long)(skeys[i - 1] >> shift);
    for (long long c = kp + 1; c <= k; c++) start[c] = i;
    if (i == n - 1)
        for (long long c = k + 1; c <= ncell; c++) start[c] = n;
}

__global__ void k_fill_int(long long count, int *p, int v)
{
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i < count) p[i] = v;
}

__global__ void k_hmax_fine(int n, const unsigned long long *__restrict__ skeys, int shift, const double *__restrict__ h,
                            unsigned long long *hmax_fine)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double hv = h[i] > 0 ? h[i] : 0.0;  // non-negative doubles order as their bit patterns
    atomicMax(hmax_fine + (skeys[i] >> shift), (unsigned long long)__double_as_longlong(hv));
}

__global__ void k_hmax_level(long long nodes, const double *__restrict__ child, double *parent)
{
    const long long m = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (m >= nodes) return;
    double v = 0;
    for (int k = 0; k < 8; k++) v = fmax(v, child[8 * m + k]);
    parent[m] = v;
}

__global__ void k_block_max(int n, const double *__restrict__ h, double *bmax)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const double v = (i < n && h[i] > 0) ? h[i] : 0.0;
    const double m = warp_max(v, 0xffffffffu, 32);
    if ((threadIdx.x & 31) == 0 && i < n) bmax[i >> 5] = m;
}

// periodic gap between a node interval [o, o+s) and a point on one axis
GZ_DEV double point_gap(double x, double o, double s, double box)
{
    double d = fabs(x - (o + 0.5 * s));
    if (d > 0.5 * box) d = box - d;
    d -= 0.5 * s;
    return d > 0 ? d : 0;
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

constexpr int kStack = 176;
constexpr int kLeaf = 32;

// Warp-cooperative octree walk. FILL=false counts rows; FILL=true writes them.
// A node is descended when the search sphere of at least one lane reaches
// it (each lane tests its own target against the node box), so 32 targets
// that straddle a jump of the Morton curve cost two small searches, not one
// search of their joint bounding box. Leaf candidates are staged in shared
// memory and read back by every lane as broadcasts.
template <bool SYM, bool FILL>
__global__ void __launch_bounds__(256) k_walk(Grid g, const double *__restrict__ x, const double *__restrict__ y,
                                              const double *__restrict__ z, const double *__restrict__ reach,
                                              const double *__restrict__ hsym, const int *__restrict__ targets,
                                              int n_targets, int *counts, const long long *__restrict__ off,
                                              int *nbr, DevStatus *st)
{
    __shared__ unsigned long long s_m[8][kStack];
    __shared__ int2 s_ab[8][kStack];
    __shared__ unsigned char s_L[8][kStack];
    __shared__ double4 s_c[8][32];
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    const int group = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int slot = group * 32 + lane;
    if (group * 32 >= n_targets) return;
    const bool valid = slot < n_targets;
    const int t = valid ? targets[slot] : -1;
    const double box = g.box, half = 0.5 * box;
    double xi = 0, yi = 0, zi = 0, ri = 0;
    if (valid) { xi = x[t]; yi = y[t]; zi = z[t]; ri = reach[t]; }
    const unsigned full = 0xffffffffu;
    const double ri2 = ri * ri;
    long long base = 0;
    if (FILL && valid) base = off[slot];
    int cnt = 0;
    if (lane == 0) { s_m[wib][0] = 0ull; s_ab[wib][0] = make_int2(0, g.n); s_L[wib][0] = 0; }
    int sp = 1;
    __syncwarp();
    const int D = g.D;
    while (sp > 0) {
        sp--;
        const unsigned long long m = s_m[wib][sp];
        const int2 ab = s_ab[wib][sp];
        const int L = s_L[wib][sp];
        __syncwarp();
        const int a = ab.x, b = ab.y;
        double R = ri;
        if (SYM) {
            double hn;
            if (L <= D) {
                hn = g.hmax[g.level_off[L] + (long long)m];
            } else {
                double v = 0;
                for (int blk = (a >> 5) + lane; blk <= ((b - 1) >> 5); blk += 32) v = fmax(v, g.bmax[blk]);
                hn = warp_max(v, full, 32);
            }
            R = fmax(R, hn);
        }
        const double s = box / (double)(1ll << L);
        const double gx = point_gap(xi, (double)compact21(m) * s, s, box);
        const double gy = point_gap(yi, (double)compact21(m >> 1) * s, s, box);
        const double gz = point_gap(zi, (double)compact21(m >> 2) * s, s, box);
        const bool need = valid && (gx * gx + gy * gy + gz * gz <= R * R * (1.0 + 1e-9) + 1e-300);
        if (!__any_sync(full, need)) continue;
        if (L == kBits || b - a <= kLeaf) {
            for (int c0 = a; c0 < b; c0 += 32) {
                const int jl = c0 + lane;
                if (jl < b) s_c[wib][lane] = make_double4(x[jl], y[jl], z[jl], SYM ? hsym[jl] : 0.0);
                __syncwarp();
                const int nk = min(32, b - c0);
                if (need) {
                    for (int k = 0; k < nk; k++) {
                        const double4 cj = s_c[wib][k];
                        double dx, dy, dz;
                        const double r2 = sep2(xi, yi, zi, cj.x, cj.y, cj.z, box, half, dx, dy, dz);
                        bool acc;
                        if (SYM) acc = (r2 > 0) && !((r2 >= ri2) && (r2 >= __dmul_rn(cj.w, cj.w)));
                        else acc = r2 < ri2;
                        if (acc) {
                            if (FILL) nbr[base + cnt] = c0 + k;
                            cnt++;
                        }
                    }
                }
                __syncwarp();
            }
            continue;
        }
        // expand into the 8 children (level L+1): ranges from the dense table
        // above level D, by binary search inside [a, b) below it
        if (sp + 8 > kStack) {
            if (lane == 0) record_status(st, 5 /* GZ_ERR_CAPACITY */, t);
            break;
        }
        const unsigned long long child = 8ull * m + (unsigned long long)(lane & 7);
        int ca, cb;
        if (L + 1 <= D) {
            const int sh = 3 * (D - L - 1);
            ca = g.cell_start[child << sh];
            cb = g.cell_start[(child + 1) << sh];
        } else {
            const int sh = 3 * (kBits - L - 1);
            int lo = a;
            if (lane < 8 && (lane & 7) != 0) lo = lower_bound_key(g.keys, a, b, child << sh);
            ca = (lane & 7) == 0 ? a : lo;
            const int nxt = __shfl_down_sync(full, ca, 1);
            cb = ((lane & 7) == 7) ? b : nxt;
        }
        const unsigned nonempty = __ballot_sync(full, lane < 8 && cb > ca);
        const int npush = __popc(nonempty);
        // push the non-empty children so that child 0 is popped first
        if (lane < 8 && cb > ca) {
            const int pos = sp + __popc(nonempty >> (lane + 1));
            s_m[wib][pos] = child;
            s_ab[wib][pos] = make_int2(ca, cb);
            s_L[wib][pos] = (unsigned char)(L + 1);
        }
        sp += npush;
        __syncwarp();
    }
    if (!FILL && valid) counts[slot] = cnt;
}

void grid_keys(int n, const double *pos, double box, unsigned long long *keys, int *idx, cudaStream_t s)
{
    if (n > 0) k_keys<<<(n + 255) / 256, 256, 0, s>>>(n, pos, box, keys, idx);
}

void grid_cell_start(int n, const unsigned long long *skeys, int D, int *start, cudaStream_t s)
{
    const long long ncell = 1ll << (3 * D);
    if (n == 0) {
        k_fill_int<<<(unsigned)((ncell + 1 + 255) / 256), 256, 0, s>>>(ncell + 1, start, 0);
        return;
    }
    k_cell_start<<<(n + 255) / 256, 256, 0, s>>>(n, skeys, 3 * (kBits - D), ncell, start);
}

int grid_hmax(int n, const unsigned long long *skeys, const double *h, int D, double *hmax, const long long *level_off,
              double *bmax, cudaStream_t s)
{
    double *fine = hmax + level_off[D];
    const long long ncell = 1ll << (3 * D);
    cudaMemsetAsync(fine, 0, sizeof(double) * (size_t)ncell, s);
    int launches = 0;
    if (n > 0) {
        k_hmax_fine<<<(n + 255) / 256, 256, 0, s>>>(n, skeys, 3 * (kBits - D), h, (unsigned long long *)fine);
        k_block_max<<<(n + 255) / 256, 256, 0, s>>>(n, h, bmax);
        launches += 2;
    }
    for (int L = D - 1; L >= 0; L--) {
        const long long nodes = 1ll << (3 * L);
        k_hmax_level<<<(unsigned)((nodes + 255) / 256), 256, 0, s>>>(nodes, hmax + level_off[L + 1], hmax + level_off[L]);
        launches++;
    }
    return launches;
}

void walk_rows(const Grid &g, const double *x, const double *y, const double *z, const double *reach,
               const double *hsym, int symmetric, const int *targets, int n_targets, int *counts,
               const long long *off, int *nbr, DevStatus *st, cudaStream_t s)
{
    if (n_targets <= 0) return;
    const int warps = (n_targets + 31) / 32;
    const int blocks = (warps + 7) / 8;
    if (symmetric) {
        if (nbr) k_walk<true, true><<<blocks, 256, 0, s>>>(g, x, y, z, reach, hsym, targets, n_targets, counts, off, nbr, st);
        else k_walk<true, false><<<blocks, 256, 0, s>>>(g, x, y, z, reach, hsym, targets, n_targets, counts, off, nbr, st);
    } else {
        if (nbr) k_walk<false, true><<<blocks, 256, 0, s>>>(g, x, y, z, reach, hsym, targets, n_targets, counts, off, nbr, st);
        else k_walk<false, false><<<blocks, 256, 0, s>>>(g, x, y, z, reach, hsym, targets, n_targets, counts, off, nbr, st);
    }
}

}  // namespace gz

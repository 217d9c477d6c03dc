// gizmo_b200/csrc/grid.cu -- Morton neighbour grid and exact neighbour rows.
//
// Replaces the reference's SIDX spatial index + BVH walk + two-pass CSR
// (src/mesh/gpu_neighbor_list.cc:1134-1169, 1736-1816;
// src/mesh/gpu_neighbor_list.h:207-264). Particles are sorted by the Morton
// key of their fine cell (radix sort), giving an octree pyramid in which
// every node is one contiguous run of the sorted arrays. Neighbour rows are
// produced by a warp-cooperative walk: one warp takes 32 consecutive sorted
// targets, descends the pyramid once for the whole group (pruning nodes by
// periodic box distance against the group's bounding box), and streams each
// surviving leaf through the warp 32 candidates at a time with shuffles,
// every lane testing its own target. Membership uses the reference
// predicates on FP64 minimum-image separations rounded exactly as the CPU
// does, so the rows are bit-identical to an exact CPU search:
//   one-way   r2 < R_i^2                                (density, R = buffered h)
//   symmetric r2 > 0 and !(r2 >= h_i^2 and r2 >= h_j^2) (gradients, force)
#include <cub/cub.cuh>

#include "launch.h"

namespace gz {

__global__ void k_keys(int n, const double *__restrict__ pos, double box, int F, uint32_t *keys, int *idx)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int G = 1 << F;
    uint32_t c[3];
    for (int k = 0; k < 3; k++) {
        int v = (int)(pos[3 * (size_t)i + k] / box * (double)G);
        v = v < 0 ? 0 : (v >= G ? G - 1 : v);
        c[k] = (uint32_t)v;
    }
    keys[i] = spread3(c[0]) | (spread3(c[1]) << 1) | (spread3(c[2]) << 2);
    idx[i] = i;
}

// first sorted position of every fine cell (lower bound of the sorted keys)
__global__ void k_cell_start(int n, const uint32_t *__restrict__ skeys, uint32_t ncell, int *start)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const long long k = skeys[i];
    const long long kp = (i == 0) ? -1 : (long long)skeys[i - 1];
    for (long long c = kp + 1; c <= k; c++) start[c] = i;
    if (i == n - 1)
        for (long long c = k + 1; c <= (long long)ncell; c++) start[c] = n;
}

__global__ void k_fill_int(long long count, int *p, int v)
{
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i < count) p[i] = v;
}

__global__ void k_hmax_fine(int n, const uint32_t *__restrict__ skeys, const double *__restrict__ h,
                            unsigned long long *hmax_fine)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double hv = h[i] > 0 ? h[i] : 0.0;  // non-negative doubles order as their bit patterns
    atomicMax(hmax_fine + skeys[i], (unsigned long long)__double_as_longlong(hv));
}

__global__ void k_hmax_level(long long nodes, const double *__restrict__ child, double *parent)
{
    const long long m = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (m >= nodes) return;
    double v = 0;
    for (int k = 0; k < 8; k++) v = fmax(v, child[8 * m + k]);
    parent[m] = v;
}

// periodic gap between a node interval [o, o+s) and the group extent [lo, hi] on one axis
GZ_DEV double axis_gap(double o, double s, double lo, double hi, double box)
{
    double d = fabs((o + 0.5 * s) - 0.5 * (lo + hi));
    if (d > 0.5 * box) d = box - d;
    d -= 0.5 * s + 0.5 * (hi - lo);
    return d > 0 ? d : 0;
}

constexpr int kStack = 160;

// Warp-cooperative pyramid walk. FILL=false counts rows; FILL=true writes them.
template <bool SYM, bool FILL>
__global__ void __launch_bounds__(256) k_walk(Grid g, const double *__restrict__ x, const double *__restrict__ y,
                                              const double *__restrict__ z, const double *__restrict__ reach,
                                              const double *__restrict__ hsym, const int *__restrict__ targets,
                                              int n_targets, int *counts, const long long *__restrict__ off,
                                              int *nbr, DevStatus *st)
{
    __shared__ unsigned long long stack_all[8][kStack];
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    unsigned long long *stack = stack_all[wib];
    const int group = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int slot = group * 32 + lane;
    if (group * 32 >= n_targets) return;
    const bool valid = slot < n_targets;
    const int t = valid ? targets[slot] : -1;
    const double box = g.box, half = 0.5 * box;
    double xi = 0, yi = 0, zi = 0, ri = 0;
    if (valid) { xi = x[t]; yi = y[t]; zi = z[t]; ri = reach[t]; }
    const unsigned full = 0xffffffffu;
    const double lox = warp_min(valid ? xi : 1e300, full, 32), hix = warp_max(valid ? xi : -1e300, full, 32);
    const double loy = warp_min(valid ? yi : 1e300, full, 32), hiy = warp_max(valid ? yi : -1e300, full, 32);
    const double loz = warp_min(valid ? zi : 1e300, full, 32), hiz = warp_max(valid ? zi : -1e300, full, 32);
    const double Rg = warp_max(valid ? ri : 0.0, full, 32);
    const double ri2 = ri * ri;
    long long base = 0;
    if (FILL && valid) base = off[slot];
    int cnt = 0;
    if (lane == 0) stack[0] = 0ull;
    int sp = 1;
    __syncwarp();
    const int F = g.F;
    while (sp > 0) {
        sp--;
        const unsigned long long node = stack[sp];
        __syncwarp();
        const int L = (int)(node >> 32);
        const uint32_t m = (uint32_t)node;
        const int sh = 3 * (F - L);
        const int a = g.cell_start[(size_t)m << sh];
        const int b = g.cell_start[(size_t)(m + 1) << sh];
        if (a == b) continue;
        double R = Rg;
        if (SYM) R = fmax(R, g.hmax[g.level_off[L] + m]);
        const double s = box / (double)(1 << L);
        const double gx = axis_gap((double)compact3(m) * s, s, lox, hix, box);
        const double gy = axis_gap((double)compact3(m >> 1) * s, s, loy, hiy, box);
        const double gz = axis_gap((double)compact3(m >> 2) * s, s, loz, hiz, box);
        if (gx * gx + gy * gy + gz * gz > R * R * (1.0 + 1e-9) + 1e-300) continue;
        if (L == F || b - a <= 32) {
            for (int c0 = a; c0 < b; c0 += 32) {
                const int jl = c0 + lane;
                double xj = 0, yj = 0, zj = 0, hj = 0;
                if (jl < b) { xj = x[jl]; yj = y[jl]; zj = z[jl]; if (SYM) hj = hsym[jl]; }
                const int nk = min(32, b - c0);
                for (int k = 0; k < nk; k++) {
                    const double xk = __shfl_sync(full, xj, k), yk = __shfl_sync(full, yj, k), zk = __shfl_sync(full, zj, k);
                    double hk = 0;
                    if (SYM) hk = __shfl_sync(full, hj, k);
                    if (!valid) continue;
                    double dx, dy, dz;
                    const double r2 = sep2(xi, yi, zi, xk, yk, zk, box, half, dx, dy, dz);
                    bool acc;
                    if (SYM) acc = (r2 > 0) && !((r2 >= ri2) && (r2 >= __dmul_rn(hk, hk)));
                    else acc = r2 < ri2;
                    if (acc) {
                        if (FILL) nbr[base + cnt] = c0 + k;
                        cnt++;
                    }
                }
            }
        } else {
            if (sp + 8 > kStack) {
                if (lane == 0) record_status(st, 5 /* GZ_ERR_CAPACITY */, t);
                break;
            }
            if (lane < 8) stack[sp + lane] = ((unsigned long long)(L + 1) << 32) | (unsigned long long)(8u * m + (7 - lane));
            sp += 8;
            __syncwarp();
        }
    }
    if (!FILL && valid) counts[slot] = cnt;
}

void grid_keys(int n, const double *pos, double box, int F, uint32_t *keys, int *idx, cudaStream_t s)
{
    if (n > 0) k_keys<<<(n + 255) / 256, 256, 0, s>>>(n, pos, box, F, keys, idx);
}

void grid_cell_start(int n, const uint32_t *skeys, int F, int *start, cudaStream_t s)
{
    const long long ncell = 1ll << (3 * F);
    if (n == 0) {
        k_fill_int<<<(unsigned)((ncell + 1 + 255) / 256), 256, 0, s>>>(ncell + 1, start, 0);
        return;
    }
    k_cell_start<<<(n + 255) / 256, 256, 0, s>>>(n, skeys, (uint32_t)ncell, start);
}

void grid_hmax(int n, const uint32_t *skeys, const double *h, int F, double *hmax, const long long *level_off,
               cudaStream_t s)
{
    double *fine = hmax + level_off[F];
    const long long ncell = 1ll << (3 * F);
    cudaMemsetAsync(fine, 0, sizeof(double) * (size_t)ncell, s);
    if (n > 0) k_hmax_fine<<<(n + 255) / 256, 256, 0, s>>>(n, skeys, h, (unsigned long long *)fine);
    for (int L = F - 1; L >= 0; L--) {
        const long long nodes = 1ll << (3 * L);
        k_hmax_level<<<(unsigned)((nodes + 255) / 256), 256, 0, s>>>(nodes, hmax + level_off[L + 1], hmax + level_off[L]);
    }
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

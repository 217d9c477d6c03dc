// gizmo_b200/csrc/common.cuh -- shared device helpers for the B200 hydro pass.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#define GZ_DEV __device__ __forceinline__
// pair and per-particle math: callable from host code too (CPU emulation in tests)
#define GZ_HD __host__ __device__ __forceinline__

namespace gz {

constexpr double kMinReal = 1e-56;          // MIN_REAL_NUMBER, constants.h:220
constexpr double kCnDanger = 1.0e3;         // CONDITION_NUMBER_DANGER, constants.h:225
constexpr int kMaxIter = 150;               // MAXITER, constants.h:340
constexpr double kVolNorm = 4.188790204786; // VOLUME_NORM_COEFF_FOR_NDIMS (3-D), constants.h:445
constexpr int kWarp = 32;

// Device status word: the first recorded error wins; device code never traps.
struct DevStatus {
    int code;
    int index;  // sorted particle index, -1 if none
};

GZ_DEV void record_status(DevStatus *st, int code, int index)
{
    if (atomicCAS(&st->code, 0, code) == 0) st->index = index;
}

// Squared periodic minimum-image separation with the reference's operation
// order (NEAREST_XYZ, declarations/macros.h:58-109; Vec3::norm_sq,
// math_types/vec3.h:32). Explicit round-to-nearest intrinsics keep the
// membership test bit-identical to the CPU whatever the contraction flags.
GZ_DEV double wrap1(double x, double box, double half)
{
    return (x > half) ? __dsub_rn(x, box) : ((x < -half) ? __dadd_rn(x, box) : x);
}

GZ_DEV double sep2(double xi, double yi, double zi, double xj, double yj, double zj, double box, double half,
                   double &dx, double &dy, double &dz)
{
    dx = wrap1(__dsub_rn(xi, xj), box, half);
    dy = wrap1(__dsub_rn(yi, yj), box, half);
    dz = wrap1(__dsub_rn(zi, zj), box, half);
    return __dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(dz, dz));
}

GZ_DEV uint32_t spread3(uint32_t x)
{
    x &= 0x3ff;
    x = (x | (x << 16)) & 0x030000ff;
    x = (x | (x << 8)) & 0x0300f00f;
    x = (x | (x << 4)) & 0x030c30c3;
    x = (x | (x << 2)) & 0x09249249;
    return x;
}

GZ_DEV uint32_t compact3(uint32_t x)
{
    x &= 0x09249249;
    x = (x | (x >> 2)) & 0x030c30c3;
    x = (x | (x >> 4)) & 0x0300f00f;
    x = (x | (x >> 8)) & 0x030000ff;
    x = (x | (x >> 16)) & 0x000003ff;
    return x;
}

// Raises *slot (non-negative doubles as their bit patterns, which order like
// the values) to the largest v of the warp; every lane of the warp calls it,
// at one call site (a lane with nothing to report passes 0). One lane reads
// the slot and takes the atomic only when the warp's maximum is larger, so a
// launch of millions of threads costs a few atomics, not millions on one
// address.
GZ_DEV void warp_atomic_max_nonneg(unsigned long long *slot, double v)
{
    unsigned long long b = (unsigned long long)__double_as_longlong(v);
    for (int o = 16; o > 0; o >>= 1) {
        const unsigned long long x = __shfl_xor_sync(0xffffffffu, b, o);
        if (x > b) b = x;
    }
    if ((threadIdx.x & 31) == 0 && b > *(volatile unsigned long long *)slot) atomicMax(slot, b);
}

GZ_DEV double warp_sum(double v, unsigned mask, int width)
{
    for (int o = width / 2; o > 0; o >>= 1) v += __shfl_xor_sync(mask, v, o, width);
    return v;
}

GZ_DEV double warp_max(double v, unsigned mask, int width)
{
    for (int o = width / 2; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(mask, v, o, width));
    return v;
}

GZ_DEV double warp_min(double v, unsigned mask, int width)
{
    for (int o = width / 2; o > 0; o >>= 1) v = fmin(v, __shfl_xor_sync(mask, v, o, width));
    return v;
}

}  // namespace gz

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
};

// Octree over the Morton-sorted particles (63-bit keys, 21 levels): node i
// owns the sorted run [first, first + count); an internal node's children
// are the nodes [child, child + nchild); a leaf (child = -1) has at most
// kLeafMax particles unless it is at the deepest level (coincident keys).
// Leaves are tested 32 particles at a time; leaves of up to 96 particles
// (measured against 8 to 128) cost the walk fewer node openings than the extra
// candidate tests they bring.
constexpr int kLeafMax = 96;

struct Tree {
    double box;
    int n_nodes;
    int n_particles;
    const int4 *node;               // {first, count, child or -1, nchild}
    const double4 *lo;              // tight box minimum xyz; w = maximum h in the node
    const double4 *hi;              // tight box maximum xyz
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

struct Csr {
    const long long *off;           // [rows + 1]
    const int *nbr;                 // sorted particle indices
};

}  // namespace gz

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
    int *iters;
    const unsigned char *active;    // 1 for particles of the current active set
};

// Implicit octree over the Morton-sorted particles (63-bit keys, 21 levels):
// node (level L, Morton index m) owns the sorted run of keys with prefix m.
// The top D levels have a dense table of node starts (cell_start, level D)
// and node maxima of h (hmax, levels 0..D); below D, children are found by
// binary search in `keys` and h maxima come from 32-particle block maxima.
struct Grid {
    int D;
    int n;
    double box;
    const unsigned long long *keys; // sorted keys [n]
    const int *cell_start;          // [8^D + 1]
    const double *hmax;             // node maxima of h, levels 0..D
    const double *bmax;             // [ceil(n/32)] block maxima of h
    long long level_off[12];
};

// Compressed neighbour rows: row r of `slot_of` targets.
struct Csr {
    const long long *off;           // [rows + 1]
    const int *nbr;                 // sorted particle indices
};

}  // namespace gz

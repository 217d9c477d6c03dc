/* oracle/gizmo_oracle.h -- CPU restatement of GIZMO's meshless hydro pass.
 *
 * TEST INFRASTRUCTURE ONLY. This is the checker the CUDA path is compared
 * against; nothing in the product (gizmo_b200/, include/) links it. It is
 * loaded by tests/, by __graft_entry__.smoke() and by bench.py's CPU-baseline
 * leg, and nowhere else.
 *
 * It restates, in plain C with no fused multiply-adds, the reference's
 *   - density / kernel-length solve   (hydro/density_loop.h:515-961, 1140-1385;
 *                                      hydro/density_loop.cc:303-733)
 *   - gradient pass + slope limiter   (hydro/gradient_functions.h:304-665;
 *                                      hydro/gradients_loop.cc:76-136, 848-1130)
 *   - MFM/MFV force pass              (hydro/hydro_functions.h:56-546;
 *                                      hydro/hydro_core_meshless_functions.h:48-616;
 *                                      hydro/compute_finitevol_faces_functions.h:46-168;
 *                                      hydro/reimann.h:125-1090;
 *                                      hydro/hydro_toplevel.cc:133-253, 457-565)
 * for the ideal-gas, non-MHD, non-cosmological, 3-D, periodic-box build, and
 * an exact neighbour search applying the reference predicates
 * (density_loop.h:1163-1171 one-way; hydro_functions.h:77-83 symmetric).
 *
 * Parity is pinned against the reference's own pair bodies compiled from
 * its sources by oracle/build_ref.sh (see tests/test_oracle_vs_reference.py).
 */
#ifndef GIZMO_ORACLE_H
#define GIZMO_ORACLE_H

#include "../include/gizmo_hydro.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Particle state in original (unsorted) order, all FP64, row-major [n][k]. */
typedef struct orc_state {
    int n;
    /* inputs */
    double *pos;       /* [n][3] P.Pos */
    double *vel;       /* [n][3] CellP.VelPred */
    double *mass;      /* [n]    P.Mass */
    double *u;         /* [n]    CellP.InternalEnergyPred */
    double *dt;        /* [n]    physical timestep (get_particle_timestep_in_physical) */
    double *h;         /* [n]    P.KernelRadius (in: seed, out: converged) */
    double *cond;      /* [n]    CellP.ConditionNumber (in: previous value, out: new) */
    /* density outputs */
    double *num_ngb;   /* [n]    P.NumNgb (after the ^(1/3) transform) */
    double *drkern;    /* [n]    P.DrkernNgbFactor */
    double *divvel;    /* [n]    P.Particle_DivVel */
    double *rho;       /* [n]    CellP.Density */
    double *pressure;  /* [n]    CellP.Pressure */
    double *nvt;       /* [n][6] CellP.NV_T inverse, {xx,yy,zz,xy,yz,xz} */
    double *fce;       /* [n]    CellP.FaceClosureError */
    double *pvel;      /* [n][3] CellP.ParticleVel (MFV) */
    int    *iters;     /* [n]    density iterations taken */
    /* gradient outputs */
    double *grad_rho;  /* [n][3] */
    double *grad_p;    /* [n][3] */
    double *grad_v;    /* [n][9] row k = d v_k / d x */
    /* force outputs */
    double *accel;     /* [n][3] CellP.HydroAccel */
    double *dudt;      /* [n]    CellP.DtInternalEnergy */
    double *vsig;      /* [n]    CellP.MaxSignalVel */
    double *dtmass;    /* [n]    CellP.DtMass (MFV) */
    double *dmass;     /* [n]    CellP.dMass (MFV) */
    double *gravwork;  /* [n][3] CellP.GravWorkTerm (MFV) */
    /* individual timesteps (read only by orc_force_wakeup) */
    int    *timebin;   /* [n]    P.TimeBin */
    int    *wakeup;    /* [n]    P.wakeup (in/out: the largest wake-up flag set) */
} orc_state;

/* Neighbour sets in CSR form, original indices, each row sorted ascending. */
typedef struct orc_csr {
    long long *offsets;  /* [n_rows + 1] */
    int       *nbrs;     /* [offsets[n_rows]] */
    int        n_rows;
} orc_csr;

/* Runs the three passes (or one of them) on the active set (NULL = all).
 * Return 0 on success or a reference stop code (1155 density did not
 * converge, 90001009 empty bracket, 1234 no positive-pressure Riemann
 * solution). n_threads <= 0 uses the OpenMP default. */
int orc_density(const gz_params *p, orc_state *s, const int *active, int n_active, int n_threads);
/* The largest kernel length at which the last orc_density evaluated sums. */
double orc_density_h_iter_max(void);
int orc_gradients(const gz_params *p, orc_state *s, const int *active, int n_active, int n_threads);
int orc_force(const gz_params *p, orc_state *s, const int *active, int n_active, int n_threads);
/* orc_force with the wake-up of inactive neighbours (hydro_functions.h:534-544):
 * bin_active is TimeBinActive[60]; NULL switches the wake-up off, as orc_force does. */
int orc_force_wakeup(const gz_params *p, orc_state *s, const int *active, int n_active, int n_threads,
                     const int *bin_active);

/* Pair evaluations of the last orc_force that took each rare branch of the
 * Riemann cascade (test instrumentation): [0] Kurganov-Tadmor, [1] the exact
 * iterative solver, [2] the second attempt (cell-centred states), [3] the
 * third attempt (at rest). */
void orc_riemann_branches(long long out[4]);

/* make_list_of_active_particles (core/run.cc:997-1010), ascending: returns
 * the count and writes the indices into out (may be NULL). */
int orc_active_list(int n, const int *timebin, const double *mass, const int *bin_active, int *out);
/* The timebin each woken cell moves to, by process_wake_ups' rule
 * (core/timestep.cc:1565-1700); returns the number of cells moved. */
int orc_wakeup_bins(int n, const int *timebin, const int *wakeup, const double *mass, const int *bin_active,
                    int max_time_bin_active, int lowest_occupied_active_bin, int *out);

/* Density sums at a fixed kernel length, no iteration: writes the raw
 * accumulator of density_loop.h:1140-1385 for each active into acc[a][14]:
 * {Ngb, Rho, DrkernNgb, DivVel, NV_T xx,yy,zz,xy,yz,xz, face x,y,z, 0}
 * plus ParticleVel into pv[a][3] (MFV). */
int orc_density_sums(const gz_params *p, const orc_state *s, const int *active, int n_active,
                     double *acc, double *pv, int n_threads);

/* Exact neighbour sets. mode 0: one-way r < h_i (density); mode 1:
 * symmetric 0 < r and (r < h_i or r < h_j) (gradients, force).
 * Rows follow the active list. Free with orc_csr_free. */
int orc_neighbors(const gz_params *p, const orc_state *s, const int *active, int n_active,
                  int mode, orc_csr *out, int n_threads);
void orc_csr_free(orc_csr *c);

/* Half-step kick state (core/kicks.cc:284-545, do_the_kick), original
 * order, FP64, row-major [n][k]. The MFV fields are ignored under MFM. */
typedef struct orc_kick_state {
    int n;
    double *vel;        /* [n][3] P.Vel                          (in/out) */
    double *u;          /* [n]    CellP.InternalEnergy           (in/out) */
    double *mass;       /* [n]    P.Mass (MFV: MassTrue after the second half kick) (in/out) */
    double *mass_true;  /* [n]    CellP.MassTrue (MFV)           (in/out) */
    double *dmass;      /* [n]    CellP.dMass (MFV)              (in/out) */
    double *dtmass;     /* [n]    CellP.DtMass (MFV) */
    double *accel;      /* [n][3] CellP.HydroAccel */
    double *dudt;       /* [n]    CellP.DtInternalEnergy (the temperature floor zeroes it) (in/out) */
    double *grav;       /* [n][3] P.GravAccel */
    double *gravwork;   /* [n][3] CellP.GravWorkTerm (MFV) */
    double *vel_pred;   /* [n][3] CellP.VelPred           (out after the second half kick) */
    double *u_pred;     /* [n]    CellP.InternalEnergyPred (out after the second half kick) */
    double *dp;         /* [n][3] P.dp, the momentum kick accumulates here (in/out) */
    long long *tstart;  /* [n]    integer time the half step starts */
    long long *tend;    /* [n]    integer time it ends */
    int *active;        /* [n]    TimeBinActive of the particle's bin (0/1) */
} orc_kick_state;

/* One half-step kick of every particle with P.Mass > 0, as the kick loops
 * select them: mode 0 is the first half kick (kicks.cc:34-97), 1 the second
 * (kicks.cc:99-182). `timebase` is
 * All.Timebase_interval (physical time per integer tick), `min_egy_spec`
 * All.MinEgySpec (0: no floor). Non-comoving, no dilation. Returns 0. */
int orc_kick(const gz_params *p, orc_kick_state *k, int mode, double timebase, double min_egy_spec);

/* Drift state (core/drift_particle_functions.h:86-260, drift_particle_impl),
 * original order, FP64, row-major [n][k]. The MFV fields are ignored under
 * MFM, `vel` under MFV. */
typedef struct orc_drift_state {
    int n;
    double *pos;        /* [n][3] P.Pos                                  (in/out) */
    double *vel;        /* [n][3] P.Vel: an MFM cell moves with it */
    double *pvel;       /* [n][3] CellP.ParticleVel: an MFV cell moves with it */
    double *vel_pred;   /* [n][3] CellP.VelPred                          (in/out) */
    double *grav;       /* [n][3] P.GravAccel */
    double *accel;      /* [n][3] CellP.HydroAccel */
    double *divvel;     /* [n]    P.Particle_DivVel */
    double *mass;       /* [n]    P.Mass (MFV: the drifted mass)         (in/out) */
    double *dtmass;     /* [n]    CellP.DtMass (MFV) */
    double *mass_true;  /* [n]    CellP.MassTrue (MFV) */
    double *rho;        /* [n]    CellP.Density                          (in/out) */
    double *u_pred;     /* [n]    CellP.InternalEnergyPred               (in/out) */
    double *dudt;       /* [n]    CellP.DtInternalEnergy */
    double *h;          /* [n]    P.KernelRadius                         (in/out) */
    double *pressure;   /* [n]    CellP.Pressure                         (out for drifted cells) */
    long long *ti_current; /* [n] P.Ti_current, set to time1             (in/out) */
} orc_drift_state;

/* Drifts every gas cell from its Ti_current to the integer time `time1`
 * (drift_particle_impl; non-comoving, no dilation, ideal gas). `timebase` is
 * All.Timebase_interval, `min_egy_spec` All.MinEgySpec; the kernel-radius
 * bounds and gamma come from p. Returns 0, or 90001004 (the reference's
 * stop code) when a cell's Ti_current lies after time1; that cell is left
 * as it was. */
int orc_drift(const gz_params *p, orc_drift_state *d, long long time1, double timebase, double min_egy_spec);

/* Timestep state of gas cells (core/timestep.cc:357-1416 get_timestep, and
 * the per-particle binning of find_timesteps, timestep.cc:176-270),
 * original order. */
typedef struct orc_timestep_state {
    int n;
    double *grav;        /* [n][3] P.GravAccel */
    double *accel;       /* [n][3] CellP.HydroAccel */
    double *vsig;        /* [n]    CellP.MaxSignalVel */
    double *h;           /* [n]    P.KernelRadius */
    double *num_ngb;     /* [n]    P.NumNgb (after the ^(1/3) transform) */
    double *divvel;      /* [n]    P.Particle_DivVel */
    double *mass;        /* [n]    P.Mass */
    double *softening;   /* [n]    P.ForceSoftening (ForceSoftening_KernelRadius) */
    double *aphys;       /* [n]    out: the physical acceleration get_timestep returns through aphys */
    long long *ti_want;  /* [n]    out: get_timestep's integer step, before the binning */
    int *bin;            /* [n]    P.TimeBin                              (in/out) */
    long long *ti_begstep; /* [n]  P.Ti_begstep                           (in/out) */
    long long *dt_step;  /* [n]    P.dt_step                              (in/out) */
} orc_timestep_state;

typedef struct orc_timestep_params {
    double err_tol_int_accuracy;  /* All.ErrTolIntAccuracy */
    double courant_fac;           /* All.CourantFac */
    double max_size_timestep;     /* All.MaxSizeTimestep */
    double min_size_timestep;     /* All.MinSizeTimestep */
    double timebase;              /* All.Timebase_interval */
    long long ti_current;         /* All.Ti_Current */
    int bin_active[60];           /* TimeBinActive[TIMEBINS] */
} orc_timestep_params;

/* New timesteps of every gas cell (all taken as active), non-comoving, no
 * dilation. Returns 0, or the first stop code: 888 (a step below
 * MinSizeTimestep, STOP_WHEN_BELOW_MINTIMESTEP), 90001005 (beyond the end of
 * the timeline). */
int orc_timestep(const gz_params *p, const orc_timestep_params *tp, orc_timestep_state *t);

/* One-time timing helper for the CPU baseline: runs density (from the
 * given h seeds) -> gradients -> force on `n_active` targets and returns
 * wall seconds. */
double orc_full_pass_seconds(const gz_params *p, orc_state *s, const int *active, int n_active,
                             int n_threads, int *status);

#ifdef __cplusplus
}
#endif
#endif

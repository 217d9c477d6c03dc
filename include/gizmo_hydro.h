/* include/gizmo_hydro.h -- C ABI of the B200 meshless hydro pass.
 *
 * Drop-in boundary for GIZMO's hydro neighbour loops. In the reference the
 * three host entry points
 *     void density(void)             src/hydro/density_loop.cc:764
 *     void hydro_gradient_calc(void) src/hydro/gradients_loop.cc:458
 *     void hydro_force(void)         src/hydro/hydro_force_loop.cc:423
 * drive the neighbour-loop runner (run_neighbor_loop_iterative<DensitySpec>,
 * run_neighbor_loop<GradientsSpec>, run_neighbor_loop<HydroForceSpec>;
 * src/mesh/neighbor_loop_runner.h:1614-1629) over the global P[] / CellP[]
 * arrays. A shim compiled into the reference host replaces those three
 * runner calls with the gz_hydro_* calls below; the host keeps gravity,
 * cooling, domain, timestep and I/O. The shim gathers the P/CellP fields
 * listed in gz_particles (AoS -> SoA) for gz_upload and scatters the
 * gz_outputs fields back after gz_download.
 *
 * Conventions (mirroring the reference's endrun() semantics without a stop):
 *   - every call returns GZ_OK (0) or a nonzero code; reference stop codes
 *     are kept where one exists (1155, 90001009, 1234);
 *   - no exceptions cross the ABI and device code never traps: device-side
 *     failures are recorded in a status word and read by gz_status;
 *   - the library owns all device memory; the caller owns host arrays;
 *   - one context per thread at a time; each context has its own stream.
 * Plain pointers and sizes only. Arrays are row-major [n][k] FP64 in the
 * caller's original particle order.
 */
#ifndef GIZMO_HYDRO_H
#define GIZMO_HYDRO_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Kernel functions (KERNEL_FUNCTION, src/mesh/kernel.h:268-438). */
#define GZ_KERNEL_CUBIC        3   /* Morris cubic spline, norm 8/pi */
#define GZ_KERNEL_WENDLAND_C2  6   /* Wendland C2, norm 21/(2 pi) */

/* Hydro methods (HYDRO_MESHLESS_FINITE_MASS / _VOLUME). */
#define GZ_METHOD_MFM 0
#define GZ_METHOD_MFV 1

/* Arithmetic forms of the pass. */
#define GZ_PRECISION_FP64  0   /* every pair and per-particle operation in FP64 */
#define GZ_PRECISION_MIXED 1   /* FP32 force-pair arithmetic (pairs whose FP32 decisions are too close
                                  to call evaluated again in FP64); FP64 positions, membership,
                                  density and h-iteration, gradients, 3x3 inversion and flux sums */

/* Return codes. */
#define GZ_OK                   0
#define GZ_ERR_ARG              1       /* bad argument or size */
#define GZ_ERR_CUDA             2       /* CUDA runtime error (message in gz_status) */
#define GZ_ERR_NO_DEVICE        3
#define GZ_ERR_ORDER            4       /* pass called before its inputs exist */
#define GZ_ERR_CAPACITY         5       /* a device work buffer would exceed its limit */
#define GZ_ERR_INTERNAL         6       /* an internal consistency check failed (a bug: please report) */
#define GZ_ERR_DENSITY_MAXITER  1155    /* neighbor_loop_runner.cc:7485 endrun(1155) */
#define GZ_ERR_EMPTY_BRACKET    90001009 /* density_loop.h:891-895 */
#define GZ_ERR_RIEMANN          1234    /* hydro_core_meshless_functions.h:403-425 */
#define GZ_ERR_NO_PAST_DRIFT    90001004 /* drift_particle_functions.h:90-95: a drift into the past */
#define GZ_ERR_MIN_TIMESTEP     888      /* timestep.cc (STOP_WHEN_BELOW_MINTIMESTEP): a step below MinSizeTimestep */
#define GZ_ERR_END_OF_TIMELINE  90001005 /* timestep.cc:265-270: a step beyond the end of the timeline */

/* Run-time configuration: the All.* fields and compile-time flags the pass
 * reads. Non-cosmological (cf_atime = 1, ComovingIntegrationOn = 0). */
typedef struct gz_params {
    int    kernel;             /* GZ_KERNEL_* */
    int    method;             /* GZ_METHOD_* */
    int    precision;          /* GZ_PRECISION_* */
    int    first_step;         /* 1 when All.Time == All.TimeBegin (density_loop.h:523-525) */
    int    selfgravity_off;    /* SELFGRAVITY_OFF: limiter h_lim/stol (gradients_loop.cc:1094-1096)
                                  and MFM entropic thresholds (hydro_functions.h:175-183) */
    int    reserved;
    double box_size;           /* All.BoxSize, periodic in x, y, z */
    double gamma;              /* EOS_GAMMA (ideal gas P = (gamma-1) rho u) */
    double des_num_ngb;        /* All.DesNumNgb */
    double max_num_ngb_dev;    /* All.MaxNumNgbDeviation */
    double min_kernel_radius;  /* All.MinKernelRadius */
    double max_kernel_radius;  /* All.MaxKernelRadius */
} gz_params;

/* Inputs per gas particle (the P / CellP fields the pass reads). */
typedef struct gz_particles {
    int64_t       n;
    const double *pos;    /* [n][3] P[i].Pos, inside [0, box_size); a position outside is
                             reported as GZ_ERR_ARG (with its index) by the next pass */
    const double *vel;    /* [n][3] CellP[i].VelPred */
    const double *mass;   /* [n]    P[i].Mass */
    const double *u;      /* [n]    CellP[i].InternalEnergyPred */
    const double *dt;     /* [n]    get_particle_timestep_in_physical(i) */
    const double *h;      /* [n]    P[i].KernelRadius seed for the density iteration */
    const double *cond;   /* [n]    CellP[i].ConditionNumber from the previous step (0 if none) */
    /* individual timesteps (both may be NULL: no wake-up) */
    const int32_t *timebin; /* [n]  P[i].TimeBin */
    const double  *vsig;    /* [n]  CellP[i].MaxSignalVel from the cell's last force pass: the wake-up
                               test (hydro_functions.h:534-544) reads it for inactive neighbours */
} gz_particles;

/* Outputs; any pointer may be NULL to skip that field. */
typedef struct gz_outputs {
    double *h;         /* [n]    P.KernelRadius */
    double *num_ngb;   /* [n]    P.NumNgb (after ^(1/3)) */
    double *drkern;    /* [n]    P.DrkernNgbFactor */
    double *divvel;    /* [n]    P.Particle_DivVel */
    double *rho;       /* [n]    CellP.Density */
    double *pressure;  /* [n]    CellP.Pressure */
    double *nvt;       /* [n][6] CellP.NV_T (inverse, xx yy zz xy yz xz) */
    double *cond;      /* [n]    CellP.ConditionNumber */
    double *fce;       /* [n]    CellP.FaceClosureError */
    double *pvel;      /* [n][3] CellP.ParticleVel (MFV) */
    double *grad_rho;  /* [n][3] CellP.Gradients.Density */
    double *grad_p;    /* [n][3] CellP.Gradients.Pressure */
    double *grad_v;    /* [n][9] CellP.Gradients.Velocity (row k = grad v_k) */
    double *accel;     /* [n][3] CellP.HydroAccel (dv/dt) */
    double *dudt;      /* [n]    CellP.DtInternalEnergy (du/dt) */
    double *vsig;      /* [n]    CellP.MaxSignalVel */
    double *dtmass;    /* [n]    CellP.DtMass (MFV) */
    double *dmass;     /* [n]    CellP.dMass (MFV) */
    double *gravwork;  /* [n][3] CellP.GravWorkTerm (MFV) */
    int    *iters;     /* [n]    density iterations taken */
    int32_t *wakeup;   /* [n]    the wake-up flag the last force pass gave each cell (hydro_functions.h:
                          534-544): the largest bin + 1 of an active neighbour whose pair signal speed
                          exceeded WAKEUP (4.1) x the cell's stored MaxSignalVel; 0 for none. Merge it
                          into P.wakeup with a max (the reference's HYDRO_ATOMIC_MAX) */
    double *flux_abs;  /* [n][3] diagnostic (GZ_DIAG_FLUX_ABS), no reference counterpart: the sums over the
                          force row of |mass flux|, |momentum flux| and |energy flux| of
                          the pairs, the scale against which the cancelling sums dtmass,
                          mass * accel and mass * dudt are accurate */
} gz_outputs;

typedef struct gz_status_info {
    int      code;              /* first recorded error code, 0 if none */
    int      index;             /* original particle index it refers to, -1 if none */
    int      density_iterations;/* iterations of the last density pass */
    int      reserved;
    int64_t  pairs_density;     /* density-row entries built (candidates within the row radii) */
    int64_t  pairs_symmetric;   /* symmetric pairs (rows of the gradient/force lists) */
    int64_t  device_bytes;      /* device memory held by the context */
    int64_t  kernel_launches;   /* kernels of this library launched by the context so far */
    char     message[256];
    double   h_iter_max;        /* the largest kernel length at which the last density pass took
                                   sums: its seeds (after the clamp of density_loop.cc:837-840) and
                                   every radius its iteration moved to */
    int64_t  pairs_refined;     /* mixed form: pairs of the last force pass evaluated again in FP64
                                   because an FP32 branch decision was too close to call or its
                                   arithmetic cancelled beyond FP32's reach */
} gz_status_info;

typedef struct gz_context gz_context;

/* Create a context on CUDA device `device` (its own stream). */
int gz_create(const gz_params *params, int device, gz_context **out);
int gz_destroy(gz_context *ctx);
/* Replace the run-time configuration (keeps particle data). */
int gz_set_params(gz_context *ctx, const gz_params *params);

/* Diagnostics the force pass computes besides the reference's outputs (no
 * reference counterpart). GZ_DIAG_FLUX_ABS: the flux_abs sums of gz_outputs.
 * Off by default, so that the pass pays for none; gz_download of flux_abs
 * returns GZ_ERR_ORDER unless the last force pass ran with it on. */
#define GZ_DIAG_FLUX_ABS 1
int gz_set_diagnostics(gz_context *ctx, int flags);

/* Copy inputs host -> device, sort the particles by Morton key, build the
 * octree and the sorted particle mirror. Replaces the arena acquire of
 * neighbor_loop_runner.cc:2297-2302 and the spatial-index build of
 * gpu_neighbor_list.cc:1134-1169. */
int gz_upload(gz_context *ctx, const gz_particles *in);

/* Rebuild the octree and the sorted mirror from the inputs already resident
 * on the device (the last gz_upload), resetting kernel lengths and condition
 * numbers to the uploaded values: the start of a pass without host traffic. */
int gz_restage(gz_context *ctx);

/* The three passes. `active` lists original indices (NULL = all particles),
 * like ActiveParticleList filtered by density_isactive / GasGrad_isactive.
 *   gz_hydro_density   : DensitySpec loop + density_finalize_post_runner
 *   gz_hydro_gradients : GradientsSpec loop + gradient finalize/limiter
 *   gz_hydro_force     : preloop + HydroForceSpec loop + hydro_final_operations
 * With no target (no particles, or n_active == 0) a call returns GZ_OK,
 * launches nothing and changes no output, as the reference's loops do not
 * run on an empty active list. */
int gz_hydro_density(gz_context *ctx, const int *active, int n_active);
int gz_hydro_gradients(gz_context *ctx, const int *active, int n_active);
int gz_hydro_force(gz_context *ctx, const int *active, int n_active);

/* The three passes over every particle in one call (compute_hydro_densities_
 * and_forces, src/core/accel.cc:80-169, with all gas active). With
 * GZ_PASS_GRAPH the pass runs as one CUDA graph with no host round trip: the
 * density iteration as a device-driven loop, then the symmetric rows, gradients
 * and force. The graph is captured at the first such call after a plain pass
 * has sized its buffers (the first call runs plain) and replayed while the
 * context's buffers and settings are unchanged (a gz_restage keeps them); its
 * results equal the three calls' bit for bit. Where a device-sized buffer
 * would overflow, the call runs the plain pass from the same inputs
 * (gz_graph_stats counts those). Kernel timing (gz_kernel_timing) runs plain. */
#define GZ_PASS_GRAPH 1
/* GZ_PASS_RESTAGE: the pass starts with gz_restage (inside the graph with
 * GZ_PASS_GRAPH, the octree then built on the device with nothing read back;
 * a pipelined upload is copied into the resident inputs instead of swapped). */
#define GZ_PASS_RESTAGE 2
int gz_hydro_pass(gz_context *ctx, int flags);

/* Box sets: the particles of the following uploads are n_boxes consecutive
 * runs of counts[b] particles, each an independent periodic box of the
 * context's box_size and parameters (a pair never joins two boxes). The passes
 * then cover all boxes in one launch per kernel (and gz_hydro_pass in one
 * graph): the Morton keys carry the box index above 21 - box_bits/3 bits per
 * axis (box_bits = 3 ceil(log2(n_boxes) / 3)), so each box is one run of the
 * sorted particles and one subtree of the octree, where the walks of its
 * particles start. n_boxes <= 1 returns to one box; at most 32768 boxes.
 * The next gz_upload must hold sum(counts) particles. */
int gz_set_boxes(gz_context *ctx, int n_boxes, const int64_t *counts);

typedef struct gz_graph_info {
    int64_t captures;               /* graphs captured (a change of buffers or settings captures again) */
    int64_t replays;                /* passes run through a graph */
    int64_t fallbacks;              /* ... of which ran again as plain passes */
    int64_t kernels_top;            /* kernels of one replay outside the conditional bodies */
    int64_t kernels_per_iteration;  /* kernels of one density iteration */
    int64_t kernels_after;          /* kernels of the symmetric rows, gradients and force */
} gz_graph_info;
int gz_graph_stats(gz_context *ctx, gz_graph_info *out);

/* Copy outputs device -> host (original order). */
int gz_download(gz_context *ctx, const gz_outputs *out);

/* Pipelined transfers, for a host that overlaps the copies of one step with
 * the pass of another (from pinned host memory they run on a copy stream of
 * the context, beside its kernels):
 *   gz_upload_async  : the inputs of the next step (same n, no timebins; other
 *                      uploads fall back to gz_upload) are copied while the
 *                      current pass runs; the next gz_restage makes them the
 *                      resident inputs. The host arrays must stay untouched
 *                      until that gz_restage returns.
 *   gz_download_async: the outputs of the last pass are scattered to a device
 *                      staging area on the context's stream and copied to the
 *                      host arrays on the copy stream; the next pass does not
 *                      wait for the copies. The host arrays are filled when
 *                      gz_wait returns.
 *   gz_wait          : waits for the pending output copies (and orders the
 *                      context's stream after them). */
int gz_upload_async(gz_context *ctx, const gz_particles *in);
int gz_download_async(gz_context *ctx, const gz_outputs *out);
int gz_wait(gz_context *ctx);

/* gz_upload and gz_download with the caller's arrays in DEVICE memory (the
 * same layouts; device-to-device copies and scatters, no host traffic), for a
 * host that keeps its particle arena on the GPU and chains the pass with
 * gz_timestep, gz_kick and gz_drift there. gz_upload_device does not check
 * the timebin range (gz_upload does); gz_download_device returns with its
 * scatters queued on the context's stream (gz_stream): order later work on
 * other streams after it. */
int gz_upload_device(gz_context *ctx, const gz_particles *in);
int gz_download_device(gz_context *ctx, const gz_outputs *out);

/* Tuning of the neighbour walk (no reference counterpart). Neither setting
 * changes a result -- the rows are the exact neighbour sets in ascending order
 * whatever the tree -- both change what the walk costs:
 *   leaf_max   octree leaf size (particles), 96 by default;
 *   row_slots  slots per padded density row, as a multiple of the expected row
 *              length (2.5 by default); a longer row is rebuilt behind the
 *              padded block.
 * gz_set_tuning takes effect at the next gz_upload or gz_restage.
 * gz_autotune times a rebuild of the grid and a density pass over every
 * particle of the uploaded set for leaf_max in {32, 64, 96, 128} and then
 * row_slots in {1.5, 2.0, 2.5, 3.0}, keeps the fastest, remembers it for the
 * device, the particle count (to a power of two), DesNumNgb and the kernel
 * (a later context with the same key takes it without timing), and leaves
 * the set restaged as after gz_upload. */
typedef struct gz_tuning {
    int    leaf_max;
    int    reserved;
    double row_slots;
} gz_tuning;
int gz_get_tuning(gz_context *ctx, gz_tuning *out);
int gz_set_tuning(gz_context *ctx, const gz_tuning *t);
int gz_autotune(gz_context *ctx, gz_tuning *chosen);

/* Individual timesteps. GZ_TIMEBINS is TIMEBINS (declarations/allvars.h). */
#define GZ_TIMEBINS 60
/* TimeBinActive[GZ_TIMEBINS] for the wake-up test of the following force
 * passes over an active subset (hydro_functions.h:534-544; the reference reads
 * the global table). NULL switches the wake-up off, the default. Needs the
 * timebin and vsig inputs of gz_upload. */
int gz_set_bin_active(gz_context *ctx, const int *bin_active);
/* make_list_of_active_particles (core/run.cc:997-1010) on the device: the
 * cells whose TimeBin is active in bin_active[GZ_TIMEBINS] and whose mass is
 * positive, as original indices in ascending order (the reference walks the
 * bins' lists; the passes accept any order). *n_out receives the count; out
 * (NULL: count only) holds it. */
int gz_active_list(gz_context *ctx, const int *bin_active, int *out, int *n_out);
/* The bin rule of process_wake_ups (core/timestep.cc:1565-1700) on the device,
 * for the cells the last force pass woke: bin = the waker's bin less the bins
 * WAKEUP spans (3), floored at lowest_occupied_active_bin, capped at
 * max_time_bin_active (the highest bin active at the next kick) and never
 * above the cell's own; active cells and cells without mass keep theirs.
 * timebin_out[n] (original order) receives every cell's bin, *n_moved the
 * cells that moved. The timebin lists, the step truncation and the kicks of
 * the woken cells stay with the caller (gz_kick gives the kicks). */
int gz_wakeup_bins(gz_context *ctx, const int *bin_active, int max_time_bin_active, int lowest_occupied_active_bin,
                   int *timebin_out, int *n_moved);

/* Error/progress record of the context (device status word included). */
int gz_status(gz_context *ctx, gz_status_info *info);

/* CUDA stream of the context (cudaStream_t), for callers that time or
 * order work around the passes. */
void *gz_stream(gz_context *ctx);

/* CUDA-event timing of the passes' main kernels on the context's stream (no
 * reference counterpart: a measurement aid). gz_kernel_timing(ctx, 1) starts
 * recording and clears the totals, 0 stops it. gz_kernel_time synchronises the
 * stream and returns, for one timer, the summed kernel time in milliseconds,
 * the launches and the work units since the last clear, then clears them.
 * Units: GZ_TIMER_DENSITY_SUMS rows summed; GZ_TIMER_WALK targets walked;
 * GZ_TIMER_GRADIENTS rows; GZ_TIMER_FORCE pair evaluations (each pair once in
 * a pass over every particle, otherwise every row entry). */
#define GZ_TIMER_DENSITY_SUMS 0
#define GZ_TIMER_WALK         1
#define GZ_TIMER_GRADIENTS    2
#define GZ_TIMER_FORCE        3
#define GZ_TIMERS             4
int gz_kernel_timing(gz_context *ctx, int enable);
int gz_kernel_time(gz_context *ctx, int timer, double *ms, int64_t *launches, int64_t *units);

/* Exact neighbour sets of the last pass, for bit-exact checks against a CPU
 * search. mode 0: one-way r < h_i at the converged h; mode 1: symmetric
 * 0 < r and (r < h_i or r < h_j), from a tree walk; mode 2: the symmetric
 * rows the last gradient/force pass over all particles used (derived from
 * the density rows when the density pass covered every particle; otherwise
 * GZ_ERR_ORDER). Rows follow `active` (NULL = all),
 * entries are original indices sorted ascending. Call once with
 * nbrs == NULL to get offsets (n_active + 1 entries); then with nbrs sized
 * offsets[n_active]. */
int gz_neighbors(gz_context *ctx, const int *active, int n_active, int mode,
                 int64_t *offsets, int *nbrs);

/* Density accumulator at the current kernel lengths, no iteration: for each
 * active, acc[a][14] = {Ngb, Rho, DrkernNgb, DivVel, NV_T xx,yy,zz,xy,yz,xz,
 * face x,y,z, 0} and pv[a][3] = ParticleVel sum (MFV), exactly the
 * DensitySpec::pair_kernel sums (density_loop.h:1140-1385). */
int gz_density_sums(gz_context *ctx, const int *active, int n_active, double *acc, double *pv);

/* No counterpart in the reference. Density sums as gz_density_sums computes
 * them (same layout of acc[a][14] and pv[a][3], same pair arithmetic in
 * FP64), for callers that cannot allocate device memory: a host code whose own
 * memory pool already owns the device, or a loop that cannot afford the
 * device-wide synchronisation that cudaMalloc/cudaFree implies. It needs no
 * gz_context and allocates nothing:
 *   - pos [n][3], vel [n][3], mass [n], h [n] (inputs, particles in [0, box)) and
 *     acc [n][14], pv [n][3] (outputs; pv may be NULL) are DEVICE pointers that
 *     the caller owns; rows follow the caller's order, every particle is a
 *     target and a candidate;
 *   - the only scratch is a static device array of GZ_NOALLOC_MAX_PARTICLES
 *     packed records (4 MiB), held by every GPU that loads the library until
 *     the process exits; n above that limit returns GZ_ERR_CAPACITY;
 *   - work is queued on `stream` (a cudaStream_t, NULL for the default
 *     stream) and the call returns without waiting: synchronise the stream
 *     before reading acc;
 *   - the first call on each device looks up that array's device address
 *     (a one-time set-up on the current device): make that first call before
 *     any stream capture. Under CUDA's lazy module loading (the default since
 *     CUDA 12.2) that first call is also where the library's device code is
 *     loaded on the device and the 4 MiB array is reserved, so it must come
 *     before the caller's memory pool reserves the device; setting
 *     CUDA_MODULE_LOADING=EAGER reserves it when the process first creates
 *     its CUDA context instead. A failed set-up returns GZ_ERR_CUDA;
 *   - every call on a device uses the same array and rewrites it; two calls
 *     whose work overlaps on the GPU (different streams, no ordering between
 *     them) race on it and their results are undefined.
 * The neighbour loop is all-pairs over the set, which is what bounds n. */
#define GZ_NOALLOC_MAX_PARTICLES 65536
int gz_density_sums_noalloc(const gz_params *params, int n, const double *pos, const double *vel,
                            const double *mass, const double *h, double *acc, double *pv, void *stream);

/* One half-step kick, do_the_kick (core/kicks.cc:284-545), for every
 * particle of a set the caller holds in DEVICE memory (the reference's
 * particle arena, structure of arrays): the loops of do_first_halfstep_kick
 * (mode 0, kicks.cc:34-97) and do_second_halfstep_kick (mode 1,
 * kicks.cc:99-182) over gas cells, which kick only cells with P.Mass > 0.
 * Rows follow the caller's order; FP64 row-major [n][k] like gz_particles. */
typedef struct gz_kick_fields {
    int64_t n;
    double        *vel;        /* [n][3] P.Vel                                   in/out */
    double        *u;          /* [n]    CellP.InternalEnergy                    in/out */
    double        *mass;       /* [n]    P.Mass (MFV: MassTrue after mode 1)     in/out */
    double        *mass_true;  /* [n]    CellP.MassTrue (MFV; NULL under MFM)    in/out */
    double        *dmass;      /* [n]    CellP.dMass (MFV; NULL under MFM)       in/out */
    const double  *dtmass;     /* [n]    CellP.DtMass (MFV; NULL under MFM) */
    const double  *accel;      /* [n][3] CellP.HydroAccel */
    double        *dudt;       /* [n]    CellP.DtInternalEnergy (the temperature floor zeroes it) in/out */
    const double  *grav;       /* [n][3] P.GravAccel (NULL: zero) */
    const double  *gravwork;   /* [n][3] CellP.GravWorkTerm (MFV; NULL: zero) */
    double        *vel_pred;   /* [n][3] CellP.VelPred, written by mode 1 */
    double        *u_pred;     /* [n]    CellP.InternalEnergyPred, written by mode 1 */
    double        *dp;         /* [n][3] P.dp, the momentum kick is added    in/out */
    const int64_t *tstart;     /* [n]    integer time the half step starts (Ti_begstep or its midpoint) */
    const int64_t *tend;       /* [n]    integer time it ends */
    const int32_t *active;     /* [n]    TimeBinActive[P.TimeBin] (NULL: all active) */
} gz_kick_fields;

/* Kicks every particle of `f` by one half step. `timebase` is
 * All.Timebase_interval (physical time per integer tick, non-comoving, no
 * timestep dilation) and `min_egy_spec` All.MinEgySpec (0: no floor). Work is
 * queued on `stream` (a cudaStream_t, NULL for the default stream) and the
 * call returns without waiting; it needs no gz_context and allocates
 * nothing. Arithmetic is FP64 without contraction, bit-identical to the
 * reference's expression order. */
int gz_kick(const gz_params *params, const gz_kick_fields *f, int mode, double timebase, double min_egy_spec,
            void *stream);

/* The drift, drift_particle_impl (core/drift_particle_functions.h:86-260),
 * of every gas cell of a set the caller holds in DEVICE memory, from its
 * Ti_current to the integer time `time1`, as move_particles
 * (core/predict.cc:171) drifts them. Rows follow the caller's order; FP64 row-major [n][k]. Positions
 * are not wrapped into the box, as in the reference. */
typedef struct gz_drift_fields {
    int64_t n;
    double        *pos;        /* [n][3] P.Pos                                          in/out */
    const double  *vel;        /* [n][3] P.Vel: an MFM cell moves with it (unused under MFV) */
    const double  *pvel;       /* [n][3] CellP.ParticleVel: an MFV cell moves with it (unused under MFM) */
    double        *vel_pred;   /* [n][3] CellP.VelPred                                  in/out */
    const double  *grav;       /* [n][3] P.GravAccel (NULL: zero) */
    const double  *accel;      /* [n][3] CellP.HydroAccel */
    const double  *divvel;     /* [n]    P.Particle_DivVel */
    double        *mass;       /* [n]    P.Mass (MFV: the drifted mass)                 in/out */
    const double  *dtmass;     /* [n]    CellP.DtMass (MFV; NULL under MFM) */
    const double  *mass_true;  /* [n]    CellP.MassTrue (MFV; NULL under MFM) */
    double        *rho;        /* [n]    CellP.Density                                  in/out */
    double        *u_pred;     /* [n]    CellP.InternalEnergyPred                       in/out */
    const double  *dudt;       /* [n]    CellP.DtInternalEnergy */
    double        *h;          /* [n]    P.KernelRadius                                 in/out */
    double        *pressure;   /* [n]    CellP.Pressure (ideal gas), written for drifted cells */
    int64_t       *ti_current; /* [n]    P.Ti_current, set to time1                     in/out */
    int32_t       *status;     /* [1]    device word: a cell whose Ti_current lies after time1 is left as
                                  it was and GZ_ERR_NO_PAST_DRIFT is written here unless a code
                                  is already there (the kernel never clears it) */
} gz_drift_fields;

/* Drifts every cell of `f` to `time1`. `timebase` is All.Timebase_interval
 * (non-comoving, no timestep dilation), `min_egy_spec` All.MinEgySpec; the
 * kernel-radius bounds and gamma come from `params`. Queued on `stream` (a
 * cudaStream_t, NULL for the default stream) without waiting; no context, no
 * allocation. FP64 without contraction; the two exponentials are correctly
 * rounded, so results match the reference bit for bit except where its
 * libm exp is one ulp off: then the density and the kernel radius differ by
 * at most 2 ulp and the pressure by at most 4. */
int gz_drift(const gz_params *params, const gz_drift_fields *f, int64_t time1, double timebase, double min_egy_spec,
             void *stream);

/* The timestep of every gas cell of a set the caller holds in DEVICE memory:
 * get_timestep (core/timestep.cc:357-1416) -- the acceleration criterion on
 * the force softening (KERNEL_CORE_SIZE of params->kernel), the Courant
 * criterion CourantFac L / (MaxSignalVel / 2) with L = 1.61199 h / NumNgb,
 * the 1.5 / |divv| limit, MaxSizeTimestep, the MinSizeTimestep floor and the
 * integer step -- then the per-particle binning of find_timesteps
 * (timestep.cc:176-215, 265-270): the largest power of two not above it, a
 * larger bin only where it is active (synchronised), the end of the
 * timeline; Ti_begstep moves on by the old step. Non-comoving, no dilation;
 * every cell of the set is treated as active, as gz_kick does. Rows follow
 * the caller's order; FP64 row-major [n][k]. */
typedef struct gz_timestep_params {
    double  err_tol_int_accuracy;  /* All.ErrTolIntAccuracy */
    double  courant_fac;           /* All.CourantFac */
    double  max_size_timestep;     /* All.MaxSizeTimestep */
    double  min_size_timestep;     /* All.MinSizeTimestep */
    double  timebase;              /* All.Timebase_interval */
    int64_t ti_current;            /* All.Ti_Current */
    int32_t bin_active[GZ_TIMEBINS]; /* TimeBinActive after this step's sync point */
} gz_timestep_params;

typedef struct gz_timestep_fields {
    int64_t n;
    const double *grav;       /* [n][3] P.GravAccel (NULL: zero) */
    const double *accel;      /* [n][3] CellP.HydroAccel */
    const double *vsig;       /* [n]    CellP.MaxSignalVel */
    const double *h;          /* [n]    P.KernelRadius */
    const double *num_ngb;    /* [n]    P.NumNgb (after ^(1/3)) */
    const double *divvel;     /* [n]    P.Particle_DivVel */
    const double *mass;       /* [n]    P.Mass */
    const double *softening;  /* [n]    ForceSoftening_KernelRadius (NULL: zero, the kernel-size fallback) */
    double       *aphys;      /* [n]    out: |a| as get_timestep returns it through aphys (NULL: skip) */
    int64_t      *ti_want;    /* [n]    out: get_timestep's integer step before the binning (NULL: skip) */
    int32_t      *bin;        /* [n]    P.TimeBin                                    in/out */
    int64_t      *ti_begstep; /* [n]    P.Ti_begstep                                 in/out */
    int64_t      *dt_step;    /* [n]    P.dt_step                                    in/out */
    int32_t      *status;     /* [1]    device word: GZ_ERR_MIN_TIMESTEP or GZ_ERR_END_OF_TIMELINE is written
                                 here unless a code is already there (NULL: not reported) */
} gz_timestep_fields;

/* New steps and bins of every cell of `f`, queued on `stream` (a
 * cudaStream_t, NULL for the default stream) without waiting; no context, no
 * allocation. FP64 without contraction, bit-identical to the reference. */
int gz_timestep(const gz_params *params, const gz_timestep_params *tp, const gz_timestep_fields *f, void *stream);

#ifdef __cplusplus
}
#endif
#endif

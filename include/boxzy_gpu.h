/*
 * boxzy_gpu.h -- C ABI of the B200 (sm_100a) FP64 hydrodynamic step of BOXZYHYDRO.
 *
 * The reference has no plugin or FFI API: its hot path is a set of argument-less
 * Fortran subroutines that share module arrays (grid_commons.f90:11-24) and are
 * called from the main time loop (main.f90:211-555).  Each entry point below
 * replaces one of those subroutines (cited beside it) or the whole loop body,
 * with the module arrays held in device memory by an opaque handle.
 *
 * Conventions
 *  - Every function returns an int status: BX_OK (0) or a BX_ERR_* code; the
 *    message of the last error is bx_last_error(h).  No C++ exception crosses
 *    this boundary.
 *  - Host arrays use the reference layout: cons(5,ngrid), u(3,ngrid) and
 *    p(ngrid), Fortran column-major, i.e. 5 (resp. 3, 1) doubles per cell, cells
 *    in igrid order (ix fastest).  A Fortran caller passes its allocatable
 *    arrays directly (assumed-size dummies of a bind(c) interface).
 *  - Calls on one handle are single-threaded (outside OpenMP parallel regions or
 *    under !$OMP MASTER).  Each handle owns one CUDA stream unless one is given.
 *  - Steps run on the fused stage kernels: the fixed-gamma EOS (H2STAT=-1)
 *    with or without a gravitational force (bx_set_gforce, bx_set_phi), and,
 *    without a force, the tabulated EOS (H2STAT>=0 with nz != 1,
 *    bx_set_eos_table) and angular-momentum fluxing (fluxangmom=1).  The other
 *    combinations, grids whose ghost rule the fused kernels do not take, and
 *    steps in which the velocity limiter or the low-density branch fires run on
 *    the per-phase kernels.  Both give the reference's results bit for bit.
 */
#ifndef BOXZY_GPU_H
#define BOXZY_GPU_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define BX_OK 0
#define BX_ERR_ARG 1          /* bad argument or size */
#define BX_ERR_CUDA 2         /* CUDA runtime error */
#define BX_ERR_UNSUPPORTED 3  /* configuration outside the GPU path */
#define BX_ERR_STATE 4        /* non-finite state or zero HLL wave speed */
#define BX_ERR_NOMEM 5        /* device allocation failed */

/* status bits reported by bx_status */
#define BX_STATUS_VLIMIT 1u     /* velocity limiter fired (velocity.f90:31-50) */
#define BX_STATUS_LOWRHO 2u     /* low-density EOS branch taken (state.f90:52-56) */
#define BX_STATUS_NONFINITE 4u  /* NaN or Inf produced */
#define BX_STATUS_ZEROWAVE 8u   /* ap+am == 0 at a face (flux.f90:588) */

/* bx_params.flags */
#define BX_FLAG_PHASE_ONLY 1    /* always run the per-phase kernels, never the fused stages */

typedef struct bx_params {
  int32_t nx, ny, nz;     /* grid_params nx,ny,nz: cells incl. two ghost layers per side
                             (z ghosts only when nz>=6), init_grid.f90:18,76-107 */
  int32_t h2stat;         /* eos_input H2STAT: -1 fixed gamma (state.f90:49-59); >= 0
                             tabulated EOS (state.f90:60-79, bx_set_eos_table) */
  double dx, dy, dz;      /* grid_params dx,dy,dz */
  double cfl;             /* hydro cfl (courant.f90:28) */
  double small_rho;       /* hydro small_rho (flux.f90:225) */
  double small_eps;       /* hydro small_eps */
  double vlimit;          /* hydro vlimit (velocity.f90:32) */
  double gammafix;        /* eos_input gammafix */
  double muc;             /* mean molecular weight, eos.f90:144 */
  double rgas;            /* scale%rgas of get_units, units.f90:17 */
  int32_t no_outflow[6];  /* grid_params no_outflow_xl,xr,yl,yr,zl,zr (reflective walls) */
  int32_t fluxangmom;     /* grid_params fluxangmom: 1 = flux_ang.f90 in place of flux.f90
                             (angular-momentum fluxing) */
  int32_t flags;          /* BX_FLAG_* */
  double yoffset;         /* grid_params yoffset (flux_ang.f90:46,251) */
} bx_params;

typedef struct bx_handle bx_handle;

/* Library version string. */
const char *bx_version(void);

/* Allocate one grid on the current CUDA device and build its ghost tables.
 * Replaces init_grid (init_grid.f90:7-265) and the allocation of the module
 * arrays of grid_commons.f90:11-24. */
int bx_create(const bx_params *params, bx_handle **out);

/* Free all device memory of the handle (cleanup.f90:1-16). */
int bx_destroy(bx_handle *h);

/* Run all work of the handle on the given cudaStream_t (NULL = own stream). */
int bx_set_stream(bx_handle *h, void *cuda_stream);

/* Copy the reference's state arrays in: cons(5,ngrid), u(3,ngrid), p(ngrid), as left by
 * init_conditions (init_conditions.f90:26-77) or read_hydro (read_hydro.f90:122-160).
 * adindx is set to gammafix everywhere (the value state() gives it).  u or p may be
 * NULL, meaning zero. */
int bx_upload(bx_handle *h, const double *cons, const double *u, const double *p);

/* Upload a state at a step boundary from the conserved variables alone: u is set
 * to m/rho (the loop body ends with state() and velocity(), main.f90:513-515)
 * and p to the pressure state() gives with it, which is what the reference
 * holds there when no force acted and no cell lies below rho = 1e-4 (the
 * low-density branch of state.f90:50-55 keeps a p that cons does not
 * determine: use bx_upload for such states; after a step with a force the
 * reference's p used the velocity of before source(1) -- the next step
 * recomputes p before reading it either way).  Moves 40 bytes per cell instead
 * of 72.  Fixed-gamma grids only. */
int bx_upload_conserved(bx_handle *h, const double *cons);

/* Copy the state arrays out (what write_files.f90:55-63 writes after state()).
 * Any pointer may be NULL. */
int bx_download(bx_handle *h, double *cons, double *u, double *p);

/* The main-loop clock of main.f90:102,196-199: time, dtold and step. */
int bx_set_clock(bx_handle *h, double time, double dtold, int64_t step);
int bx_get_clock(bx_handle *h, double *time, double *dt, double *dtold, int64_t *step);

/* One iteration of the main loop body (main.f90:212-545 with default flags:
 * state, courant, dt control, half-dt source, two flux stages of SSP-RK2, half-dt
 * source).  If time >= endtime the loop would have exited: nothing runs and
 * *ran = 0 (ran may be NULL). */
int bx_step(bx_handle *h, double endtime, int32_t *ran);

/* One loop iteration (main.f90:212-545) on a state held on the host: the result
 * of bx_upload_conserved(h, cons_in), bx_step(h, endtime, ran) and
 * bx_download(h, cons_out, NULL, NULL), bit for bit, with the copies overlapped
 * with the work: the upload goes in z slabs, each transposed as it lands, and the
 * second flux stage runs slab by slab while the finished slabs are converted to
 * the (5, ngrid) layout and copied back.  cons_in and cons_out may be the same
 * array; pinned (page-locked) host memory lets the copies run asynchronously.
 * A force set with bx_set_phi or bx_set_gforce applies to the step.  States the
 * fused path does not take (see bx_upload_conserved), and the tabulated EOS and
 * angular-momentum fluxing, run the three calls in sequence.  Uses the handle's reference cons array as
 * staging; returns after the result is in cons_out. */
int bx_step_host(bx_handle *h, const double *cons_in, double *cons_out, double endtime,
                 int32_t *ran);

/* Repeat bx_step until time >= endtime or nsteps steps ran. */
int bx_run(bx_handle *h, double endtime, int64_t nsteps, int64_t *steps_taken);

/* celldump files (Fortran unformatted sequential, 4-byte record markers as built
 * with -frecord-marker=4): readtest=1234, (time, step), the 8 units of
 * units.f90:10-17, then per cell (x, y, z, rho, p, u1, u2, u3, phi, E, muc, boundary).
 *
 * bx_write_celldump replaces write_files.f90:28-65 (hydro part): it applies
 * state() to the handle's arrays first (write_files.f90:32, with the same effect
 * on them), then writes the arrays with the handle's clock.  phi: ngrid host
 * doubles, or NULL for zeros (phi is zero without gravity, main.f90:185).
 *
 * bx_read_celldump replaces read_hydro.f90:122-187 plus main.f90:196-199: reads
 * rho, p, u, E, rebuilds m = u*rho, resets the outermost cell layer to
 * (small_rho, 0, 0, 0, small_eps), uploads, applies state() and sets the clock to
 * the file's time and step with dtold = 0.  phi (ngrid host doubles), time and
 * step receive the file's values when not NULL. */
int bx_write_celldump(bx_handle *h, const char *path, const double *phi);
int bx_read_celldump(bx_handle *h, const char *path, double *phi, double *time, int64_t *step);

/* Tabulated EOS (H2STAT >= 0): the tables of the reference's eos module, built on
 * the host by its own calc_eos_table (eos.f90:127-520) after initialize_eos
 * (eos.f90:30-51), in Fortran order (energy index fastest).  state() then takes
 * gamma, mu and T from them by get_gamma2 (eos.f90:653-699) as state.f90:60-79
 * does (including the disk scale-height branch for nz == 1).  Such grids run the
 * fused stage kernels (nz != 1, no force) or the per-phase kernels;
 * bx_set_eos_table must come before the first step. */
typedef struct bx_eos_table {
  int32_t neos;            /* NEOS = NEOS_T: entries per density (eng_table2 rows) */
  int32_t neos_rho;        /* NEOS_RHO */
  double log_rho_eos_low;  /* eos module log_rho_eos_low */
  double drho_eos;         /* drho_eos */
  double density_unit;     /* scl%density (units.f90:12) */
  double tk_bgrnd;         /* parameters tk_bgrnd (state.f90:74) */
  const double *eng_table2, *gamma_table2, *muc_table2, *tk_table2; /* (neos, neos_rho) */
  const double *rho_table;       /* (neos_rho) */
  const double *deng_eos_array;  /* (neos_rho) */
} bx_eos_table;
int bx_set_eos_table(bx_handle *h, const bx_eos_table *t);

/* Per-phase entry points on the handle's module arrays, for bisection against the
 * reference.  They act exactly like the subroutines they replace. */
int bx_state(bx_handle *h);                /* state.f90:6-89 (H2STAT=-1 branch) */
int bx_velocity(bx_handle *h);             /* velocity.f90:4-64 */
int bx_courant(bx_handle *h, double *dt);  /* courant.f90:4-39; sets and returns dt */
int bx_source(bx_handle *h, int32_t siter);/* source.f90:5-205 (gravity coupling via gforce) */
int bx_ghost(bx_handle *h);                /* utils.f90:305-480 set_ghost_cells */
int bx_flux(bx_handle *h, int32_t avg);    /* flux.f90:6-235 */
int bx_avisc(bx_handle *h);                /* avisc.f90:4-26 into the handle's qq array;
                                              the reference never calls it or reads qq */
int bx_save_cons_old(bx_handle *h);        /* main.f90:327-333 */
/* The hydro namelist's avmagx, avmagy, avmagz (input.f90:12, parameters.f90:77; all 0 by
 * default) for bx_avisc. */
int bx_set_avmag(bx_handle *h, double avmagx, double avmagy, double avmagz);
/* The artificial-viscosity array qq(3,ngrid) (grid_commons.f90:14), host layout: what the
 * last bx_avisc computed, zero before the first (init_grid.f90:298).  qq is computed
 * as avisc.f90:13-23 writes it: qq(d) = avmag_d*min(0, u_d(+) - u_d(-))**2 on the cells
 * with boundary > 0, the ghost layers (the reference's test, kept as written), and 0
 * on the interior cells; neighbours in a ghost layer resolve to the cell itself
 * (get_boundary, utils.f90:62-73), and so do the five neighbour slots that
 * init_grid.f90:178 leaves at 0 for the outer ghost layer (the reference reads
 * grid(0) there, outside the array). */
int bx_download_qq(bx_handle *h, double *qq);
int bx_set_dt(bx_handle *h, double dt);    /* the module variable dt (grid_commons.f90:12) */

/* Gravitational acceleration gforce(3,ngrid) consumed by source() (source.f90:161-182);
 * NULL restores the zero force of a run without a gravity solver. */
int bx_set_gforce(bx_handle *h, const double *gforce);

/* The gravity coupling of a run with a potential solver (main.f90:143-149,477-483
 * under USEPOTENTIAL): phi(ngrid) from the host's solver, turned into gforce on the
 * device by calc_gforce (utils.f90:549-571, central differences on interior cells).
 * Call it whenever the solver updates phi (each step); NULL removes the force.
 * Both sources of the next step apply the force; grids the fused path takes run
 * it in the stage kernels. */
int bx_set_phi(bx_handle *h, const double *phi);

/* Status bits accumulated since the last call (BX_STATUS_*) and the path the
 * last step took (0 = per-phase kernels, 1 = fused stage kernels). */
int bx_status(bx_handle *h, uint32_t *status_bits, int32_t *last_path);

/* Device pointers of the current conserved planes (5 x ngrid doubles, SoA) for
 * zero-copy users; valid until the next call on the handle. */
int bx_device_cons(bx_handle *h, double **cons_soa, int64_t *ngrid);

/* Timing hooks: with profiling on, every fused step records CUDA events around
 * its two stage kernels on the handle's stream; bx_profile_read returns the
 * accumulated stage times (ms), the number of fused steps timed and the number
 * of this library's kernels launched since bx_profile was called. */
int bx_profile(bx_handle *h, int32_t enable);
int bx_profile_read(bx_handle *h, double *ms_stage0, double *ms_stage1, int64_t *fused_steps,
                    int64_t *launches);
/* Timeline of bx_step_host (a measurement aid): with enable != 0, each call records
 * CUDA events per slab of its pipeline.  bx_step_host_timeline with ms == NULL sets
 * *nslabs to the slab count; with ms of at least 7 x *nslabs doubles it fills, per
 * slab k, ms[7k..7k+6] = milliseconds from the call's start to: upload start,
 * upload end, the end of the stage-0 launches enqueued after that upload, the
 * slab's stage-1 end, its conversion to the host layout, download start, download
 * end (-1 where the last call recorded no such event). */
int bx_step_host_profile(bx_handle *h, int32_t enable);
int bx_step_host_timeline(bx_handle *h, int32_t *nslabs, double *ms);

/* Host-only query (no GPU needed): the ghost-fill plan bx_create builds for a grid.
 * For each ghost cell in index order: dst = cell, src1/sgn1 = source cell and
 * momentum sign mask (bit0 m1, bit1 m2, bit2 m3 negated) of one set_ghost_cells
 * sweep (utils.f90:305-480) with all sources read before the sweep; src2/sgn2 =
 * the same for two consecutive sweeps.  Call with dst==NULL to get *nghost;
 * *fused_ok is 1 when the fused stage kernels can run on this grid. */
int bx_ghost_plan(const bx_params *params, int64_t *nghost, int32_t *dst, int32_t *src1,
                  uint8_t *sgn1, int32_t *src2, uint8_t *sgn2, int32_t *fused_ok);

/* ---- Batched ensembles.  No counterpart in the reference, which advances one grid
 * per process.  Many independent grids ("boxes", each with its own size, gamma, cfl,
 * dt and clock) advance together: one tile list spans all boxes, a step is four
 * launches for the whole ensemble, and a run of n steps is replayed as one CUDA
 * graph.  Each box evolves bit for bit as it would under bx_step on its own.  Boxes
 * must be fused-eligible (bx_ghost_plan fused_ok) and all 3-D (nz>=6) or all 2-D;
 * an uploaded state must be one the fused stages start from (interior rho >= 1e-4,
 * u == m/rho, ghosts equal to the two-sweep fill), else BX_ERR_STATE.  A box whose
 * step fires the velocity limiter or the low-density EOS branch continues on a
 * single-grid handle of its own after the run. */
typedef struct bx_batch bx_batch;
int bx_batch_create(int32_t nbox, const bx_params *params, bx_batch **out);
int bx_batch_destroy(bx_batch *b);
int bx_batch_set_stream(bx_batch *b, void *cuda_stream);
int bx_batch_upload(bx_batch *b, int32_t box, const double *cons);
int bx_batch_set_clock(bx_batch *b, int32_t box, double time, double dtold, int64_t step);
int bx_batch_get_clock(bx_batch *b, int32_t box, double *time, double *dt, double *dtold,
                       int64_t *step);
/* nsteps iterations of every box's main loop (boxes at endtime stop).  use_graph != 0:
 * the run is captured once into a CUDA graph and replayed.  The launches are four per
 * step (dt, stage 0, stage 1, clock), or, in persistent mode (bx_batch_set_persistent,
 * or chosen by bx_batch_autotune), one launch for the whole run after the first
 * step's dt: its blocks take (step, stage, tile) items from a queue in step order and
 * wait for what an item reads (a stage-0 tile for its box's dt, a stage-1 tile for
 * every stage-0 tile of its box), each wait bounded by a poll limit (BX_ERR_STATE
 * if one gave up).  Both forms give the same results bit for bit. */
int bx_batch_run(bx_batch *b, int64_t nsteps, double endtime, int32_t use_graph);
int bx_batch_set_persistent(bx_batch *b, int32_t enable);
/* Tile shape of the stage kernels for the ensemble: 0 = 32 x 8 columns, 1 = 16 x 16
 * (both in 256-thread blocks); bx_batch_autotune picks it.  The getter also gives the
 * shape's extents and the tile depth (as bx_batch_autotune's zc). */
int bx_batch_set_tile_shape(bx_batch *b, int32_t shape);
int bx_batch_get_tile_shape(bx_batch *b, int32_t *shape, int32_t *tx, int32_t *ty,
                            int32_t *depth);
int bx_batch_get_persistent(bx_batch *b, int32_t *enabled);
/* The bounded wait of the persistent launch, run on a counter that nothing advances
 * with the given poll limit: *gave_up = 1 when the wait ended without it (the limit
 * ran out), *ms its device time.  A check of the limit that needs no fault. */
int bx_batch_wait_selftest(int64_t poll_limit, int32_t *gave_up, double *ms);
/* Run configuration of the ensemble picked by measurement: every candidate tile shape
 * (32 x 8, 16 x 16) and tile depth (the default rule, whole box depths, 64, 32, 16, 8
 * planes) runs reps trial steps from the boxes' current states, which the trials leave
 * unchanged (inputs are not overwritten; clocks are restored), and the fastest is kept
 * for the following runs; with it the persistent launch is timed too and kept if
 * faster (bx_batch_get_persistent, bx_batch_get_tile_shape).  *zc = the chosen depth
 * (0 = default rule, >= 2^30 = whole depths), *ms = its trial step time.  Results do
 * not depend on any of them. */
int bx_batch_autotune(bx_batch *b, int32_t reps, int32_t *zc, double *ms);
int bx_batch_download(bx_batch *b, int32_t box, double *cons, double *u, double *p);
/* device time of the last run (ms), kernels it launched, boxes running on their own
 * handles, cells in the pool */
int bx_batch_info(bx_batch *b, double *last_run_ms, int64_t *launches, int32_t *n_solo,
                  int64_t *cells);
const char *bx_batch_last_error(bx_batch *b);

/* ---- Discrete adjoint.  No counterpart in the reference.  Reverse-mode derivative
 * of an nsteps-step run of the fused stage arithmetic (the step of bx_step), with the
 * dt sequence of the forward run held fixed and every limiter/max/min branch taken as
 * in the forward.  Grids: fixed gamma, no flux_ang, face ghosts on the donor rule of
 * the stage kernels.  Where the two-sweep ghost plan leaves corner ghosts lagging
 * (reflective 3-D boxes), which enter only the Courant maximum, an unfrozen forward
 * first runs the per-phase kernels from cons0 to take their dt sequence (its time is
 * part of the forward's).  Device arrays are SoA planes (5 x ngrid doubles, rho, m1,
 * m2, m3, E) of the reference cons; ghost entries of the inputs are ignored (the run
 * starts with the ghosts two calls of the fill give) and those of gradients are zero.
 * The forward refuses runs in which the velocity limiter or the low-density branch
 * fires (BX_ERR_STATE).  Snapshots follow a binomial schedule in `snapshots` plane
 * sets. */
typedef struct bx_adj bx_adj;
int bx_adj_create(const bx_params *params, int64_t nsteps, int32_t snapshots, bx_adj **out);
int bx_adj_destroy(bx_adj *a);
int bx_adj_set_stream(bx_adj *a, void *cuda_stream);
/* enable != 0: the next unfrozen forward keeps the stage-0 result of every step
 * (nsteps x 5 x ngrid doubles more), and backward passes use them instead of
 * recomputing stage 0 of each step; BX_ERR_NOMEM if they do not fit. */
int bx_adj_keep_stage0(bx_adj *a, int32_t enable);
/* Entries (>= 2, default 2; 5 x ngrid doubles each) of the cache of stage-0
 * results the backward pass keeps from the last step of each recompute advance,
 * so the reverse of that step skips its stage-0 recompute; more entries keep
 * results for longer.  BX_ERR_NOMEM if they do not fit. */
int bx_adj_stage0_cache(bx_adj *a, int32_t entries);
/* Host level of the checkpoint schedule.  stride >= 2: the next unfrozen forward
 * copies the state of steps stride, 2 stride, ... (below nsteps) into pinned host
 * memory, on a copy stream beside the step kernels (the forward's time includes
 * the copies), and backward passes reverse the segments between those steps from
 * the last to the first, each with the device snapshots; the start of the next
 * segment is copied back while the current one is reversed.  Two of the
 * `snapshots` plane sets hold segment starts, so snapshots >= 3.  A segment of
 * stride steps with at least stride - 1 free plane sets recomputes each of its
 * states once.  stride = 0 (or >= nsteps) turns the level off and frees the host
 * memory.  *host_bytes (may be NULL) receives the pinned bytes.  BX_ERR_NOMEM
 * when they exceed half of the host's available memory (/proc/meminfo) or the
 * allocation fails.  No reference counterpart (the reference has no adjoint). */
int bx_adj_host_level(bx_adj *a, int64_t stride, int64_t *host_bytes);
/* frozen=0: dt by the CFL rule (main.f90:266-281) and recorded; frozen=1: the recorded
 * dt sequence (for finite differences).  BX_ERR_STATE if a guard fired. */
int bx_adj_forward(bx_adj *a, const double *cons0, double *consT, int32_t frozen);
/* lam0 = (d consT / d cons0)^T lamT for the last unfrozen forward run */
int bx_adj_backward(bx_adj *a, const double *lamT, double *lam0);
int bx_adj_stats(bx_adj *a, double *ms_forward, double *ms_backward, int64_t *recomputed_steps,
                 int64_t *device_bytes);
/* Host only (no device, no handle): the checkpoint schedule of an nsteps run with
 * `snapshots` plane sets, for choosing the snapshot count before allocating.
 * recomputed_first: forward steps the first bx_adj_backward after an unfrozen
 * forward recomputes (bx_adj_stats' recomputed_steps); recomputed_again: those of a
 * further backward of the same run; chain_snapshots: snapshots the forward run
 * stores on its way.  Any output may be NULL. */
int bx_adj_plan(int64_t nsteps, int32_t snapshots, int64_t *recomputed_first,
                int64_t *recomputed_again, int32_t *chain_snapshots);
/* Host only: the device bytes an engine for this grid holds (bx_adj_stats'
 * device_bytes) with `snapshots` plane sets, `stage0_cache_entries` cache
 * entries (>= 2; bx_adj_stage0_cache) and the stage-0 results of every step kept
 * or not (bx_adj_keep_stage0), to size a run to the device before allocating.
 * The handle beneath the engine adds its ghost tables and tile list.  Grids that
 * bx_adj_create refuses are refused here too: BX_ERR_ARG beyond 2^31 cells,
 * BX_ERR_UNSUPPORTED for grids off the fused stage kernels (checked on the host
 * by building the grid's ghost plan). */
int bx_adj_device_bytes(const bx_params *params, int64_t nsteps, int32_t snapshots,
                        int32_t stage0_cache_entries, int32_t keep_stage0, int64_t *bytes);
int bx_adj_dts(bx_adj *a, double *dts);
/* The last unfrozen forward run, with its dt sequence, from two initial states at once
 * (device SoA planes as for bx_adj_forward): a base state and a perturbed one.  Every
 * max/min, floor, limiter selection and HLL wave-speed choice of the perturbed run is
 * the one the base run makes (by the rules the backward pass differentiates), so the
 * perturbed run is smooth in its input; central differences of it, with the base the
 * unperturbed state, check bx_adj_backward where the step itself is not differentiable
 * (limiter and wave-speed ties).  consT_base equals bx_adj_forward's consT on the
 * interior cells bit for bit; ghost entries of both outputs are zero.  Uses the engine's
 * work planes (like a frozen bx_adj_forward), not its snapshots. */
int bx_adj_forward_branches(bx_adj *a, const double *cons_base0, const double *cons_pert0,
                            double *consT_base, double *consT_pert);
const char *bx_adj_last_error(bx_adj *a);

/* No counterpart in the reference.  One set_ghost_cells sweep -- the same result as
 * bx_ghost -- that allocates nothing, for callers that cannot allocate device memory
 * (a host program that has reserved the device's memory for its own pool, or a
 * runtime held to a fixed device-memory budget).  The caller passes device memory it
 * owns: the conserved planes cons_soa (5 x ngrid doubles, SoA, updated in place) and
 * the sweep plan dst/src/sgn of bx_ghost_plan (src1, sgn1).  The gather scratch is a
 * static device array of BX_NOALLOC_MAX_GHOSTS x 5 doubles (40 MiB) that every GPU
 * loading the library holds until exit; larger nghost is rejected with BX_ERR_ARG.
 * The first call on a device looks up that array's device address (make it before
 * any stream capture), and so does the first call after another CUDA context became
 * current on the device (cudaDeviceReset, or a context of the caller's own); calls
 * that overlap on the GPU race on the shared array.  Errors are reported by
 * bx_noalloc_last_error, per host thread. */
#define BX_NOALLOC_MAX_GHOSTS 1048576
int bx_ghost_fill_noalloc(double *cons_soa, int64_t ngrid, const int32_t *dst,
                          const int32_t *src, const uint8_t *sgn, int64_t nghost,
                          void *cuda_stream);
const char *bx_noalloc_last_error(void);

/* Message of the last error on the handle (or, when h is NULL, of the calling thread's
 * last failed bx_create; bx_batch_last_error(NULL) and bx_adj_last_error(NULL) likewise
 * report the calling thread's last failed bx_batch_create / bx_adj_create). */
const char *bx_last_error(bx_handle *h);

#ifdef __cplusplus
}
#endif
#endif /* BOXZY_GPU_H */

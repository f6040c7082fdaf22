/*
 * bx_oracle.h -- CPU restatement of BOXZYHYDRO's fixed-gamma hydrodynamic step.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker for the CUDA path
 * (tests/, __graft_entry__.smoke() and the cpu_baseline leg of bench.py use it);
 * the product never links or calls it.
 *
 * Parity status: the reference (Fortran 95, gfortran) cannot be compiled in
 * this image (no Fortran front end), so per-step parity of this restatement is
 * NOT pinned by a reference binary.  End states are pinned against the
 * reference's own golden files (analysis/sod.ana exact Sod solution and
 * analysis/sodtest.dat reference output) by tests/test_oracle_golden.py.
 *
 * Every routine follows the reference file:line given in bx_oracle.c, in the
 * same evaluation order, compiled with -ffp-contract=off (no FMA contraction,
 * no reassociation), which is how gfortran -O3 evaluates the same expressions
 * on x86-64 without -march (SSE2, no FMA instructions).
 *
 * Layout follows the reference exactly: cons(5,ngrid) column-major = AoS with
 * 5 doubles per cell, u(3,ngrid) AoS, p/adindx/muc_array(ngrid); cell index
 * igrid = ix + (iy-1)*nx + (iz-1)*nx*ny (1-based in Fortran, 0-based here).
 */
#ifndef BX_ORACLE_H
#define BX_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct ox_params {
  int32_t nx, ny, nz;
  int32_t h2stat;          /* -1 fixed gamma; >= 0 tables (ox_set_eos_table) */
  double dx, dy, dz;
  double cfl, small_rho, small_eps, vlimit, gammafix;
  double muc, rgas;        /* eos.f90:144 and units.f90:17 */
  int32_t no_outflow[6];   /* xl, xr, yl, yr, zl, zr (parameters.f90:32-37) */
  int32_t racy_ghosts;     /* 1: parallel ghost loop like the reference (timing only) */
  int32_t pad;
  int32_t fluxangmom;      /* parameters.f90:31: flux_ang.f90 in place of flux.f90 */
  int32_t pad2;
  double yoffset;          /* parameters.f90:30 */
} ox_params;

typedef struct ox_sim ox_sim;

/* tables of the eos module for H2STAT >= 0 (eos.f90:30-51), energy index fastest */
typedef struct ox_eos_table {
  int32_t neos, neos_rho;
  double log_rho_eos_low, drho_eos, density_unit, tk_bgrnd;
  const double *eng_table2, *gamma_table2, *muc_table2, *tk_table2;
  const double *rho_table, *deng_eos_array;
} ox_eos_table;
/* copies the tables; state() then follows state.f90:60-79 */
void ox_set_eos_table(ox_sim *s, const ox_eos_table *t);
void ox_get_muc(const ox_sim *s, double *muc);

ox_sim *ox_create(const ox_params *p);
void ox_destroy(ox_sim *s);
int64_t ox_ngrid(const ox_sim *s);
int64_t ox_nghost(const ox_sim *s);
void ox_grid_info(const ox_sim *s, int32_t *boundary, int32_t *ineigh6);
void ox_ghost_list(const ox_sim *s, int64_t *idx);

/* state arrays (reference layout) */
void ox_set_state(ox_sim *s, const double *cons5, const double *u3, const double *p,
                  const double *adindx);
void ox_get_state(const ox_sim *s, double *cons5, double *u3, double *p, double *adindx);
void ox_set_gforce(ox_sim *s, const double *g3);
void ox_get_cons_old(const ox_sim *s, double *cons5);
void ox_set_cons_old(ox_sim *s, const double *cons5);

/* clock: time, dt, dtold and step of main.f90 */
void ox_set_clock(ox_sim *s, double time, double dt, double dtold, int64_t step);
void ox_get_clock(const ox_sim *s, double *time, double *dt, double *dtold, int64_t *step,
                  double *dtrate);

/* phases (argument-less subroutines of the reference, acting on the arrays) */
void ox_state(ox_sim *s);
void ox_velocity(ox_sim *s);
void ox_courant(ox_sim *s);
void ox_source(ox_sim *s, int siter);
void ox_set_ghost_cells(ox_sim *s);
void ox_flux(ox_sim *s, int avg);
void ox_flux_ang(ox_sim *s, int avg); /* flux_ang.f90:6-281 */
void ox_save_cons_old(ox_sim *s);
/* avisc.f90:4-26: qq(3,ngrid) (host layout) from the velocity array u */
void ox_avisc(const ox_sim *s, double avmagx, double avmagy, double avmagz, double *qq);

/* one iteration of the main loop (main.f90:212-545); returns 0 if it ran,
 * 1 if the loop would have exited (time>=endtime). */
int ox_step(ox_sim *s, double endtime);
/* one iteration with the full step dt given (dt sequence held fixed) */
void ox_step_dt(ox_sim *s, double dt_full);
/* run until time>=endtime or nsteps steps were taken; returns steps taken */
int64_t ox_run(ox_sim *s, double endtime, int64_t nsteps);

void ox_set_threads(int n);

/* constants of the reference's units module and EOS */
double ox_rgas_code_units(void);   /* units.f90:10-17 */
double ox_muc(double xabun, double yabun, double zabun, double mu_z); /* eos.f90:144 */

/* Known-answer probes (tests only): genminmod (utils.f90:696-707), slope with
 * theta = SLOPE_THETA (utils.f90:738-741), interface_muscl (flux.f90:299-308) and
 * the HLL flux of one face (flux.f90:513-590) from left/right reconstructed
 * states (rho, u1, u2, u3, p, eps, gamma). */
double ox_kat_genminmod(double x1, double x2, double x3);
double ox_kat_slope(double c0, double c1, double c2);
void ox_kat_muscl(double q, double lm, double lp, double sl, double *minus, double *plus);
void ox_kat_face_flux(const double *left7, const double *right7, int idir, double *f5);

#ifdef __cplusplus
}
#endif
#endif

/*
 * bx_oracle.c -- CPU restatement of BOXZYHYDRO's hydrodynamic step (fixed gamma).
 *
 * TEST INFRASTRUCTURE ONLY: the checker for the CUDA path.  Nothing in the
 * product links or calls this file.  Per-step parity is unpinned by a reference
 * binary (no Fortran compiler in this image); end states are pinned against the
 * reference's golden files analysis/sod.ana and analysis/sodtest.dat.
 *
 * Build: gcc -O2 -ffp-contract=off -fopenmp (see Makefile).  No -ffast-math:
 * every expression below is evaluated in the order the Fortran source writes it,
 * with x**2 as x*x and Fortran's left-to-right association of + - * /.
 *
 * Ghost fill: the reference fills ghosts inside an OpenMP DO loop, where corner
 * ghosts may read other ghosts that another thread has or has not yet updated
 * (utils.f90:215 tests iz>=6 where nz>=6 is meant; reflective walls read
 * ghosts three cells inward).  This restatement defines the ghost fill as the
 * single-threaded loop in index order (OMP_NUM_THREADS=1 behaviour), which is
 * deterministic.  racy_ghosts=1 runs the loop in parallel exactly like the
 * reference (used only for CPU timing, never for checking).
 */
#include "bx_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define ZERO 0.0
#define ONE 1.0
#define TWO 2.0
#define HALF (ONE / TWO)     /* parameters.f90:143 */
#define THETA 1.25           /* -DSLOPE_THETA=1.25, Makefile:20, utils.f90:739 */

struct ox_sim {
  ox_params P;
  int64_t ng, nghost, nbound;
  int32_t *bnd, *ix, *iy, *iz;
  int64_t *ineigh;   /* 6 per cell, 0-based, -1 = unset */
  int64_t *indx_ghost, *indx_bound;
  double *cons, *cons_old, *fluxtmp, *u, *p, *adindx, *muc_array, *gforce;
  double *slope_u, *slope_p, *slope_d, *slope_e, *slope_g;             /* (3[,3],ng) */
  double *st_u_p, *st_u_m, *st_p_p, *st_p_m, *st_d_p, *st_d_m, *st_e_p, *st_e_m, *st_g_p,
      *st_g_m;
  /* flux_ang: slopes and states of the transformed momenta (init_grid.f90:56-63) */
  double *slope_rmom, *slope_amom, *st_rmom_p, *st_rmom_m, *st_amom_p, *st_amom_m;
  double time, dt, dtold, dtrate, maxv;
  int64_t step;
  /* eos module tables (H2STAT >= 0) */
  int32_t neos, neos_rho;
  double log_rho_eos_low, drho_eos, density_unit, tk_bgrnd;
  double *eng_table2, *gamma_table2, *muc_table2, *tk_table2, *rho_table, *deng_eos_array;
};

static inline double fmax_f(double a, double b) { return a > b ? a : b; }
static inline double fmin_f(double a, double b) { return a < b ? a : b; }

/* init_grid.f90:7-265 -- flags, donor/neighbour table, ghost list */
ox_sim *ox_create(const ox_params *prm) {
  ox_sim *s = (ox_sim *)calloc(1, sizeof(ox_sim));
  s->P = *prm;
  const int nx = prm->nx, ny = prm->ny, nz = prm->nz;
  const int64_t ng = (int64_t)nx * ny * nz;
  s->ng = ng;
  if (nz < 6) { /* init_grid.f90:76-79 */
    s->P.no_outflow[4] = 0;
    s->P.no_outflow[5] = 0;
  }
  s->bnd = (int32_t *)calloc(ng, sizeof(int32_t));
  s->ix = (int32_t *)calloc(ng, sizeof(int32_t));
  s->iy = (int32_t *)calloc(ng, sizeof(int32_t));
  s->iz = (int32_t *)calloc(ng, sizeof(int32_t));
  s->ineigh = (int64_t *)malloc(ng * 6 * sizeof(int64_t));
  s->cons = (double *)calloc(ng * 5, sizeof(double));
  s->cons_old = (double *)calloc(ng * 5, sizeof(double));
  s->fluxtmp = (double *)calloc(ng * 5, sizeof(double));
  s->u = (double *)calloc(ng * 3, sizeof(double));
  s->gforce = (double *)calloc(ng * 3, sizeof(double));
  s->p = (double *)calloc(ng, sizeof(double));
  s->adindx = (double *)calloc(ng, sizeof(double));
  s->muc_array = (double *)calloc(ng, sizeof(double));
  s->slope_u = (double *)calloc(ng * 9, sizeof(double));
  s->st_u_p = (double *)calloc(ng * 9, sizeof(double));
  s->st_u_m = (double *)calloc(ng * 9, sizeof(double));
  double **a3[] = {&s->slope_p, &s->slope_d, &s->slope_e, &s->slope_g, &s->st_p_p, &s->st_p_m,
                   &s->st_d_p, &s->st_d_m, &s->st_e_p, &s->st_e_m, &s->st_g_p, &s->st_g_m,
                   &s->slope_rmom, &s->slope_amom, &s->st_rmom_p, &s->st_rmom_m,
                   &s->st_amom_p, &s->st_amom_m};
  for (unsigned k = 0; k < sizeof(a3) / sizeof(a3[0]); ++k)
    *a3[k] = (double *)calloc(ng * 3, sizeof(double));

  int64_t nghost = 0, nbound = 0;
  int64_t igrid = 0;
  for (int iz = 1; iz <= nz; ++iz) {
    int f1z = 0, f2z = 0;
    if (nz >= 6) {
      if (iz == 1 || iz == nz) f1z = 1;
      if (iz == 2 || iz == nz - 1) f2z = 1;
    }
    for (int iy = 1; iy <= ny; ++iy) {
      int f1y = (iy == 1 || iy == ny), f2y = (iy == 2 || iy == ny - 1);
      for (int ix = 1; ix <= nx; ++ix, ++igrid) {
        int f1x = (ix == 1 || ix == nx), f2x = (ix == 2 || ix == nx - 1);
        int f1 = f1z + f1x + f1y, f2 = f2z + f2x + f2y;
        s->bnd[igrid] = 0;
        if (f1 > 0) {
          s->bnd[igrid] = 1;
          nbound++;
          nghost++;
        } else if (f2 > 0) {
          s->bnd[igrid] = 2;
          nghost++;
        }
        s->ix[igrid] = ix;
        s->iy[igrid] = iy;
        s->iz[igrid] = iz;
      }
    }
  }
  s->nghost = nghost;
  s->nbound = nbound;
  s->indx_ghost = (int64_t *)malloc((nghost ? nghost : 1) * sizeof(int64_t));
  s->indx_bound = (int64_t *)malloc((nbound ? nbound : 1) * sizeof(int64_t));
  const int64_t sx = 1, sy = nx, sz = (int64_t)nx * ny;
  int64_t ib = 0, ib2 = 0;
  for (igrid = 0; igrid < ng; ++igrid) {
    int64_t *nb = s->ineigh + igrid * 6;
    for (int k = 0; k < 6; ++k) nb[k] = -1;
    int ix = s->ix[igrid], iy = s->iy[igrid], iz = s->iz[igrid];
    if (s->bnd[igrid] == 1) {
      s->indx_bound[ib++] = igrid;
      s->indx_ghost[ib2++] = igrid;
      /* init_grid.f90:180-203: outer ghost keeps its donor in ineigh(1) */
      if (ix == 1) nb[0] = igrid + 2 * sx;
      else if (ix == nx) nb[0] = igrid - 2 * sx;
      else if (iy == 1) nb[0] = igrid + 2 * sy;
      else if (iy == ny) nb[0] = igrid - 2 * sy;
      else if (iz == 1) nb[0] = (nz < 6) ? igrid : igrid + 2 * sz;
      else nb[0] = (nz < 6) ? igrid : igrid - 2 * sz;
    } else {
      if (s->bnd[igrid] == 2) s->indx_ghost[ib2++] = igrid;
      /* init_grid.f90:237-261: ineigh(1)=+y,(2)=-y,(3)=+x,(4)=-x,(5)=+z,(6)=-z */
      nb[0] = igrid + sy;
      nb[1] = igrid - sy;
      nb[2] = igrid + sx;
      nb[3] = igrid - sx;
      if (nz < 6) {
        nb[4] = igrid;
        nb[5] = igrid;
      } else {
        nb[4] = igrid + sz;
        nb[5] = igrid - sz;
      }
    }
  }
  s->time = 0;
  s->dt = 0;
  s->dtold = 0;
  s->step = 0;
  return s;
}

void ox_destroy(ox_sim *s) {
  if (!s) return;
  void *ptrs[] = {s->bnd, s->ix, s->iy, s->iz, s->ineigh, s->indx_ghost, s->indx_bound,
                  s->cons, s->cons_old, s->fluxtmp, s->u, s->p, s->adindx, s->muc_array,
                  s->gforce, s->slope_u, s->slope_p, s->slope_d, s->slope_e, s->slope_g,
                  s->st_u_p, s->st_u_m, s->st_p_p, s->st_p_m, s->st_d_p, s->st_d_m,
                  s->st_e_p, s->st_e_m, s->st_g_p, s->st_g_m, s->slope_rmom, s->slope_amom,
                  s->st_rmom_p, s->st_rmom_m, s->st_amom_p, s->st_amom_m,
                  s->eng_table2, s->gamma_table2, s->muc_table2, s->tk_table2, s->rho_table,
                  s->deng_eos_array};
  for (unsigned k = 0; k < sizeof(ptrs) / sizeof(ptrs[0]); ++k) free(ptrs[k]);
  free(s);
}

int64_t ox_ngrid(const ox_sim *s) { return s->ng; }
int64_t ox_nghost(const ox_sim *s) { return s->nghost; }
void ox_grid_info(const ox_sim *s, int32_t *boundary, int32_t *ineigh6) {
  for (int64_t i = 0; i < s->ng; ++i) {
    if (boundary) boundary[i] = s->bnd[i];
    if (ineigh6)
      for (int k = 0; k < 6; ++k) ineigh6[i * 6 + k] = (int32_t)s->ineigh[i * 6 + k];
  }
}
void ox_ghost_list(const ox_sim *s, int64_t *idx) {
  memcpy(idx, s->indx_ghost, s->nghost * sizeof(int64_t));
}

void ox_set_state(ox_sim *s, const double *c, const double *u, const double *p,
                  const double *g) {
  if (c) memcpy(s->cons, c, s->ng * 5 * sizeof(double));
  if (u) memcpy(s->u, u, s->ng * 3 * sizeof(double));
  if (p) memcpy(s->p, p, s->ng * sizeof(double));
  if (g) memcpy(s->adindx, g, s->ng * sizeof(double));
}
void ox_get_state(const ox_sim *s, double *c, double *u, double *p, double *g) {
  if (c) memcpy(c, s->cons, s->ng * 5 * sizeof(double));
  if (u) memcpy(u, s->u, s->ng * 3 * sizeof(double));
  if (p) memcpy(p, s->p, s->ng * sizeof(double));
  if (g) memcpy(g, s->adindx, s->ng * sizeof(double));
}
void ox_set_gforce(ox_sim *s, const double *g3) {
  if (g3) memcpy(s->gforce, g3, s->ng * 3 * sizeof(double));
  else memset(s->gforce, 0, s->ng * 3 * sizeof(double));
}
void ox_get_cons_old(const ox_sim *s, double *c) {
  memcpy(c, s->cons_old, s->ng * 5 * sizeof(double));
}
void ox_set_cons_old(ox_sim *s, const double *c) {
  memcpy(s->cons_old, c, s->ng * 5 * sizeof(double));
}
void ox_set_clock(ox_sim *s, double time, double dt, double dtold, int64_t step) {
  s->time = time;
  s->dt = dt;
  s->dtold = dtold;
  s->step = step;
}
void ox_get_clock(const ox_sim *s, double *time, double *dt, double *dtold, int64_t *step,
                  double *dtrate) {
  if (time) *time = s->time;
  if (dt) *dt = s->dt;
  if (dtold) *dtold = s->dtold;
  if (step) *step = s->step;
  if (dtrate) *dtrate = s->dtrate;
}
void ox_set_threads(int n) {
#ifdef _OPENMP
  omp_set_num_threads(n);
#else
  (void)n;
#endif
}

/* units.f90:10-17 (get_units): scale%rgas in code units */
double ox_rgas_code_units(void) {
  const double pi = 3.1415926535897931;      /* parameters.f90:11 */
  const double rgasCGS = 8.254e7;            /* parameters.f90:9 */
  double length = 1.496e13;
  double time = (3600.0 * 365.25 * 24.0) / (TWO * pi);
  double vel = length / time;
  double kelvin = ONE;
  return rgasCGS / ((vel * vel) / kelvin);
}
/* eos.f90:144 */
double ox_muc(double xabun, double yabun, double zabun, double mu_z) {
  return ONE / (xabun * HALF + yabun * 0.25 + zabun / mu_z);
}

/* ---------------------------------------------------------------- state.f90:29-87 */
void ox_set_eos_table(ox_sim *s, const ox_eos_table *t) {
  const int64_t n2 = (int64_t)t->neos * t->neos_rho;
  double **dst[4] = {&s->eng_table2, &s->gamma_table2, &s->muc_table2, &s->tk_table2};
  const double *src[4] = {t->eng_table2, t->gamma_table2, t->muc_table2, t->tk_table2};
  for (int k = 0; k < 4; ++k) {
    free(*dst[k]);
    *dst[k] = (double *)malloc(n2 * sizeof(double));
    memcpy(*dst[k], src[k], n2 * sizeof(double));
  }
  free(s->rho_table);
  free(s->deng_eos_array);
  s->rho_table = (double *)malloc(t->neos_rho * sizeof(double));
  s->deng_eos_array = (double *)malloc(t->neos_rho * sizeof(double));
  memcpy(s->rho_table, t->rho_table, t->neos_rho * sizeof(double));
  memcpy(s->deng_eos_array, t->deng_eos_array, t->neos_rho * sizeof(double));
  s->neos = t->neos;
  s->neos_rho = t->neos_rho;
  s->log_rho_eos_low = t->log_rho_eos_low;
  s->drho_eos = t->drho_eos;
  s->density_unit = t->density_unit;
  s->tk_bgrnd = t->tk_bgrnd;
}
void ox_get_muc(const ox_sim *s, double *muc) {
  memcpy(muc, s->muc_array, s->ng * sizeof(double));
}

/* eos.f90:653-699 get_gamma2; tables (ientry, irho) 1-based, ientry fastest */
static void get_gamma2(const ox_sim *s, double *eps, double rho, double *tk, double *m,
                       double *gam) {
#define TAB(t, ie, ir) (t)[((ie) - 1) + (int64_t)((ir) - 1) * s->neos]
  int irho = (int)((log10(rho * s->density_unit) - s->log_rho_eos_low) / s->drho_eos) + 1;
  if (irho > s->neos_rho) irho = s->neos_rho;
  if (irho < 1) irho = 1;
  int irhop = irho + 1;
  if (irhop > s->neos_rho) irhop = irho;
  double eng = *eps / rho;
  int ientry =
      (int)((log10(eng) - log10(TAB(s->eng_table2, 1, irho))) / s->deng_eos_array[irho - 1]) + 1;
  if (ientry > s->neos - 1) {
    ientry = s->neos - 1;
    eng = TAB(s->eng_table2, s->neos, irho);
    *eps = eng * rho;
  }
  if (ientry < 1 || eng < TAB(s->eng_table2, 1, irho)) {
    ientry = 1;
    eng = TAB(s->eng_table2, 1, irho);
    *eps = eng * rho;
  }
  const double *E = s->eng_table2;
#define LIN(t, ir)                                                                        \
  (TAB(t, ientry, ir) + (TAB(t, ientry + 1, ir) - TAB(t, ientry, ir)) /                  \
                            (TAB(E, ientry + 1, ir) - TAB(E, ientry, ir)) *              \
                            (eng - TAB(E, ientry, ir)))
  *gam = LIN(s->gamma_table2, irho);
  *m = LIN(s->muc_table2, irho);
  *tk = LIN(s->tk_table2, irho);
  if (!(s->rho_table[irho - 1] == s->rho_table[irhop - 1])) {
    const double gamp = LIN(s->gamma_table2, irhop), mp = LIN(s->muc_table2, irhop),
                 tkp = LIN(s->tk_table2, irhop);
    const double slope =
        ONE / (s->rho_table[irhop - 1] - s->rho_table[irho - 1]) * (rho - s->rho_table[irho - 1]);
    *gam = *gam + (gamp - *gam) * slope;
    *m = *m + (mp - *m) * slope;
    *tk = *tk + (tkp - *tk) * slope;
  }
#undef LIN
#undef TAB
}

void ox_state(ox_sim *s) {
  const double gam = s->P.gammafix, muc = s->P.muc, rgas = s->P.rgas, seps = s->P.small_eps;
  double *c = s->cons, *u = s->u, *p = s->p;
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < s->ng; ++i) {
    double *ci = c + 5 * i, *ui = u + 3 * i;
    double ekin = ci[0] * HALF * (ui[0] * ui[0] + ui[1] * ui[1] + ui[2] * ui[2]);
    double eps = fmax_f(ci[4] - ekin, seps);
    if (s->P.h2stat != -1) {
      /* state.f90:60-79 */
      double tk, m, gg;
      if (s->P.nz == 1) {
        const double x = s->P.dx * ((double)s->ix[i] - ((double)s->P.nx + ONE) / TWO);
        const double y = s->P.dy * ((double)s->iy[i] - ((double)s->P.ny + ONE) / TWO);
        const double hscale = sqrt((s->adindx[i] - ONE) * eps / (TWO * ekin) * (x * x + y * y));
        eps = eps / (TWO * hscale);
        const double rho = ci[0] / (TWO * hscale);
        get_gamma2(s, &eps, rho, &tk, &m, &gg);
      } else {
        get_gamma2(s, &eps, ci[0], &tk, &m, &gg);
      }
      s->muc_array[i] = m;
      s->adindx[i] = gg;
      p[i] = (ci[0] * tk * rgas / s->muc_array[i]);
      if (ci[0] < 1e-4) {
        p[i] = rgas * s->tk_bgrnd / muc * ci[0];
        eps = p[i] / (gam - ONE);
        ci[4] = eps + ekin;
      }
      continue;
    }
    s->adindx[i] = gam;
    s->muc_array[i] = muc;
    if (ci[0] < 1e-4) {
      double tk = fmin_f(5e3, p[i] / (ci[0] * rgas) * muc);
      p[i] = (ci[0] * tk * rgas / s->muc_array[i]);
      eps = p[i] / (gam - ONE);
      ci[4] = eps + ekin;
    } else {
      p[i] = eps * (gam - ONE);
    }
  }
}

/* ---------------------------------------------------------------- velocity.f90:18-53 */
void ox_velocity(ox_sim *s) {
  double *c = s->cons, *u = s->u;
  const double vlimit = s->P.vlimit, seps = s->P.small_eps;
  double maxv = ZERO;
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < s->ng; ++i)
    for (int d = 0; d < 3; ++d) u[3 * i + d] = c[5 * i + d + 1] / c[5 * i];
#pragma omp parallel for schedule(static) reduction(max : maxv)
  for (int64_t i = 0; i < s->ng; ++i) {
    double *ci = c + 5 * i, *ui = u + 3 * i;
    int flag = 0;
    for (int d = 0; d < 3; ++d) {
      maxv = fmax_f(maxv, fabs(ui[d]));
      if (fabs(ui[d]) > vlimit) flag = 1;
    }
    if (flag == 1) {
      double ekin = HALF * (ci[1] * ci[1] + ci[2] * ci[2] + ci[3] * ci[3]) / ci[0];
      double speed = ZERO;
      for (int d = 0; d < 3; ++d) speed = speed + ui[d] * ui[d];
      speed = sqrt(speed);
      for (int d = 0; d < 3; ++d) {
        ui[d] = ui[d] * vlimit / speed;
        ci[d + 1] = ui[d] * ci[0];
      }
      ci[4] = ci[4] - ekin;
      ekin = HALF * (ci[1] * ci[1] + ci[2] * ci[2] + ci[3] * ci[3]) / ci[0];
      ci[4] = fmax_f(ci[4], seps) + ekin;
    }
  }
  s->maxv = maxv;
}

/* ---------------------------------------------------------------- courant.f90:17-29 */
void ox_courant(ox_sim *s) {
  const double dx = s->P.dx, dy = s->P.dy, dz = s->P.dz;
  double dtrate = ZERO;
#pragma omp parallel for schedule(static) reduction(max : dtrate)
  for (int64_t i = 0; i < s->ng; ++i) {
    const double *ui = s->u + 3 * i;
    double sound = sqrt(s->adindx[i] * s->p[i] / s->cons[5 * i]);
    double r0 = (sound + fabs(ui[0])) / dx + (sound + fabs(ui[1])) / dy +
                (sound + fabs(ui[2])) / dz;
    dtrate = fmax_f(dtrate, r0);
  }
  s->dtrate = dtrate;
  s->dt = s->P.cfl / dtrate;
}

/* ---------------------------------------------------------------- utils.f90:200-281 */
static inline int64_t get_id(const ox_sim *s, int ix, int iy, int iz) {
  return (int64_t)(ix - 1) + (int64_t)(iy - 1) * s->P.nx +
         (int64_t)(iz - 1) * s->P.nx * s->P.ny;
}

static int64_t check_corner(const ox_sim *s, int ix, int iy, int iz, int64_t ineigh) {
  const int nx = s->P.nx, ny = s->P.ny, nz = s->P.nz;
  if (ix < 3) {
    if (iy < 3) {
      if (nz >= 6) {
        if (iz < 3) ineigh = get_id(s, 3, 3, 3);
        else if (iz > nz - 2) ineigh = get_id(s, 3, 3, nz - 2);
        else ineigh = get_id(s, 3, 3, iz);
      } else ineigh = get_id(s, 3, 3, iz);
    } else if (iy > ny - 2) {
      if (iz >= 6) { /* utils.f90:215 tests iz, not nz */
        if (iz < 3) ineigh = get_id(s, 3, ny - 2, 3);
        else if (iz > nz - 2) ineigh = get_id(s, 3, ny - 2, nz - 2);
        else ineigh = get_id(s, 3, ny - 2, iz);
      } else ineigh = get_id(s, 3, ny - 2, iz);
    } else {
      if (nz >= 6) {
        if (iz < 3) ineigh = get_id(s, 3, iy, 3);
        else if (iz > nz - 2) ineigh = get_id(s, 3, iy, nz - 2);
      } else ineigh = get_id(s, 3, iy, iz);
    }
  } else if (ix > nx - 2) {
    if (iy < 3) {
      if (nz >= 6) {
        if (iz < 3) ineigh = get_id(s, nx - 2, 3, 3);
        else if (iz > nz - 2) ineigh = get_id(s, nx - 2, 3, nz - 2);
        else ineigh = get_id(s, nx - 2, 3, iz);
      } else ineigh = get_id(s, nx - 2, 3, iz);
    } else if (iy > ny - 2) {
      if (nz >= 6) {
        if (iz < 3) ineigh = get_id(s, nx - 2, ny - 2, 3);
        else if (iz > nz - 2) ineigh = get_id(s, nx - 2, ny - 2, nz - 2);
        else ineigh = get_id(s, nx - 2, ny - 2, iz);
      } else ineigh = get_id(s, nx - 2, ny - 2, iz);
    } else {
      if (nz >= 6) {
        if (iz < 3) ineigh = get_id(s, nx - 2, iy, 3);
        else if (iz > nz - 2) ineigh = get_id(s, nx - 2, iy, nz - 2);
      } else ineigh = get_id(s, nx - 2, iy, iz);
    }
  } else {
    if (iy < 3) {
      if (nz >= 6) {
        if (iz < 3) ineigh = get_id(s, ix, 3, 3);
        else if (iz > nz - 2) ineigh = get_id(s, ix, 3, nz - 2);
      } else ineigh = get_id(s, ix, 3, iz);
    } else if (iy > ny - 2) {
      if (nz >= 6) {
        if (iz < 3) ineigh = get_id(s, ix, ny - 2, 3);
        else if (iz > nz - 2) ineigh = get_id(s, ix, ny - 2, nz - 2);
      } else ineigh = get_id(s, ix, ny - 2, iz);
    }
  }
  return ineigh;
}

/* utils.f90:287-296 */
static inline void set_ghost_helper(double *c, int64_t idx, int64_t ip, const double fac[3]) {
  c[5 * idx + 0] = c[5 * ip + 0];
  c[5 * idx + 1] = c[5 * ip + 1] * fac[0];
  c[5 * idx + 2] = c[5 * ip + 2] * fac[1];
  c[5 * idx + 3] = c[5 * ip + 3] * fac[2];
  c[5 * idx + 4] = c[5 * ip + 4];
}

static void ghost_one(ox_sim *s, int64_t idx) {
  const int nx = s->P.nx, ny = s->P.ny, nz = s->P.nz;
  const int32_t *w = s->P.no_outflow;
  double *c = s->cons;
  int ix = s->ix[idx], iy = s->iy[idx], iz = s->iz[idx];
  int64_t ineigh = -1;
  const int64_t *nb = s->ineigh + 6 * idx;
  if (s->bnd[idx] == 1) {
    ineigh = nb[0];
  } else { /* utils.f90:320-330 */
    if (ix == 2) ineigh = nb[2];
    else if (ix == nx - 1) ineigh = nb[3];
    else if (iy == 2) ineigh = nb[0];
    else if (iy == ny - 1) ineigh = nb[1];
    else if (iz == 2) ineigh = nb[4];
    else if (iz == nz - 1) ineigh = nb[5];
  }
  ineigh = check_corner(s, ix, iy, iz, ineigh);
  for (int d = 0; d < 5; ++d) c[5 * idx + d] = c[5 * ineigh + d];
  double fac[3];
  int64_t ip;
  /* utils.f90:338-403: reflective walls */
  if (w[0]) {
    fac[0] = -ONE; fac[1] = ONE; fac[2] = ONE;
    if (ix == 1) { ip = get_id(s, ix + 3, iy, iz); set_ghost_helper(c, idx, ip, fac); }
    else if (ix == 2) { ip = get_id(s, ix + 1, iy, iz); set_ghost_helper(c, idx, ip, fac); }
  }
  if (w[1]) {
    fac[0] = -ONE; fac[1] = ONE; fac[2] = ONE;
    if (ix == nx) { ip = get_id(s, ix - 3, iy, iz); set_ghost_helper(c, idx, ip, fac); }
    else if (ix == nx - 1) { ip = get_id(s, ix - 1, iy, iz); set_ghost_helper(c, idx, ip, fac); }
  }
  if (w[2]) {
    fac[0] = ONE; fac[1] = -ONE; fac[2] = ONE;
    if (iy == 1) { ip = get_id(s, ix, iy + 3, iz); set_ghost_helper(c, idx, ip, fac); }
    else if (iy == 2) { ip = get_id(s, ix, iy + 1, iz); set_ghost_helper(c, idx, ip, fac); }
  }
  if (w[3]) {
    fac[0] = ONE; fac[1] = -ONE; fac[2] = ONE;
    if (iy == ny) { ip = get_id(s, ix, iy - 3, iz); set_ghost_helper(c, idx, ip, fac); }
    else if (iy == ny - 1) { ip = get_id(s, ix, iy - 1, iz); set_ghost_helper(c, idx, ip, fac); }
  }
  if (w[4]) {
    fac[0] = ONE; fac[1] = ONE; fac[2] = -ONE;
    if (iz == 1) { ip = get_id(s, ix, iy, iz + 3); set_ghost_helper(c, idx, ip, fac); }
    else if (iz == 2) { ip = get_id(s, ix, iy, iz + 1); set_ghost_helper(c, idx, ip, fac); }
  }
  if (w[5]) {
    fac[0] = ONE; fac[1] = ONE; fac[2] = -ONE;
    if (iz == nz) { ip = get_id(s, ix, iy, iz - 3); set_ghost_helper(c, idx, ip, fac); }
    else if (iz == nz - 1) { ip = get_id(s, ix, iy, iz - 1); set_ghost_helper(c, idx, ip, fac); }
  }
}

/* utils.f90:305-480 (set_ghost_cells), single-threaded order unless racy_ghosts */
void ox_set_ghost_cells(ox_sim *s) {
  if (s->P.racy_ghosts) {
#pragma omp parallel for schedule(static)
    for (int64_t g = 0; g < s->nghost; ++g) ghost_one(s, s->indx_ghost[g]);
  } else {
    for (int64_t g = 0; g < s->nghost; ++g) ghost_one(s, s->indx_ghost[g]);
  }
}

/* ---------------------------------------------------------------- source.f90:58-199 */
void ox_source(ox_sim *s, int siter) {
  (void)siter;
  const double dt = s->dt, seps = s->P.small_eps;
  double *c = s->cons;
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < s->ng; ++i) {
    if (s->bnd[i] > 0) continue;
    double *ci = c + 5 * i;
    const double *g = s->gforce + 3 * i;
    double ux = s->u[3 * i], uy = s->u[3 * i + 1], uz = s->u[3 * i + 2];
    ci[2] = ci[2] + (ci[0] * (g[1])) * dt;
    ci[1] = ci[1] + (ci[0] * (g[0])) * dt;
    ci[3] = ci[3] + ((g[2]) * ci[0]) * dt;
    double ekin = HALF * (ci[1] * ci[1] + ci[2] * ci[2] + ci[3] * ci[3]) / ci[0];
    ci[4] = fmax_f(ci[4] - ekin + dt * ci[0] * (((ux) * (g[0]) + (uy) * (g[1]) + (uz) * (g[2]))),
                   seps) + ekin;
  }
  ox_set_ghost_cells(s);
}

/* ---------------------------------------------------------------- flux.f90 */
/* utils.f90:696-707 */
static inline double genminmod(double x1, double x2, double x3) {
  double tmp;
  if ((x1 > ZERO) && ((x2 > ZERO) && (x3 > ZERO))) {
    tmp = fmin_f(x2, x3);
    return fmin_f(x1, tmp);
  } else if ((x1 < ZERO) && ((x2 < ZERO) && (x3 < ZERO))) {
    tmp = fmax_f(x2, x3);
    return fmax_f(x1, tmp);
  }
  return ZERO;
}
/* utils.f90:738-741 */
static inline double slope(double c0, double c1, double c2) {
  return genminmod(THETA * (c1 - c0), HALF * (c2 - c0), THETA * (c2 - c1));
}

/* flux.f90:253-295; idx = (minus, centre, plus), idir 0..2 */
static void calculate_slopes(ox_sim *s, const int64_t idx[3], int idir) {
  const double *c = s->cons, *u = s->u;
  const int64_t i2 = idx[1];
  for (int idim = 0; idim < 3; ++idim)
    s->slope_u[9 * i2 + 3 * idir + idim] =
        slope(u[3 * idx[0] + idim], u[3 * idx[1] + idim], u[3 * idx[2] + idim]);
  double eps[3];
  for (int k = 0; k < 3; ++k) {
    const int64_t j = idx[k];
    eps[k] = fmax_f(c[5 * j + 4] - HALF * c[5 * j] *
                                       (u[3 * j] * u[3 * j] + u[3 * j + 1] * u[3 * j + 1] +
                                        u[3 * j + 2] * u[3 * j + 2]),
                    s->P.small_eps);
  }
  s->slope_p[3 * i2 + idir] = slope(s->p[idx[0]], s->p[idx[1]], s->p[idx[2]]);
  s->slope_d[3 * i2 + idir] = slope(c[5 * idx[0]], c[5 * idx[1]], c[5 * idx[2]]);
  s->slope_e[3 * i2 + idir] = slope(eps[0], eps[1], eps[2]);
  s->slope_g[3 * i2 + idir] = slope(s->adindx[idx[0]], s->adindx[idx[1]], s->adindx[idx[2]]);
}

/* flux.f90:299-308 */
static inline void interface_muscl(double q, double lm, double lp, double sl, double *minus,
                                   double *plus) {
  *minus = q + HALF * (-ONE - lm) * sl;
  *plus = q + HALF * (ONE - lp) * sl;
}

/* flux.f90:312-482 */
static void calculate_states(ox_sim *s, int64_t idx) {
  const double *c = s->cons, *u = s->u + 3 * idx;
  const double dt = s->dt;
  const double ds[3] = {s->P.dx, s->P.dy, s->P.dz};
  double sound = sqrt(s->p[idx] * s->adindx[idx] / c[5 * idx]);
  for (int idim = 0; idim < 3; ++idim) {
    double lambda_p = fmax_f(u[idim] + sound, ZERO) * dt / ds[idim];
    double lambda_m = fmin_f(u[idim] - sound, ZERO) * dt / ds[idim];
    for (int jdim = 0; jdim < 3; ++jdim)
      interface_muscl(u[jdim], lambda_m, lambda_p, s->slope_u[9 * idx + 3 * idim + jdim],
                      &s->st_u_m[9 * idx + 3 * idim + jdim], &s->st_u_p[9 * idx + 3 * idim + jdim]);
    double eps = fmax_f(c[5 * idx + 4] - HALF * c[5 * idx] *
                                             (u[0] * u[0] + u[1] * u[1] + u[2] * u[2]),
                        s->P.small_eps);
    interface_muscl(s->p[idx], lambda_m, lambda_p, s->slope_p[3 * idx + idim],
                    &s->st_p_m[3 * idx + idim], &s->st_p_p[3 * idx + idim]);
    interface_muscl(c[5 * idx], lambda_m, lambda_p, s->slope_d[3 * idx + idim],
                    &s->st_d_m[3 * idx + idim], &s->st_d_p[3 * idx + idim]);
    interface_muscl(eps, lambda_m, lambda_p, s->slope_e[3 * idx + idim],
                    &s->st_e_m[3 * idx + idim], &s->st_e_p[3 * idx + idim]);
    interface_muscl(s->adindx[idx], lambda_m, lambda_p, s->slope_g[3 * idx + idim],
                    &s->st_g_m[3 * idx + idim], &s->st_g_p[3 * idx + idim]);
  }
  /* flux.f90:391-479: transverse corrections, all source terms are zero */
  const double sr0 = ZERO, su0 = ZERO, sv0 = ZERO, sw0 = ZERO, sp0 = ZERO, se0 = ZERO,
               sg0 = ZERO;
  for (int d = 0; d < 3; ++d) {
    double cc = dt * HALF / ds[d];
    double *sup = s->st_u_p + 9 * idx + 3 * d, *sum = s->st_u_m + 9 * idx + 3 * d;
    s->st_d_p[3 * idx + d] = s->st_d_p[3 * idx + d] + sr0 * cc;
    sup[0] = sup[0] + su0 * cc;
    sup[1] = sup[1] + sv0 * cc;
    sup[2] = sup[2] + sw0 * cc;
    s->st_p_p[3 * idx + d] = s->st_p_p[3 * idx + d] + sp0 * cc;
    s->st_g_p[3 * idx + d] = s->st_g_p[3 * idx + d] + sg0 * cc;
    s->st_e_p[3 * idx + d] = s->st_e_p[3 * idx + d] + se0 * cc;
    s->st_d_m[3 * idx + d] = s->st_d_m[3 * idx + d] + sr0 * cc;
    sum[0] = sum[0] + su0 * cc;
    sum[1] = sum[1] + sv0 * cc;
    sum[2] = sum[2] + sw0 * cc;
    s->st_p_m[3 * idx + d] = s->st_p_m[3 * idx + d] + sp0 * cc;
    s->st_g_m[3 * idx + d] = s->st_g_m[3 * idx + d] + sg0 * cc;
    s->st_e_m[3 * idx + d] = s->st_e_m[3 * idx + d] + se0 * cc;
  }
}

/* flux.f90:575-590 */
static void flux_hll(const double fl[5], const double fr[5], const double ul[5],
                     const double ur[5], double gl, double gr, double dl, double dr, double pl,
                     double pr, double vl, double vr, double fhll[5]) {
  double cr = sqrt(gr * pr / dr);
  double cl = sqrt(gl * pl / dl);
  double ap = fmax_f(fmax_f(ZERO, vr + cr), vl + cl);
  double am = fmax_f(fmax_f(ZERO, -(vr - cr)), -(vl - cl));
  for (int i = 0; i < 5; ++i) fhll[i] = (ap * fl[i] + am * fr[i] - ap * am * (ur[i] - ul[i])) / (ap + am);
}

/* flux.f90:513-573: the HLL flux of one face from its left and right
 * reconstructed states, each (rho, u1, u2, u3, p, eps, gamma); idir 0..2 */
static void face_flux(const double L[7], const double R[7], int idir, double fhll[5]) {
  double dl = L[0], pl = L[4], el = L[5], gl = L[6];
  double vxl = L[1], vyl = L[2], vzl = L[3];
  double sl[5], sr[5], fl[5], fr[5];
  sl[0] = dl;
  sl[1] = dl * vxl;
  sl[2] = dl * vyl;
  sl[3] = dl * vzl;
  sl[4] = el + HALF * dl * (vxl * vxl + vyl * vyl + vzl * vzl);
  double dr = R[0], pr = R[4], er = R[5], gr = R[6];
  double vxr = R[1], vyr = R[2], vzr = R[3];
  sr[0] = dr;
  sr[1] = dr * vxr;
  sr[2] = dr * vyr;
  sr[3] = dr * vzr;
  sr[4] = er + HALF * dr * (vxr * vxr + vyr * vyr + vzr * vzr);
  for (int k = 0; k < 5; ++k) { fl[k] = ZERO; fr[k] = ZERO; }
  double vr, vl;
  if (idir == 0) { vr = vxr; vl = vxl; fl[1] = pl; fr[1] = pr; }
  else if (idir == 1) { vr = vyr; vl = vyl; fl[2] = pl; fr[2] = pr; }
  else { vr = vzr; vl = vzl; fl[3] = pl; fr[3] = pr; }
  fl[0] = sl[0] * vl;
  fl[1] = fl[1] + sl[1] * vl;
  fl[2] = fl[2] + sl[2] * vl;
  fl[3] = fl[3] + sl[3] * vl;
  fl[4] = (sl[4] + pl) * vl;
  fr[0] = sr[0] * vr;
  fr[1] = fr[1] + sr[1] * vr;
  fr[2] = fr[2] + sr[2] * vr;
  fr[3] = fr[3] + sr[3] * vr;
  fr[4] = (sr[4] + pr) * vr;
  flux_hll(fl, fr, sl, sr, gl, gr, dl, dr, pl, pr, vl, vr, fhll);
}

/* flux.f90:487-573; isten = (minus, centre, plus), idir 0..2; fhll[2][5] */
static void get_fluxes(const ox_sim *s, const int64_t isten[3], int idir, double fhll[2][5]) {
  for (int m_or_p = 0; m_or_p <= 1; ++m_or_p) {
    const int64_t a = isten[m_or_p], b = isten[1 + m_or_p];
    /* left: the plus state of cell a, right: the minus state of cell b */
    const double L[7] = {s->st_d_p[3 * a + idir], s->st_u_p[9 * a + 3 * idir + 0],
                         s->st_u_p[9 * a + 3 * idir + 1], s->st_u_p[9 * a + 3 * idir + 2],
                         s->st_p_p[3 * a + idir], s->st_e_p[3 * a + idir],
                         s->st_g_p[3 * a + idir]};
    const double R[7] = {s->st_d_m[3 * b + idir], s->st_u_m[9 * b + 3 * idir + 0],
                         s->st_u_m[9 * b + 3 * idir + 1], s->st_u_m[9 * b + 3 * idir + 2],
                         s->st_p_m[3 * b + idir], s->st_e_m[3 * b + idir],
                         s->st_g_m[3 * b + idir]};
    face_flux(L, R, idir, fhll[m_or_p]);
  }
}

/* Known-answer probes of the building blocks above, for the oracle's own tests. */
double ox_kat_genminmod(double x1, double x2, double x3) { return genminmod(x1, x2, x3); }
double ox_kat_slope(double c0, double c1, double c2) { return slope(c0, c1, c2); }
void ox_kat_muscl(double q, double lm, double lp, double sl, double *minus, double *plus) {
  interface_muscl(q, lm, lp, sl, minus, plus);
}
void ox_kat_face_flux(const double *left7, const double *right7, int idir, double *f5) {
  face_flux(left7, right7, idir, f5);
}

/* flux.f90:6-235 (anchors, flux.f90:134-184 and 592-601, need boundary>2 cells,
 * which exist only under EXTRAANCHORS; none are built here) */
void ox_flux(ox_sim *s, int avg) {
  const int64_t ng = s->ng;
  const double dx = s->P.dx, dy = s->P.dy, dz = s->P.dz, dt = s->dt;
  const double areaxy = dy * dx, areayz = dy * dz, areaxz = dx * dz, vol = dx * dy * dz;
#pragma omp parallel for schedule(static)
  for (int64_t ig = 0; ig < ng; ++ig) {
    for (int k = 0; k < 9; ++k) s->slope_u[9 * ig + k] = ZERO;
    for (int k = 0; k < 3; ++k) {
      s->slope_p[3 * ig + k] = ZERO; s->slope_d[3 * ig + k] = ZERO;
      s->slope_e[3 * ig + k] = ZERO; s->slope_g[3 * ig + k] = ZERO;
    }
    for (int k = 0; k < 5; ++k) s->fluxtmp[5 * ig + k] = ZERO;
    int64_t b[6];
    for (int k = 0; k < 6; ++k) b[k] = (s->bnd[ig] > 0) ? ig : s->ineigh[6 * ig + k];
    int64_t isten[3];
    isten[0] = b[3]; isten[1] = ig; isten[2] = b[2]; calculate_slopes(s, isten, 0);
    isten[0] = b[1]; isten[1] = ig; isten[2] = b[0]; calculate_slopes(s, isten, 1);
    isten[0] = b[5]; isten[1] = ig; isten[2] = b[4]; calculate_slopes(s, isten, 2);
  }
#pragma omp parallel for schedule(static)
  for (int64_t ig = 0; ig < ng; ++ig) calculate_states(s, ig);
#pragma omp parallel for schedule(static)
  for (int64_t ig = 0; ig < ng; ++ig) {
    if (s->bnd[ig] > 0) continue;
    const int64_t *b = s->ineigh + 6 * ig;
    double fx[2][5], fy[2][5], fz[2][5];
    int64_t isten[3];
    isten[0] = b[3]; isten[1] = ig; isten[2] = b[2]; get_fluxes(s, isten, 0, fx);
    isten[0] = b[1]; isten[1] = ig; isten[2] = b[0]; get_fluxes(s, isten, 1, fy);
    isten[0] = b[5]; isten[1] = ig; isten[2] = b[4]; get_fluxes(s, isten, 2, fz);
    for (int d = 0; d < 5; ++d)
      s->fluxtmp[5 * ig + d] = -(areayz * (fx[1][d] - fx[0][d]) + areaxz * (fy[1][d] - fy[0][d]) +
                                 areaxy * (fz[1][d] - fz[0][d])) * dt / vol;
  }
  if (avg == 0) {
#pragma omp parallel for schedule(static)
    for (int64_t ig = 0; ig < ng; ++ig)
      for (int d = 0; d < 5; ++d) s->cons[5 * ig + d] = s->cons[5 * ig + d] + s->fluxtmp[5 * ig + d];
  } else {
#pragma omp parallel for schedule(static)
    for (int64_t ig = 0; ig < ng; ++ig)
      for (int d = 0; d < 5; ++d)
        s->cons[5 * ig + d] =
            HALF * (s->cons_old[5 * ig + d] + s->cons[5 * ig + d] + s->fluxtmp[5 * ig + d]);
  }
#pragma omp parallel for schedule(static)
  for (int64_t ig = 0; ig < ng; ++ig) {
    double *c = s->cons + 5 * ig;
    c[0] = fmax_f(c[0], s->P.small_rho);
    if (c[4] < ZERO) c[4] = HALF * (c[1] * c[1] + c[2] * c[2] + c[3] * c[3]) / c[0] + s->P.small_eps;
  }
  ox_set_ghost_cells(s);
}

/* ---------------------------------------------------------------- flux_ang.f90 */
/* grid(igrid)%x, %y (init_grid.f90:88,92) */
static inline double cell_x(const ox_sim *s, int64_t i) {
  return s->P.dx * ((double)s->ix[i] - ((double)s->P.nx + ONE) / TWO);
}
static inline double cell_y(const ox_sim *s, int64_t i) {
  return s->P.dy * ((double)s->iy[i] - ((double)s->P.ny + ONE) / TWO);
}

/* flux_ang.f90:301-345: calculate_slopes plus the slopes of the transformed momenta */
static void calculate_slopes_ang(ox_sim *s, const int64_t idx[3], int idir) {
  calculate_slopes(s, idx, idir);
  const double *c = s->cons;
  const int64_t i2 = idx[1];
  s->slope_rmom[3 * i2 + idir] = slope(c[5 * idx[0] + 1], c[5 * idx[1] + 1], c[5 * idx[2] + 1]);
  s->slope_amom[3 * i2 + idir] = slope(c[5 * idx[0] + 2], c[5 * idx[1] + 2], c[5 * idx[2] + 2]);
}

/* flux_ang.f90:349-518: calculate_states plus the states of the transformed
 * momenta (which take no transverse term) */
static void calculate_states_ang(ox_sim *s, int64_t idx) {
  calculate_states(s, idx);
  const double *c = s->cons, *u = s->u + 3 * idx;
  const double dt = s->dt;
  const double ds[3] = {s->P.dx, s->P.dy, s->P.dz};
  const double sound = sqrt(s->p[idx] * s->adindx[idx] / c[5 * idx]);
  for (int idim = 0; idim < 3; ++idim) {
    const double lambda_p = fmax_f(u[idim] + sound, ZERO) * dt / ds[idim];
    const double lambda_m = fmin_f(u[idim] - sound, ZERO) * dt / ds[idim];
    interface_muscl(c[5 * idx + 1], lambda_m, lambda_p, s->slope_rmom[3 * idx + idim],
                    &s->st_rmom_m[3 * idx + idim], &s->st_rmom_p[3 * idx + idim]);
    interface_muscl(c[5 * idx + 2], lambda_m, lambda_p, s->slope_amom[3 * idx + idim],
                    &s->st_amom_m[3 * idx + idim], &s->st_amom_p[3 * idx + idim]);
  }
}

/* flux_ang.f90:523-618; x, y, r of the updated cell isten[1] (no yoffset) */
static void get_fluxes_ang(const ox_sim *s, const int64_t isten[3], int idir, double fhll[2][5]) {
  const int64_t idx = isten[1];
  const double x = cell_x(s, idx), y = cell_y(s, idx);
  const double r = sqrt(x * x + y * y);
  for (int m_or_p = 0; m_or_p <= 1; ++m_or_p) {
    const int64_t a = isten[m_or_p], b = isten[1 + m_or_p];
    double dl = s->st_d_p[3 * a + idir], pl = s->st_p_p[3 * a + idir];
    double el = s->st_e_p[3 * a + idir], gl = s->st_g_p[3 * a + idir];
    double vxl = s->st_u_p[9 * a + 3 * idir + 0], vyl = s->st_u_p[9 * a + 3 * idir + 1],
           vzl = s->st_u_p[9 * a + 3 * idir + 2];
    double sl[5], sr[5], fl[5], fr[5];
    sl[0] = dl;
    sl[1] = s->st_rmom_p[3 * a + idir];
    sl[2] = s->st_amom_p[3 * a + idir];
    sl[3] = dl * vzl;
    sl[4] = el + HALF * dl * (vxl * vxl + vyl * vyl + vzl * vzl);
    double dr = s->st_d_m[3 * b + idir], pr = s->st_p_m[3 * b + idir];
    double er = s->st_e_m[3 * b + idir], gr = s->st_g_m[3 * b + idir];
    double vxr = s->st_u_m[9 * b + 3 * idir + 0], vyr = s->st_u_m[9 * b + 3 * idir + 1],
           vzr = s->st_u_m[9 * b + 3 * idir + 2];
    sr[0] = dr;
    sr[1] = s->st_rmom_m[3 * b + idir];
    sr[2] = s->st_amom_m[3 * b + idir];
    sr[3] = dr * vzr;
    sr[4] = er + HALF * dr * (vxr * vxr + vyr * vyr + vzr * vzr);
    for (int k = 0; k < 5; ++k) { fl[k] = ZERO; fr[k] = ZERO; }
    double vr, vl;
    if (idir == 0) {
      vr = vxr; vl = vxl;
      fl[1] = pl * x / r; fr[1] = pr * x / r;
      fl[2] = -(pl * y); fr[2] = -(pr * y);
    } else if (idir == 1) {
      vr = vyr; vl = vyl;
      fl[1] = pl * y / r; fr[1] = pr * y / r;
      fl[2] = pl * x; fr[2] = pr * x;
    } else {
      vr = vzr; vl = vzl; fl[3] = pl; fr[3] = pr;
    }
    fl[0] = sl[0] * vl;
    fl[1] = fl[1] + sl[1] * vl;
    fl[2] = fl[2] + sl[2] * vl;
    fl[3] = fl[3] + sl[3] * vl;
    fl[4] = (sl[4] + pl) * vl;
    fr[0] = sr[0] * vr;
    fr[1] = fr[1] + sr[1] * vr;
    fr[2] = fr[2] + sr[2] * vr;
    fr[3] = fr[3] + sr[3] * vr;
    fr[4] = (sr[4] + pr) * vr;
    flux_hll(fl, fr, sl, sr, gl, gr, dl, dr, pl, pr, vl, vr, fhll[m_or_p]);
  }
}

/* flux_ang.f90:6-281 */
void ox_flux_ang(ox_sim *s, int avg) {
  const int64_t ng = s->ng;
  const double dx = s->P.dx, dy = s->P.dy, dz = s->P.dz, dt = s->dt;
  const double areaxy = dy * dx, areayz = dy * dz, areaxz = dx * dz, vol = dx * dy * dz;
  /* flux_ang.f90:44-62: (m1, m2) -> (rmom, angmom) */
#pragma omp parallel for schedule(static)
  for (int64_t ig = 0; ig < ng; ++ig) {
    const double x = cell_x(s, ig), y = cell_y(s, ig) + s->P.yoffset;
    const double r = sqrt(x * x + y * y);
    double *c = s->cons + 5 * ig;
    double angmom = x * c[2] - y * c[1];
    double rmom = (c[1] * x + c[2] * y) / r;
    c[1] = rmom;
    c[2] = angmom;
    if (avg > 0) {
      double *o = s->cons_old + 5 * ig;
      angmom = x * o[2] - y * o[1];
      rmom = (o[1] * x + o[2] * y) / r;
      o[1] = rmom;
      o[2] = angmom;
    }
  }
  /* flux_ang.f90:69-106 slopes */
#pragma omp parallel for schedule(static)
  for (int64_t ig = 0; ig < ng; ++ig) {
    for (int k = 0; k < 9; ++k) s->slope_u[9 * ig + k] = ZERO;
    for (int k = 0; k < 3; ++k) {
      s->slope_p[3 * ig + k] = ZERO; s->slope_d[3 * ig + k] = ZERO;
      s->slope_e[3 * ig + k] = ZERO; s->slope_g[3 * ig + k] = ZERO;
      s->slope_rmom[3 * ig + k] = ZERO; s->slope_amom[3 * ig + k] = ZERO;
    }
    for (int k = 0; k < 5; ++k) s->fluxtmp[5 * ig + k] = ZERO;
    int64_t b[6];
    for (int k = 0; k < 6; ++k) b[k] = (s->bnd[ig] > 0) ? ig : s->ineigh[6 * ig + k];
    int64_t isten[3];
    isten[0] = b[3]; isten[1] = ig; isten[2] = b[2]; calculate_slopes_ang(s, isten, 0);
    isten[0] = b[1]; isten[1] = ig; isten[2] = b[0]; calculate_slopes_ang(s, isten, 1);
    isten[0] = b[5]; isten[1] = ig; isten[2] = b[4]; calculate_slopes_ang(s, isten, 2);
  }
  /* flux_ang.f90:112-141 states */
#pragma omp parallel for schedule(static)
  for (int64_t ig = 0; ig < ng; ++ig) calculate_states_ang(s, ig);
  /* flux_ang.f90:146-223 fluxes (anchors inactive, as in flux.f90) */
#pragma omp parallel for schedule(static)
  for (int64_t ig = 0; ig < ng; ++ig) {
    if (s->bnd[ig] > 0) continue;
    const int64_t *b = s->ineigh + 6 * ig;
    double fx[2][5], fy[2][5], fz[2][5];
    int64_t isten[3];
    isten[0] = b[3]; isten[1] = ig; isten[2] = b[2]; get_fluxes_ang(s, isten, 0, fx);
    isten[0] = b[1]; isten[1] = ig; isten[2] = b[0]; get_fluxes_ang(s, isten, 1, fy);
    isten[0] = b[5]; isten[1] = ig; isten[2] = b[4]; get_fluxes_ang(s, isten, 2, fz);
    for (int d = 0; d < 5; ++d)
      s->fluxtmp[5 * ig + d] = -(areayz * (fx[1][d] - fx[0][d]) + areaxz * (fy[1][d] - fy[0][d]) +
                                 areaxy * (fz[1][d] - fz[0][d])) * dt / vol;
  }
  /* flux_ang.f90:230-245 update */
  if (avg == 0) {
#pragma omp parallel for schedule(static)
    for (int64_t ig = 0; ig < ng; ++ig)
      for (int d = 0; d < 5; ++d) s->cons[5 * ig + d] = s->cons[5 * ig + d] + s->fluxtmp[5 * ig + d];
  } else {
#pragma omp parallel for schedule(static)
    for (int64_t ig = 0; ig < ng; ++ig)
      for (int d = 0; d < 5; ++d)
        s->cons[5 * ig + d] =
            HALF * (s->cons_old[5 * ig + d] + s->cons[5 * ig + d] + s->fluxtmp[5 * ig + d]);
  }
  /* flux_ang.f90:255-270: back to (m1, m2) */
#pragma omp parallel for schedule(static)
  for (int64_t ig = 0; ig < ng; ++ig) {
    const double x = cell_x(s, ig), y = cell_y(s, ig) + s->P.yoffset;
    const double r = sqrt(x * x + y * y);
    double *c = s->cons + 5 * ig;
    double angmom = c[2], rmom = c[1];
    c[1] = (rmom * x - angmom * y / r) / r;
    c[2] = (rmom * y + angmom * x / r) / r;
    if (avg > 0) {
      double *o = s->cons_old + 5 * ig;
      angmom = o[2];
      rmom = o[1];
      o[1] = (rmom * x - angmom * y / r) / r;
      o[2] = (rmom * y + angmom * x / r) / r;
    }
  }
  /* flux_ang.f90:272-278 floors */
#pragma omp parallel for schedule(static)
  for (int64_t ig = 0; ig < ng; ++ig) {
    double *c = s->cons + 5 * ig;
    c[0] = fmax_f(c[0], s->P.small_rho);
    if (c[4] < ZERO) c[4] = HALF * (c[1] * c[1] + c[2] * c[2] + c[3] * c[3]) / c[0] + s->P.small_eps;
  }
  ox_set_ghost_cells(s);
}

/* main.f90:343-346,365-368: flux or flux_ang */
static void flux_step(ox_sim *s, int avg) {
  if (s->P.fluxangmom) ox_flux_ang(s, avg);
  else ox_flux(s, avg);
}

/* main.f90:327-333 */
void ox_save_cons_old(ox_sim *s) {
  memcpy(s->cons_old, s->cons, s->ng * 5 * sizeof(double));
}

/* get_boundary (utils.f90:62-73): neighbour idx of igrid, or igrid itself when
 * the neighbour lies in a ghost layer.  An unset slot (init_grid.f90:178 leaves
 * five of them at 0 for the outer ghost layer, an index outside grid(1:ngrid)
 * that the reference reads anyway) resolves to igrid as well. */
static int64_t get_boundary_1(const ox_sim *s, int64_t igrid, int idx) {
  const int64_t b = s->ineigh[igrid * 6 + idx];
  if (b < 0 || s->bnd[b] > 0) return igrid;
  return b;
}

/* avisc.f90:4-26, the condition as written (boundary > 0) */
void ox_avisc(const ox_sim *s, double avmagx, double avmagy, double avmagz, double *qq) {
  const int64_t ng = s->ng;
#pragma omp parallel for schedule(static)
  for (int64_t igrid = 0; igrid < ng; ++igrid) {
    double *q = qq + igrid * 3;
    if (s->bnd[igrid] > 0) {
      int64_t b[6];
      for (int k = 0; k < 6; ++k) b[k] = get_boundary_1(s, igrid, k);
      const double m1 = fmin_f(ZERO, s->u[b[2] * 3 + 0] - s->u[b[3] * 3 + 0]);
      const double m2 = fmin_f(ZERO, s->u[b[0] * 3 + 1] - s->u[b[1] * 3 + 1]);
      const double m3 = fmin_f(ZERO, s->u[b[4] * 3 + 2] - s->u[b[5] * 3 + 2]);
      q[0] = avmagx * (m1 * m1);
      q[1] = avmagy * (m2 * m2);
      q[2] = avmagz * (m3 * m3);
    } else {
      q[0] = ZERO;
      q[1] = ZERO;
      q[2] = ZERO;
    }
  }
}

/* main.f90:212-545, default flags (no gravity solver, radiation or particles) */
int ox_step(ox_sim *s, double endtime) {
  if (s->time >= endtime || s->step >= 1000000) return 1;
  s->step = s->step + 1;
  ox_state(s);
  ox_courant(s);
  const double f1 = ONE;
  s->dt = s->dt * f1;
  if (s->step > 1 && s->dtold > ZERO) s->dt = fmin_f(s->dt, s->dtold * 1.1);
  s->dtold = s->dt;
  if (s->dt + s->time > endtime) s->dt = endtime - s->time;
  s->dt = s->dt * HALF;
  ox_source(s, 0);
  ox_set_ghost_cells(s);
  ox_state(s);
  ox_velocity(s);
  ox_save_cons_old(s);
  s->dt = s->dt * TWO;
  flux_step(s, 0);
  ox_set_ghost_cells(s);
  ox_state(s);
  ox_velocity(s);
  flux_step(s, 1);
  ox_set_ghost_cells(s);
  ox_state(s);
  ox_velocity(s);
  s->dt = HALF * s->dt;
  ox_source(s, 1);
  ox_set_ghost_cells(s);
  ox_state(s);
  ox_velocity(s);
  s->dt = s->dt * TWO;
  s->time = s->time + s->dt;
  return 0;
}

/* main.f90:212-545 with the full step dt given instead of the CFL rule
 * (finite differences of a run with its dt sequence held fixed) */
void ox_step_dt(ox_sim *s, double dt_full) {
  s->step = s->step + 1;
  ox_state(s);
  ox_courant(s);
  s->dt = dt_full;
  s->dtold = s->dt;
  s->dt = s->dt * HALF;
  ox_source(s, 0);
  ox_set_ghost_cells(s);
  ox_state(s);
  ox_velocity(s);
  ox_save_cons_old(s);
  s->dt = s->dt * TWO;
  flux_step(s, 0);
  ox_set_ghost_cells(s);
  ox_state(s);
  ox_velocity(s);
  flux_step(s, 1);
  ox_set_ghost_cells(s);
  ox_state(s);
  ox_velocity(s);
  s->dt = HALF * s->dt;
  ox_source(s, 1);
  ox_set_ghost_cells(s);
  ox_state(s);
  ox_velocity(s);
  s->dt = s->dt * TWO;
  s->time = s->time + s->dt;
}

int64_t ox_run(ox_sim *s, double endtime, int64_t nsteps) {
  int64_t n = 0;
  while (n < nsteps) {
    if (ox_step(s, endtime)) break;
    ++n;
  }
  return n;
}

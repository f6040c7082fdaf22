// bx_kernels.cu -- sm_100a FP64 kernels of the hydro step.
//
// Two kernel families compute the same reference step:
//
//  * Fused stage kernels (k_stage<0|1>): one launch per SSP-RK2 stage.  A block
//    owns a TX x TY column tile of interior cells and marches through a z range.
//    For each z plane it stages primitives of the tile plus a two-cell x/y halo
//    in shared memory, builds the limited MUSCL face states once per cell and
//    direction, computes every x/y face flux once, carries the z-direction
//    states, face fluxes and primitives of its own column in registers, and
//    updates the conserved variables in the epilogue.  Sources, the EOS, the
//    velocity update and the CFL max-reduction of the following step are fused
//    into the stage kernels; ghost cells are not stored but read through a
//    fixed donor rule (validated per grid on the host), so each conserved plane
//    crosses HBM about once per stage.
//
//  * Phase kernels: one kernel per reference subroutine (state, velocity,
//    courant, source, set_ghost_cells, flux) on full arrays, exactly the
//    reference's data flow including its stored velocity and pressure arrays.
//    They serve the bisection entry points, the first step after an upload, and
//    steps where the velocity limiter or the low-density EOS branch fires.
#include <cuda_runtime.h>

#include <algorithm>
#include <map>
#include <mutex>
#include <utility>

#include "bx_internal.h"
#include "bx_math.cuh"

namespace bx {

cudaError_t ensure_dyn_smem(const void* fn, size_t bytes) {
  static std::mutex mu;
  static std::map<std::pair<const void*, int>, size_t> set;
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  std::lock_guard<std::mutex> lock(mu);
  size_t& have = set[{fn, dev}];
  if (have >= bytes) return cudaSuccess;
  e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
  if (e == cudaSuccess) have = bytes;
  return e;
}

namespace {

// get_gamma2 (eos.f90:653-699): gamma, mu and T from the tables by the specific
// internal energy eng = eps/rho, linear in eng within the density row irho, then
// linear in rho towards row irho+1.  eps is clamped like the reference's.
__device__ void get_gamma2(const EosDev& e, double& eps, double rho, double& tk, double& m,
                           double& gam) {
  int irho = min((int)((log10(rho * e.density_unit) - e.log_rho_low) / e.drho) + 1, e.neos_rho);
  if (irho < 1) irho = 1;
  int irhop = irho + 1;
  if (irhop > e.neos_rho) irhop = irho;
  const long long ne = e.neos;
  auto at = [&](const double* t, int ie, int ir) { return t[(ie - 1) + (ir - 1) * ne]; };
  double eng = eps / rho;
  // log10 of the row's first energy: precomputed with the same device log10
  int ientry = (int)((log10(eng) - e.log_eng1[irho - 1]) / e.deng[irho - 1]) + 1;
  if (ientry > e.neos - 1) {
    ientry = e.neos - 1;
    eng = at(e.eng2, e.neos, irho);
    eps = eng * rho;
  }
  if (ientry < 1 || eng < at(e.eng2, 1, irho)) {
    ientry = 1;
    eng = at(e.eng2, 1, irho);
    eps = eng * rho;
  }
  // t(ientry) + (t(ientry+1) - t(ientry)) / (eng(ientry+1) - eng(ientry)) *
  // (eng - eng(ientry)) for gamma, mu and T of density row ir: the three
  // quotients share the denominator, so one exact shared reciprocal
  auto lin3 = [&](int ir, double& g3, double& m3, double& t3) {
    const double e0 = at(e.eng2, ientry, ir);
    const SharedDiv q(at(e.eng2, ientry + 1, ir) - e0);
    const double de = eng - e0;
    g3 = at(e.gam2, ientry, ir) + q(at(e.gam2, ientry + 1, ir) - at(e.gam2, ientry, ir)) * de;
    m3 = at(e.muc2, ientry, ir) + q(at(e.muc2, ientry + 1, ir) - at(e.muc2, ientry, ir)) * de;
    t3 = at(e.tk2, ientry, ir) + q(at(e.tk2, ientry + 1, ir) - at(e.tk2, ientry, ir)) * de;
  };
  lin3(irho, gam, m, tk);
  if (!(e.rho[irho - 1] == e.rho[irhop - 1])) {
    double gamp, mp, tkp;
    lin3(irhop, gamp, mp, tkp);
    const double slope = 1.0 / (e.rho[irhop - 1] - e.rho[irho - 1]) * (rho - e.rho[irho - 1]);
    gam = gam + (gamp - gam) * slope;
    m = m + (mp - m) * slope;
    tk = tk + (tkp - tk) * slope;
  }
}


// Loads of the stage inputs: through the read-only path when the planes stay
// unchanged for the whole launch (one launch per stage), from L2 (cg) in the
// persistent batched kernel, whose other blocks write planes that this block
// reads later in the same launch.
template <bool CG = false>
__device__ __forceinline__ double ldg(const double* p) {
  return CG ? __ldcg(p) : __ldg(p);
}

// donor of a coordinate along one axis for a face ghost (fused path)
__device__ __forceinline__ int remap_axis(int c, int a0, int a1, int wl, int wr, bool& flip) {
  if (c < a0) {
    if (wl) { flip = true; return 2 * a0 - 1 - c; }
    return a0;
  }
  if (c >= a1) {
    if (wr) { flip = true; return 2 * a1 - 1 - c; }
    return a1 - 1;
  }
  return c;
}

struct Cons {
  double d, m1, m2, m3, E;
};

template <bool CG = false>
__device__ __forceinline__ Cons load_cons(const double* B, long long PS, const Geom& g, int x,
                                          int y, int z) {
  bool fx = false, fy = false, fz = false;
  const int xx = remap_axis(x, g.ax0, g.ax1, g.wall[0], g.wall[1], fx);
  const int yy = remap_axis(y, g.ay0, g.ay1, g.wall[2], g.wall[3], fy);
  const int zz = g.threed ? remap_axis(z, g.az0, g.az1, g.wall[4], g.wall[5], fz) : z;
  const long long c = g.base + xx + (long long)yy * g.sy + (long long)zz * g.sz;
  Cons r;
  r.d = ldg<CG>(B + c);
  r.m1 = ldg<CG>(B + PS + c);
  r.m2 = ldg<CG>(B + 2 * PS + c);
  r.m3 = ldg<CG>(B + 3 * PS + c);
  r.E = ldg<CG>(B + 4 * PS + c);
  if (fx) r.m1 = -r.m1;
  if (fy) r.m2 = -r.m2;
  if (fz) r.m3 = -r.m3;
  return r;
}

// the step input's velocity m/rho at a cell, as stage 0 stored it for the
// interior cells (ghost cells read their source cell, reflected components negated)
template <bool CG = false>
__device__ __forceinline__ void load_u(const double* U, long long PS, const Geom& g, int x, int y,
                                       int z, double& u1, double& u2, double& u3) {
  bool fx = false, fy = false, fz = false;
  const int xx = remap_axis(x, g.ax0, g.ax1, g.wall[0], g.wall[1], fx);
  const int yy = remap_axis(y, g.ay0, g.ay1, g.wall[2], g.wall[3], fy);
  const int zz = g.threed ? remap_axis(z, g.az0, g.az1, g.wall[4], g.wall[5], fz) : z;
  const long long c = g.base + xx + (long long)yy * g.sy + (long long)zz * g.sz;
  u1 = ldg<CG>(U + c);
  u2 = ldg<CG>(U + PS + c);
  u3 = ldg<CG>(U + 2 * PS + c);
  if (fx) u1 = -u1;
  if (fy) u2 = -u2;
  if (fz) u3 = -u3;
}

// the gravitational acceleration at a cell: the donor's for a ghost coordinate,
// reflected components negated like the momenta (the source update is exact
// under reflecting m and g together)
__device__ __forceinline__ void load_g(const double* G, long long PS, const Geom& g, int x, int y,
                                       int z, double& g1, double& g2, double& g3) {
  load_u(G, PS, g, x, y, z, g1, g2, g3);
}

// source(0) with gravity on conserved values c (source.f90:161-182 with dt/2):
// the velocity array it reads is m/rho before the kick (the last velocity() ran
// on these momenta); returns that velocity in (v1, v2, v3) for state()
__device__ __forceinline__ void gravity_source0(Cons& c, double g1, double g2, double g3,
                                                double dth, double small_eps, double& v1,
                                                double& v2, double& v3) {
  v1 = c.m1 / c.d;
  v2 = c.m2 / c.d;
  v3 = c.m3 / c.d;
  source_gravity(c.d, c.m1, c.m2, c.m3, c.E, g1, g2, g3, v1, v2, v3, dth, small_eps);
}

__device__ __forceinline__ void apply_sources(Cons& c, int nsrc, double small_eps) {
  for (int k = 0; k < nsrc; ++k) c.E = source_energy(c.d, c.m1, c.m2, c.m3, c.E, small_eps);
}

// Primitives seen by flux(avg) at a cell.
//  stage 0: cons = src^nsrc(X); u = m/rho (velocity at main.f90:318); p from
//           state() with the velocity array of the previous step, which equals
//           m/rho of the same momenta (source adds zero momentum).
//  stage 1: cons = Y; u = m/rho of Y (velocity at main.f90:355); p from state()
//           with the stage-0 velocity m0/rho0 (main.f90:353 uses the stale u),
//           which stage 0 stored in U (the same quotient, so the same bits).
//  GRAV (a gravitational force this step): stage 0 takes the nsrc-1 force-free
//           sources still pending, then source(0) with the force, which kicks
//           the momenta; state() then reads the velocity array of before the
//           kick (main.f90:318-319 call state() before velocity()).
// The values a cell's primitives are computed from: its conserved variables
// (X in stage 0, Y in stage 1) and, in stage 1, the stage-0 velocity U, or,
// in stage 0 with a force, the acceleration G.
struct Raw {
  Cons c;
  double v1, v2, v3;
};

// STAGE 0 or 1: the stage is known at compile time; STAGE 2: it is the runtime
// value rs (the persistent batched kernel runs both stages in one body)
template <int STAGE>
__device__ __forceinline__ bool stage_is0(int rs) {
  return STAGE == 2 ? rs == 0 : STAGE == 0;
}

template <int STAGE, bool GRAV = false, bool CG = false>
__device__ __forceinline__ Raw load_raw(const StageArgs& a, const Geom& g, int x, int y, int z,
                                        int rs = 0) {
  const long long PS = a.ncells_total;
  Raw r;
  if (stage_is0<STAGE>(rs)) {
    r.c = load_cons<CG>(a.X, PS, g, x, y, z);
    if (GRAV) load_g(a.G, PS, g, x, y, z, r.v1, r.v2, r.v3);
  } else {
    r.c = load_cons<CG>(a.Y, PS, g, x, y, z);
    load_u<CG>(a.U, PS, g, x, y, z, r.v1, r.v2, r.v3);
  }
  return r;
}

// Primitives of a cell without a force (stage 0 with the nsrc pending sources,
// or stage 1 with the stale velocity v), every division by the cell's density
// (the sources leave it alone) through one correctly rounded reciprocal and the
// residual correction (exact).  The corrections are valid while the numerators'
// exponents lie in their window; one check of all of them at the end, rather
// than a branch per division, and false sends the caller to prim_ieee.
template <int STAGE>
__device__ __forceinline__ bool prim_fast(const Geom& g, const Cons& c, double v1, double v2,
                                          double v3, int nsrc, bool need_c, Prim& q, int rs = 0) {
  const bool is0 = stage_is0<STAGE>(rs);
  const double d = c.d;
  bool ok = d >= 0x1p-450 && d <= 0x1p+450;
  const double r = ok ? __drcp_rn(d) : 1.0;
  double E = c.E;
  if (is0) {
    // source(): E = max(E - K, eps) + K with K = half*|m|^2/rho, the same K each time
    const double kn = kHalf * (c.m1 * c.m1 + c.m2 * c.m2 + c.m3 * c.m3);
    ok = ok && quot_fast_ok(kn);
    const double ek = quot_fast(kn, d, r);
    for (int k = 0; k < nsrc; ++k) E = fmax(E - ek, g.small_eps) + ek;
  }
  ok = ok && quot_fast_ok(c.m1) && quot_fast_ok(c.m2) && quot_fast_ok(c.m3);
  q.d = d;
  q.u1 = quot_fast(c.m1, d, r);
  q.u2 = quot_fast(c.m2, d, r);
  q.u3 = quot_fast(c.m3, d, r);
  q.e = recon_eps(d, E, q.u1, q.u2, q.u3, g.small_eps);
  q.p = is0 ? q.e * g.gm1 : eos_pressure(d, E, v1, v2, v3, g.gm1, g.small_eps);
  q.c = 0.0;
  if (need_c) {
    const double pn = q.p * g.gam;
    ok = ok && quot_fast_ok(pn);
    q.c = sqrt(quot_fast(pn, d, r));
  }
  return ok;
}

// the same with IEEE divisions (taken only outside the window)
template <int STAGE>
__device__ __forceinline__ Prim prim_ieee(double small_eps, double gm1, double gam, Cons c, double v1,
                                       double v2, double v3, int nsrc, bool need_c, int rs = 0) {
  Prim q;
  q.g = gam;
  const bool is0 = stage_is0<STAGE>(rs);
  if (is0) apply_sources(c, nsrc, small_eps);
  q.d = c.d;
  q.u1 = c.m1 / c.d;
  q.u2 = c.m2 / c.d;
  q.u3 = c.m3 / c.d;
  q.e = recon_eps(q.d, c.E, q.u1, q.u2, q.u3, small_eps);
  q.p = is0 ? q.e * gm1 : eos_pressure(q.d, c.E, v1, v2, v3, gm1, small_eps);
  q.c = need_c ? sqrt(q.p * gam / q.d) : 0.0;
  return q;
}

template <int STAGE, bool GRAV = false, bool TAB = false>
__device__ __forceinline__ Prim prim_of(const Geom& g, Raw r, unsigned& flags, int nsrc,
                                        double dth, bool need_c = true, int rs = 0,
                                        const EosDev* eos = nullptr) {
  Prim q;
  q.g = g.gam;
  if (STAGE == 0 && GRAV) {
    const SharedDiv qd(r.c.d);
    Cons c = r.c;
    double v1, v2, v3;
    apply_sources(c, nsrc - 1, g.small_eps);
    gravity_source0(c, r.v1, r.v2, r.v3, dth, g.small_eps, v1, v2, v3);
    q.d = c.d;
    q.u1 = qd(c.m1);
    q.u2 = qd(c.m2);
    q.u3 = qd(c.m3);
    q.e = recon_eps(q.d, c.E, q.u1, q.u2, q.u3, g.small_eps);
    q.p = eos_pressure(q.d, c.E, v1, v2, v3, g.gm1, g.small_eps);
    // the sound speed enters only the lambdas of cells whose face states are built
    q.c = need_c ? sqrt(qd(q.p * g.gam)) : 0.0;
  } else if (!prim_fast<STAGE>(g, r.c, r.v1, r.v2, r.v3, nsrc, need_c && !TAB, q, rs)) {
    q = prim_ieee<STAGE>(g.small_eps, g.gm1, g.gam, r.c, r.v1, r.v2, r.v3, nsrc,
                         need_c && !TAB, rs);
  }
  if (TAB) {
    // state() with the tables (state.f90:60-79): eps from the energy and the
    // velocity array state() reads (stage 0: m/rho, so the reconstruction's
    // eps; stage 1: the stage-0 velocity), then p and gamma by get_gamma2
    double eps = stage_is0<STAGE>(rs)
                     ? q.e
                     : fmax(r.c.E - kin_rho_u(q.d, r.v1, r.v2, r.v3), g.small_eps);
    double tk, m, gam;
    get_gamma2(*eos, eps, q.d, tk, m, gam);
    q.p = (q.d * tk * g.rgas / m);
    q.g = gam;
    q.c = need_c ? sqrt(q.p * gam / q.d) : 0.0;
  }
  if (q.d < kLowRho) flags |= kFlagLowRho;
  if (fabs(q.u1) > g.vlimit || fabs(q.u2) > g.vlimit || fabs(q.u3) > g.vlimit)
    flags |= kFlagVlimit;
  return q;
}

// Primitives seen by flux(avg) at a cell.
//  stage 0: cons = src^nsrc(X); u = m/rho (velocity at main.f90:318); p from
//           state() with the velocity array of the previous step, which equals
//           m/rho of the same momenta (source adds zero momentum).
//  stage 1: cons = Y; u = m/rho of Y (velocity at main.f90:355); p from state()
//           with the stage-0 velocity m0/rho0 (main.f90:353 uses the stale u),
//           which stage 0 stored in U (the same quotient, so the same bits).
//  GRAV (a gravitational force this step): stage 0 takes the nsrc-1 force-free
//           sources still pending, then source(0) with the force, which kicks
//           the momenta; state() then reads the velocity array of before the
//           kick (main.f90:318-319 call state() before velocity()).
// the centre of cell (ix, iy) in the x-y plane (flux_ang.f90:44-46 and
// :571-573, as cell_xy), and its distance from the z axis
__device__ __forceinline__ void cell_xyr(const Geom& g, int ix, int iy, double& x, double& y,
                                         double& r) {
  x = g.dx * ((double)(ix + 1) - ((double)g.nx + 1.0) / 2.0);
  y = g.dy * ((double)(iy + 1) - ((double)g.ny + 1.0) / 2.0);
  r = sqrt(x * x + y * y);
}

// (m1, m2) -> (radial momentum, angular momentum) about the z axis through
// (0, -yoffset) at cell (ix, iy) (flux_ang.f90:44-62)
__device__ __forceinline__ void ang_to(const Geom& g, int ix, int iy, double m1, double m2,
                                       double& rm, double& am) {
  double x, y, r;
  cell_xyr(g, ix, iy, x, y, r);
  y = y + g.yoff;
  r = sqrt(x * x + y * y);
  rm = (m1 * x + m2 * y) / r;
  am = x * m2 - y * m1;
}

template <int STAGE, bool GRAV = false, bool CG = false, bool TAB = false, bool ANG = false>
__device__ __forceinline__ Prim load_prim(const StageArgs& a, const Geom& g, int x, int y, int z,
                                          unsigned& flags, int nsrc, double dth,
                                          bool need_c = true, int rs = 0) {
  const Raw r = load_raw<STAGE, GRAV, CG>(a, g, x, y, z, rs);
  Prim q = prim_of<STAGE, GRAV, TAB>(g, r, flags, nsrc, dth, need_c, rs, &a.eos);
  // with flux_ang the momenta reconstructed are the transformed ones (the
  // sources leave the momenta alone)
  if (ANG) ang_to(g, x, y, r.c.m1, r.c.m2, q.rm, q.am);
  return q;
}

template <bool POW2, bool TAB = false, bool ANG = false>
__device__ __forceinline__ void dir_states(const Prim& m, const Prim& c, const Prim& p, double ud,
                                           double dt, double ds, double ids, FaceState& mi,
                                           FaceState& pl) {
  const double sd = slope3(m.d, c.d, p.d);
  const double s1 = slope3(m.u1, c.u1, p.u1);
  const double s2 = slope3(m.u2, c.u2, p.u2);
  const double s3 = slope3(m.u3, c.u3, p.u3);
  const double sp = slope3(m.p, c.p, p.p);
  const double se = slope3(m.e, c.e, p.e);
  // the tabulated EOS's gamma (adindx), reconstructed like the others (flux.f90:293,350)
  const double sg = TAB ? slope3(m.g, c.g, p.g) : 0.0;
  // flux_ang's transformed momenta (flux_ang.f90:301-345)
  const double srm = ANG ? slope3(m.rm, c.rm, p.rm) : 0.0;
  const double sam = ANG ? slope3(m.am, c.am, p.am) : 0.0;
  muscl_states<POW2, TAB, ANG>(c, ud, sd, s1, s2, s3, sp, se, dt, ds, ids, mi, pl, sg, srm, sam);
}

template <int NP, int NPF = 7>
__device__ __forceinline__ void put_prim(double* SP, int i, const Prim& q) {
  SP[0 * NP + i] = q.d;
  SP[1 * NP + i] = q.u1;
  SP[2 * NP + i] = q.u2;
  SP[3 * NP + i] = q.u3;
  SP[4 * NP + i] = q.p;
  SP[5 * NP + i] = q.e;
  SP[6 * NP + i] = q.c;
  if (NPF == 8) SP[7 * NP + i] = q.g;
  if (NPF == 9) {
    SP[7 * NP + i] = q.rm;
    SP[8 * NP + i] = q.am;
  }
}
template <int NP, int NPF = 7>
__device__ __forceinline__ Prim get_prim(const double* SP, int i) {
  Prim q;
  q.d = SP[0 * NP + i];
  q.u1 = SP[1 * NP + i];
  q.u2 = SP[2 * NP + i];
  q.u3 = SP[3 * NP + i];
  q.p = SP[4 * NP + i];
  q.e = SP[5 * NP + i];
  q.c = SP[6 * NP + i];
  if (NPF == 8) q.g = SP[7 * NP + i];
  if (NPF == 9) {
    q.rm = SP[7 * NP + i];
    q.am = SP[8 * NP + i];
  }
  return q;
}
template <int NSF = 6>
__device__ __forceinline__ void put_fs(double* S, int n, int i, const FaceState& f) {
  S[0 * n + i] = f.d;
  S[1 * n + i] = f.u1;
  S[2 * n + i] = f.u2;
  S[3 * n + i] = f.u3;
  S[4 * n + i] = f.p;
  S[5 * n + i] = f.e;
  if (NSF == 7) S[6 * n + i] = f.g;
  if (NSF == 8) {
    S[6 * n + i] = f.rm;
    S[7 * n + i] = f.am;
  }
}
template <int NSF = 6>
__device__ __forceinline__ FaceState get_fs(const double* S, int n, int i) {
  FaceState f;
  f.d = S[0 * n + i];
  f.u1 = S[1 * n + i];
  f.u2 = S[2 * n + i];
  f.u3 = S[3 * n + i];
  f.p = S[4 * n + i];
  f.e = S[5 * n + i];
  if (NSF == 7) f.g = S[6 * n + i];
  if (NSF == 8) {
    f.rm = S[6 * n + i];
    f.am = S[7 * n + i];
  }
  return f;
}

__device__ __forceinline__ double warp_max(double v) {
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}


}  // namespace

// The end of stage 1 without a force, from the updated cell n: the velocity
// after flux(1), then source(1)'s energy, state()'s pressure and the Courant
// rate of the next step (courant.f90:20-22).  Every division is by n's density:
// one correctly rounded reciprocal and the residual correction (exact) while
// all numerators lie in the window, checked once; false sends the caller to
// epi_ieee.
template <bool POW2>
__device__ __forceinline__ bool epi_fast(const Geom& g, const double n[5], double& u1, double& u2,
                                         double& u3, double& r0) {
  const double d = n[0];
  const double kn = kHalf * (n[1] * n[1] + n[2] * n[2] + n[3] * n[3]);
  bool ok = d >= 0x1p-450 && d <= 0x1p+450 && quot_fast_ok(n[1]) && quot_fast_ok(n[2]) &&
            quot_fast_ok(n[3]) && quot_fast_ok(kn);
  const double r = ok ? __drcp_rn(d) : 1.0;
  u1 = quot_fast(n[1], d, r);
  u2 = quot_fast(n[2], d, r);
  u3 = quot_fast(n[3], d, r);
  const double ek = quot_fast(kn, d, r);
  const double E3 = fmax(n[4] - ek, g.small_eps) + ek;
  const double pA = eos_pressure(d, E3, u1, u2, u3, g.gm1, g.small_eps);
  const double pn = g.gam * pA;
  ok = ok && quot_fast_ok(pn);
  const double sound = sqrt(quot_fast(pn, d, r));
  if (POW2)
    r0 = (sound + fabs(u1)) * g.idx + (sound + fabs(u2)) * g.idy + (sound + fabs(u3)) * g.idz;
  else
    r0 = cdiv(sound + fabs(u1), g.dx, g.idx) + cdiv(sound + fabs(u2), g.dy, g.idy) +
         cdiv(sound + fabs(u3), g.dz, g.idz);
  return ok;
}
template <bool POW2>
__device__ __forceinline__ void epi_ieee(const Geom& g, const double n[5], double& u1, double& u2,
                                         double& u3, double& r0) {
  u1 = n[1] / n[0];
  u2 = n[2] / n[0];
  u3 = n[3] / n[0];
  const double E3 = source_energy(n[0], n[1], n[2], n[3], n[4], g.small_eps);
  const double pA = eos_pressure(n[0], E3, u1, u2, u3, g.gm1, g.small_eps);
  r0 = courant_rate<POW2>(n[0], pA, g.gam, u1, u2, u3, g.dx, g.dy, g.dz, g.idx, g.idy, g.idz);
}

// The same end of stage 1 with the tabulated EOS: the next step's state()
// takes p and gamma from the tables (state.f90:60-79) with the velocity after
// source(1), m/rho of the new cell, and courant.f90:20-21 uses that gamma.
template <bool POW2>
__device__ __forceinline__ void epi_tab(const Geom& g, const EosDev& eos, const double n[5],
                                        double& u1, double& u2, double& u3, double& r0) {
  u1 = n[1] / n[0];
  u2 = n[2] / n[0];
  u3 = n[3] / n[0];
  const double E3 = source_energy(n[0], n[1], n[2], n[3], n[4], g.small_eps);
  double eps = fmax(E3 - kin_rho_u(n[0], u1, u2, u3), g.small_eps);
  double tk, m, gam;
  get_gamma2(eos, eps, n[0], tk, m, gam);
  const double p = (n[0] * tk * g.rgas / m);
  r0 = courant_rate<POW2>(n[0], p, gam, u1, u2, u3, g.dx, g.dy, g.dz, g.idx, g.idy, g.idz);
}

// ------------------------------------------------------------------ stage kernel
// One tile of one stage.  FULL: the tile is a whole TX x TY block of interior
// columns, so its extents are compile-time constants.
// dt: the step's full dt; nsrc: the sources the stage input is short of (both
// read from the box's control block by the caller).  CG: inputs through L2 (the
// persistent batched kernel).
template <class S, int STAGE, bool POW2, bool THREED, bool FULL, bool GRAV, bool CG = false>
__device__ __forceinline__ void stage_tile(const StageArgs& a, const Tile& t, const Geom& g,
                                           Ctrl* C, double dt, int nsrc, double* sm,
                                           double* red_rate, unsigned* red_flags, int rs = 0) {
  const bool is0 = stage_is0<STAGE>(rs);
  constexpr int TX = S::TX, TY = S::TY, NT = S::NT, PW = S::PW, NP = S::NP;
  constexpr bool TAB = S::TAB, ANG = S::ANG;
  constexpr int NPF = S::NPF, NSF = S::NSF, NFQ = S::NFQ, NOWN = S::NOWN;
  constexpr int NSX = S::NSX, NSY = S::NSY, NFX = S::NFX, NFY = S::NFY, NR0 = S::NR0;
  double* SP = sm;                    // [NPF][TY+4][TX+4] primitives of the plane
  double* SX = sm + NR0;              // [2 NSF][TY][TX+2] x states (minus, then plus)
  double* SY = SX + 2 * NSF * NSX;    // [2 NSF][TY+2][TX] y states
  double* FX = sm;                    // [NFQ][TY][TX+1] x face fluxes (aliases SP)
  double* FY = sm + NFQ * NFX;        // [NFQ][TY+1][TX] y face fluxes
  double* ZS = SY + 2 * NSF * NSY;    // [10 + NSF][NOWN]: Fzm 0-4, Fzp 5-9, plus state 10-
  const double dth = dt * kHalf;  // the sources' half step (main.f90:282,471)

  const int tid = threadIdx.x;
  const int tx = tid % TX, ty = tid / TX;
  const int NAx = g.ax1 - g.ax0, NAy = g.ay1 - g.ay0;
  const int w = FULL ? TX : min(TX, NAx - t.x0), h = FULL ? TY : min(TY, NAy - t.y0);
  const bool own = (tx < w) && (ty < h);
  const int bx0 = g.ax0 + t.x0, by0 = g.ay0 + t.y0;  // full-grid tile origin
  const int gx = bx0 + tx, gy = by0 + ty;
  const int nhalo = 4 * h + 4 * w;
  const int nxs = (w + 2) * h, nys = w * (h + 2);
  const int nxf = (w + 1) * h, nyf = w * (h + 1);
  const long long PS = a.ncells_total;
  const double idz = g.idz;

  unsigned flags = 0;
  double rate = 0.0;

  // z pipeline of the own column (3-D grids)
  Prim Pk, Pk1;
  // (columns only: the threads with a column are 0 .. NOWN-1)
  auto zs = [&](int k) -> double& { return ZS[k * NOWN + threadIdx.x]; };

  const int z0 = g.az0 + t.z0, z1 = g.az0 + t.z1;
  if (THREED && own) {
    const Prim Pm2 = load_prim<STAGE, GRAV, CG, TAB, ANG>(a, g, gx, gy, z0 - 2, flags, nsrc, dth, true, rs);
    const Prim Pm1 = load_prim<STAGE, GRAV, CG, TAB, ANG>(a, g, gx, gy, z0 - 1, flags, nsrc, dth, true, rs);
    Pk = load_prim<STAGE, GRAV, CG, TAB, ANG>(a, g, gx, gy, z0, flags, nsrc, dth, true, rs);
    Pk1 = load_prim<STAGE, GRAV, CG, TAB, ANG>(a, g, gx, gy, z0 + 1, flags, nsrc, dth, true, rs);
    FaceState mm, pm, m0;
    if (z0 - 1 < g.az0) {
      ghost_states(Pm1, mm, pm);
    } else {
      dir_states<POW2, TAB, ANG>(Pm2, Pm1, Pk, Pm1.u3, dt, g.dz, idz, mm, pm);
    }
    FaceState plusk;
    double Fzm[5];
    dir_states<POW2, TAB, ANG>(Pm1, Pk, Pk1, Pk.u3, dt, g.dz, idz, m0, plusk);
    if (ANG) {
      double F7[7];
      hll_flux_ang<2>(pm, m0, g.gam, 0.0, 0.0, 1.0, 0.0, 0.0, 1.0, F7);
      for (int q = 0; q < 5; ++q) Fzm[q] = F7[q];
    } else {
      hll_flux<2, TAB>(pm, m0, g.gam, Fzm);
    }
    for (int q = 0; q < 5; ++q) zs(q) = Fzm[q];
    zs(10) = plusk.d; zs(11) = plusk.u1; zs(12) = plusk.u2; zs(13) = plusk.u3;
    zs(14) = plusk.p; zs(15) = plusk.e;
    if (TAB) zs(16) = plusk.g;
    if (ANG) { zs(16) = plusk.rm; zs(17) = plusk.am; }
  }

  for (int z = (THREED ? z0 : g.az0 + t.z0); z < (THREED ? z1 : g.az0 + t.z1); ++z) {
    // ---- A: primitives of plane z (own from the pipeline, halo computed here)
    if (!is0 && own) {
      // the update at the end of this plane reads the step input of the own
      // cell, which nothing in this stage loaded before: start it towards L2
      const double* c = a.X + g.base + gx + (long long)gy * g.sy + (long long)z * g.sz;
#pragma unroll
      for (int q = 0; q < 5; ++q) asm volatile("prefetch.global.L2 [%0];" ::"l"(c + q * PS));
      if (THREED && z + 3 < g.az1) {
        // the own column's loads of the next plane iteration
        const long long o3 = g.base + gx + (long long)gy * g.sy + (long long)(z + 3) * g.sz;
#pragma unroll
        for (int q = 0; q < 5; ++q) asm volatile("prefetch.global.L2 [%0];" ::"l"(a.Y + o3 + q * PS));
#pragma unroll
        for (int q = 0; q < 3; ++q) asm volatile("prefetch.global.L2 [%0];" ::"l"(a.U + o3 + q * PS));
      }
    }
    if (is0 && own && THREED && z + 3 < g.az1) {
      // stage 0: the own column's step input of the next plane iteration
      const long long o3 = g.base + gx + (long long)gy * g.sy + (long long)(z + 3) * g.sz;
#pragma unroll
      for (int q = 0; q < 5; ++q) asm volatile("prefetch.global.L2 [%0];" ::"l"(a.X + o3 + q * PS));
    }
    Prim P2;
    FaceState mz1, pz1;
    if (own) {
      if (THREED) {
        P2 = load_prim<STAGE, GRAV, CG, TAB, ANG>(a, g, gx, gy, z + 2, flags, nsrc, dth, true, rs);
      } else {
        Pk = load_prim<STAGE, GRAV, CG, TAB, ANG>(a, g, gx, gy, z, flags, nsrc, dth, true, rs);
      }
      put_prim<NP, NPF>(SP, (ty + 2) * PW + (tx + 2), Pk);
      if (is0) {
        // sources change only E, so this is m/rho of the step input
        const long long o = g.base + gx + (long long)gy * g.sy + (long long)z * g.sz;
        a.U[o] = Pk.u1;
        a.U[PS + o] = Pk.u2;
        a.U[2 * PS + o] = Pk.u3;
      }
    }
    // halo cells go first to the threads without a column of their own (at most
    // one per thread: 4*(TX+TY) <= NT).  Their loads are not issued before the
    // own column's arithmetic: holding both cells' values at once spills
    // registers and measured 14 % slower.
    for (int i = (tid + NT - TX * TY) % NT; i < nhalo; i += NT) {
      int cx, cy;
      if (i < 4 * h) {
        cy = i >> 2;
        const int j = i & 3;
        cx = j < 2 ? j - 2 : w + (j - 2);
      } else {
        const int k = i - 4 * h;
        cx = k % w;
        const int j = k / w;
        cy = j < 2 ? j - 2 : h + (j - 2);
      }
      // cells two away from the tile only feed slopes; ghost cells need no lambda
      const int fx = bx0 + cx, fy = by0 + cy;
      const bool near = cx >= -1 && cx <= w && cy >= -1 && cy <= h;
      const bool inner = fx >= g.ax0 && fx < g.ax1 && fy >= g.ay0 && fy < g.ay1;
      const Prim q = load_prim<STAGE, GRAV, CG, TAB, ANG>(a, g, fx, fy, z, flags, nsrc, dth, near && inner, rs);
      put_prim<NP, NPF>(SP, (cy + 2) * PW + (cx + 2), q);
    }
    if (THREED && own) {
      if (z + 1 >= g.az1) {
        ghost_states(Pk1, mz1, pz1);
      } else {
        dir_states<POW2, TAB, ANG>(Pk, Pk1, P2, Pk1.u3, dt, g.dz, idz, mz1, pz1);
      }
      const FaceState plusk{zs(10), zs(11), zs(12), zs(13), zs(14), zs(15),
                            TAB ? zs(16) : 0.0,
                            ANG ? zs(16) : 0.0, ANG ? zs(17) : 0.0};
      double Fzp[5];
      if (ANG) {
        double F7[7];
        hll_flux_ang<2>(plusk, mz1, g.gam, 0.0, 0.0, 1.0, 0.0, 0.0, 1.0, F7);
        for (int q = 0; q < 5; ++q) Fzp[q] = F7[q];
      } else {
        hll_flux<2, TAB>(plusk, mz1, g.gam, Fzp);
      }
      for (int q = 0; q < 5; ++q) zs(5 + q) = Fzp[q];
      zs(10) = pz1.d; zs(11) = pz1.u1; zs(12) = pz1.u2; zs(13) = pz1.u3;
      zs(14) = pz1.p; zs(15) = pz1.e;
      if (TAB) zs(16) = pz1.g;
      if (ANG) { zs(16) = pz1.rm; zs(17) = pz1.am; }
    }
    __syncthreads();

    // ---- B: x and y face states of the plane.  The y items start at a warp
    // boundary, so no warp runs both the x and the y code (the x items end in
    // idle lanes instead)
    const int nxs_w = (nxs + 31) & ~31;
    for (int i = tid; i < nxs_w + nys; i += NT) {
      FaceState mi, pl;
      if (i < nxs_w) {
        if (i >= nxs) continue;
        const int cy = i / (w + 2), cx = i % (w + 2) - 1;
        const int c = (cy + 2) * PW + (cx + 2);
        const Prim q = get_prim<NP, NPF>(SP, c);
        const int fx = bx0 + cx;
        if (fx < g.ax0 || fx >= g.ax1) {
          ghost_states(q, mi, pl);
        } else {
          dir_states<POW2, TAB, ANG>(get_prim<NP, NPF>(SP, c - 1), q, get_prim<NP, NPF>(SP, c + 1), q.u1, dt, g.dx, g.idx, mi,
                           pl);
        }
        const int o = cy * (TX + 2) + (cx + 1);
        put_fs<NSF>(SX, NSX, o, mi);
        put_fs<NSF>(SX + NSF * NSX, NSX, o, pl);
      } else {
        const int k = i - nxs_w;
        const int cy = k / w - 1, cx = k % w;
        const int c = (cy + 2) * PW + (cx + 2);
        const Prim q = get_prim<NP, NPF>(SP, c);
        const int fy = by0 + cy;
        if (fy < g.ay0 || fy >= g.ay1) {
          ghost_states(q, mi, pl);
        } else {
          dir_states<POW2, TAB, ANG>(get_prim<NP, NPF>(SP, c - PW), q, get_prim<NP, NPF>(SP, c + PW), q.u2, dt, g.dy, g.idy,
                           mi, pl);
        }
        const int o = (cy + 1) * TX + cx;
        put_fs<NSF>(SY, NSY, o, mi);
        put_fs<NSF>(SY + NSF * NSY, NSY, o, pl);
      }
    }
    __syncthreads();

    // ---- C: x and y face fluxes (face f lies between cells f-1 and f); the y
    // faces start at a warp boundary as in B
    const int nxf_w = (nxf + 31) & ~31;
    for (int i = tid; i < nxf_w + nyf; i += NT) {
      double F[NFQ];
      if (i < nxf_w) {
        if (i >= nxf) continue;
        const int cy = i / (w + 1), f = i % (w + 1);
        const int base = cy * (TX + 2);
        const FaceState L = get_fs<NSF>(SX + NSF * NSX, NSX, base + f);  // plus state of cell f-1
        const FaceState R = get_fs<NSF>(SX, NSX, base + f + 1);        // minus state of cell f
        if constexpr (ANG) {
          // the momentum fluxes for both cells of the face (their own centres)
          double xl, yl, rl, xh, yh, rh;
          cell_xyr(g, bx0 + f - 1, by0 + cy, xl, yl, rl);
          cell_xyr(g, bx0 + f, by0 + cy, xh, yh, rh);
          hll_flux_ang<0>(L, R, g.gam, xl, yl, rl, xh, yh, rh, F);
        } else {
          hll_flux<0, TAB>(L, R, g.gam, F);
        }
        const int o = cy * (TX + 1) + f;
#pragma unroll
        for (int q = 0; q < NFQ; ++q) FX[q * NFX + o] = F[q];
      } else {
        const int k = i - nxf_w;
        const int f = k / w, cx = k % w;
        const FaceState L = get_fs<NSF>(SY + NSF * NSY, NSY, f * TX + cx);
        const FaceState R = get_fs<NSF>(SY, NSY, (f + 1) * TX + cx);
        if constexpr (ANG) {
          double xl, yl, rl, xh, yh, rh;
          cell_xyr(g, bx0 + cx, by0 + f - 1, xl, yl, rl);
          cell_xyr(g, bx0 + cx, by0 + f, xh, yh, rh);
          hll_flux_ang<1>(L, R, g.gam, xl, yl, rl, xh, yh, rh, F);
        } else {
          hll_flux<1, TAB>(L, R, g.gam, F);
        }
        const int o = f * TX + cx;
#pragma unroll
        for (int q = 0; q < NFQ; ++q) FY[q * NFY + o] = F[q];
      }
    }
    __syncthreads();

    // ---- D: conservative update of the own cell (flux.f90:186-230)
    if (own) {
      double ft[5];
#pragma unroll
      for (int q = 0; q < 5; ++q) {
        // with flux_ang the momentum fluxes of this cell's plus faces are the
        // versions for their low cell (planes 5, 6)
        const int qp = (ANG && (q == 1 || q == 2)) ? q + 4 : q;
        const double dfx = FX[qp * NFX + ty * (TX + 1) + tx + 1] - FX[q * NFX + ty * (TX + 1) + tx];
        const double dfy = FY[qp * NFY + (ty + 1) * TX + tx] - FY[q * NFY + ty * TX + tx];
        double sum = g.ayz * dfx + g.axz * dfy;
        if (THREED) sum = sum + g.axy * (zs(5 + q) - zs(q));
        ft[q] = POW2 ? -sum * dt * g.ivol : cdiv(-sum * dt, g.vol, g.ivol);
      }
      Cons c0 = load_cons<CG>(a.X, PS, g, gx, gy, z);
      double go1 = 0.0, go2 = 0.0, go3 = 0.0;  // the own cell's acceleration
      if (GRAV) {
        load_g(a.G, PS, g, gx, gy, z, go1, go2, go3);
        double v1, v2, v3;
        apply_sources(c0, nsrc - 1, g.small_eps);
        gravity_source0(c0, go1, go2, go3, dth, g.small_eps, v1, v2, v3);
      } else {
        const SharedDiv q0(c0.d);
        for (int k = 0; k < nsrc; ++k)
          c0.E = source_energy_q(q0, c0.m1, c0.m2, c0.m3, c0.E, g.small_eps);
      }
      double n[5];
      // flux_ang updates the transformed momenta (flux_ang.f90:44-62, 149-246)
      if (ANG) ang_to(g, gx, gy, c0.m1, c0.m2, c0.m1, c0.m2);
      if (is0) {
        n[0] = c0.d + ft[0];
        n[1] = c0.m1 + ft[1];
        n[2] = c0.m2 + ft[2];
        n[3] = c0.m3 + ft[3];
        n[4] = c0.E + ft[4];
      } else {
        Cons c1 = load_cons<CG>(a.Y, PS, g, gx, gy, z);
        if (ANG) ang_to(g, gx, gy, c1.m1, c1.m2, c1.m1, c1.m2);
        n[0] = kHalf * (c0.d + c1.d + ft[0]);
        n[1] = kHalf * (c0.m1 + c1.m1 + ft[1]);
        n[2] = kHalf * (c0.m2 + c1.m2 + ft[2]);
        n[3] = kHalf * (c0.m3 + c1.m3 + ft[3]);
        n[4] = kHalf * (c0.E + c1.E + ft[4]);
      }
      if (ANG) {
        // back to (m1, m2) (flux_ang.f90:247-270)
        double cxp, cyp, crp;
        cell_xyr(g, gx, gy, cxp, cyp, crp);
        const double tyy = cyp + g.yoff, trr = sqrt(cxp * cxp + tyy * tyy);
        const double rmom = n[1], angmom = n[2];
        n[1] = (rmom * cxp - angmom * tyy / trr) / trr;
        n[2] = (rmom * tyy + angmom * cxp / trr) / trr;
      }
      floors(n[0], n[1], n[2], n[3], n[4], g.small_rho, g.small_eps);
      if (!(isfinite(n[0]) && isfinite(n[1]) && isfinite(n[2]) && isfinite(n[3]) &&
            isfinite(n[4])))
        flags |= kFlagNonFinite;
      if (!is0) {
        // state/velocity after flux(1) and after source(1) (main.f90:372-380,490-515);
        // without a force every division here is by the new density: one
        // reciprocal and one window check for all of them (epi_fast)
        double u1, u2, u3, r0 = 0.0;
        if (GRAV) {
          const SharedDiv qn(n[0]);
          u1 = qn(n[1]);
          u2 = qn(n[2]);
          u3 = qn(n[3]);
        } else if (TAB) {
          epi_tab<POW2>(g, a.eos, n, u1, u2, u3, r0);
        } else if (!epi_fast<POW2>(g, n, u1, u2, u3, r0)) {
          epi_ieee<POW2>(g, n, u1, u2, u3, r0);
        }
        if (n[0] < kLowRho) flags |= kFlagLowRho;
        if (fabs(u1) > g.vlimit || fabs(u2) > g.vlimit || fabs(u3) > g.vlimit)
          flags |= kFlagVlimit;
        if (GRAV) {
          // source(1) with the force (main.f90:471): the planes take its result,
          // the velocity it read goes to UC for state() at the step's end
          // (main.f90:513-514), and the Courant rate of the next step is taken
          // with the velocity after it (main.f90:515)
          const long long o = g.base + gx + (long long)gy * g.sy + (long long)z * g.sz;
          a.UC[o] = u1;
          a.UC[PS + o] = u2;
          a.UC[2 * PS + o] = u3;
          source_gravity(n[0], n[1], n[2], n[3], n[4], go1, go2, go3, u1, u2, u3, dth,
                         g.small_eps);
          const double w1 = n[1] / n[0], w2 = n[2] / n[0], w3 = n[3] / n[0];
          if (fabs(w1) > g.vlimit || fabs(w2) > g.vlimit || fabs(w3) > g.vlimit)
            flags |= kFlagVlimit;
          if (!(isfinite(n[1]) && isfinite(n[2]) && isfinite(n[3]) && isfinite(n[4])))
            flags |= kFlagNonFinite;
          const double pA = eos_pressure(n[0], n[4], w1, w2, w3, g.gm1, g.small_eps);
          const double r0 = courant_rate<POW2>(n[0], pA, g.gam, w1, w2, w3, g.dx, g.dy, g.dz,
                                               g.idx, g.idy, g.idz);
          rate = fmax(rate, r0);
          if (!(r0 >= 0.0)) flags |= kFlagNonFinite;
        } else {
          rate = fmax(rate, r0);
          if (!(r0 >= 0.0)) flags |= kFlagNonFinite;
        }
      }
      const long long o = g.base + gx + (long long)gy * g.sy + (long long)z * g.sz;
#pragma unroll
      for (int q = 0; q < 5; ++q) a.out[q * PS + o] = n[q];
      if (THREED) {
#pragma unroll
        for (int q = 0; q < 5; ++q) zs(q) = zs(5 + q);
        Pk = Pk1;
        Pk1 = P2;
      }
    }
    __syncthreads();
  }

  // block reductions of the Courant rate and the status bits
  const unsigned wf = __reduce_or_sync(0xffffffffu, flags);
  const double wr = warp_max(rate);
  if ((tid & 31) == 0) {
    red_flags[tid >> 5] = wf;
    red_rate[tid >> 5] = wr;
  }
  __syncthreads();
  if (tid == 0) {
    unsigned f = 0;
    double r = 0.0;
    for (int k = 0; k < NT / 32; ++k) {
      f |= red_flags[k];
      r = fmax(r, red_rate[k]);
    }
    if (f) atomicOr(&C->flags, f);
    if (!is0) atomicMax(&C->rate_bits, (unsigned long long)__double_as_longlong(r));
  }
}

template <int SH>
struct ShapeSel {
  using type = Shape0;
};
template <>
struct ShapeSel<1> {
  using type = Shape1;
};
template <>
struct ShapeSel<2> {
  using type = Shape2;
};
template <>
struct ShapeSel<3> {
  using type = Shape3;
};

// PM: 1 = every box of the launch has power-of-two spacings (divisions by the
// cell sizes are multiplications by exact reciprocals), 0 = otherwise (cdiv,
// exact for any spacing).  SH: the tile shape (Shape0 or Shape1; Shape2 with the
// tabulated EOS, Shape3 with angular-momentum fluxing).
template <int STAGE, int PM, bool THREED, bool GRAV = false, int SH = 0>
__global__ void __launch_bounds__(NT, 65536 / (NT * 128)) k_stage(StageArgs a) {
  using S = typename ShapeSel<SH>::type;
  extern __shared__ double sm[];
  __shared__ Geom sg;
  __shared__ double red_rate[NT / 32];
  __shared__ unsigned red_flags[NT / 32];
  const Tile t = a.tiles[blockIdx.x];
  if (threadIdx.x == 0) sg = a.geom[t.box];
  __syncthreads();
  Ctrl* C = a.ctrl + t.box;
  if (!C->active) return;
  const double dt = C->dt;
  const int nsrc = a.nsrc > 0 ? a.nsrc : C->nsrc;
  const bool full = (t.x0 + S::TX <= sg.ax1 - sg.ax0) && (t.y0 + S::TY <= sg.ay1 - sg.ay0);
  constexpr bool P2 = PM == 1;
  if (full)
    stage_tile<S, STAGE, P2, THREED, true, GRAV>(a, t, sg, C, dt, nsrc, sm, red_rate, red_flags);
  else
    stage_tile<S, STAGE, P2, THREED, false, GRAV>(a, t, sg, C, dt, nsrc, sm, red_rate, red_flags);
}

// A batched box's clock at the start of a step (dt control of main.f90:266-281
// and 342, with the clock saved for a trip) and at its end (main.f90:471,544-545,
// or the trip of a box whose step raised a guard: its planes then keep the
// step's input and its clock is put back)
__device__ __forceinline__ void box_begin_step(Ctrl& c) {
  c.run_step += 1;
  if (c.tripped || !(c.time < c.endtime) || c.step >= 1000000 || c.step >= c.max_step) {
    c.active = 0;
    return;
  }
  c.time0 = c.time;
  c.dtold0 = c.dtold;
  c.step0 = c.step;
  c.rate_bits0 = c.rate_bits;
  c.step = c.step + 1;
  const double rate = __longlong_as_double((long long)c.rate_bits);
  c.rate = rate;
  c.rate_bits = 0ull;
  double dt = c.cfl / rate;
  dt = dt * 1.0;
  if (c.step > 1 && c.dtold > 0.0) dt = fmin(dt, c.dtold * 1.1);
  c.dtold = dt;
  if (dt + c.time > c.endtime) dt = c.endtime - c.time;
  dt = dt * kHalf;
  dt = dt * 2.0;
  c.dt = dt;
  c.active = 1;
}
__device__ __forceinline__ void box_end_step(Ctrl& c) {
  if (!c.active) return;
  if (c.flags & (kFlagVlimit | kFlagLowRho | kFlagNonFinite)) {
    c.tripped = 1;
    c.trip_step = c.run_step - 1;
    c.time = c.time0;
    c.dtold = c.dtold0;
    c.step = c.step0;
    c.rate_bits = c.rate_bits0;
    c.active = 0;
    return;
  }
  double dt = kHalf * c.dt;
  dt = dt * 2.0;
  c.time = c.time + dt;
  c.nsrc = 2;
}
namespace {
__device__ __forceinline__ unsigned ld_acquire_u32(const unsigned* p) {
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
// polls *p until it reaches target; false after `limit` polls (~0.1 us apart)
__device__ bool wait_at_least(const unsigned* p, unsigned target, long long limit) {
  for (long long k = 0; k < limit; ++k) {
    if (ld_acquire_u32(p) >= target) return true;
    __nanosleep(100);
  }
  return false;
}
static_assert(sizeof(Ctrl) % 8 == 0, "Ctrl moves as 8-byte words");
// a box's control block through L2 (other blocks of the launch write it)
__device__ __forceinline__ Ctrl ctrl_load_cg(const Ctrl* p) {
  Ctrl c;
  const unsigned long long* s = reinterpret_cast<const unsigned long long*>(p);
  unsigned long long* d = reinterpret_cast<unsigned long long*>(&c);
#pragma unroll
  for (int k = 0; k < (int)(sizeof(Ctrl) / 8); ++k) d[k] = __ldcg(s + k);
  return c;
}
__device__ __forceinline__ void ctrl_store_cg(Ctrl* p, const Ctrl& c) {
  unsigned long long* d = reinterpret_cast<unsigned long long*>(p);
  const unsigned long long* s = reinterpret_cast<const unsigned long long*>(&c);
#pragma unroll
  for (int k = 0; k < (int)(sizeof(Ctrl) / 8); ++k) __stcg(d + k, s[k]);
}
}  // namespace

// one tile of either stage in the persistent kernel: a single inlined body with
// the stage as a runtime value (two bodies, or bodies called out of line, spill
// registers) and the tile's extents at run time
template <class S, int PM, bool THREED>
__device__ __forceinline__ void persistent_tile(int stage, const StageArgs& a, const Tile& t,
                                                const Geom& g, Ctrl* C, double dt, int nsrc,
                                                double* sm, double* red_rate,
                                                unsigned* red_flags) {
  stage_tile<S, 2, PM == 1, THREED, false, false, true>(a, t, g, C, dt, nsrc, sm, red_rate,
                                                        red_flags, stage);
}

template <int PM, bool THREED, int SH>
__global__ void __launch_bounds__(NT, 65536 / (NT * 128)) k_batch_persistent(PersistArgs p) {
  using S = typename ShapeSel<SH>::type;
  extern __shared__ double sm[];
  __shared__ Geom sg;
  __shared__ double red_rate[NT / 32];
  __shared__ unsigned red_flags[NT / 32];
  __shared__ long long s_item;
  __shared__ int s_run, s_nsrc;
  __shared__ double s_dt;
  const long long nt = p.ntiles;
  const long long total = 2 * nt * p.nsteps;
  for (;;) {
    if (threadIdx.x == 0) s_item = (long long)atomicAdd(p.head, 1ull);
    __syncthreads();
    const long long w = s_item;
    if (w >= total) break;
    const int step = (int)(w / (2 * nt));
    const int stage = (int)((w / nt) % 2);
    const Tile t = p.a.tiles[w % nt];
    Ctrl* C = p.a.ctrl + t.box;
    const unsigned ntb = (unsigned)p.tiles_of_box[t.box];
    if (threadIdx.x == 0) {
      sg = p.a.geom[t.box];
      // a stage-0 tile needs its box's dt of the step; a stage-1 tile every
      // stage-0 tile of its box (the halo of its stencil)
      const bool ok = stage == 0
                          ? wait_at_least(p.ready + t.box, (unsigned)step + 1u, p.poll_limit)
                          : wait_at_least(p.done0 + t.box, ((unsigned)step + 1u) * ntb,
                                          p.poll_limit);
      if (!ok) atomicOr(p.status, 1);
      __threadfence();
      s_run = ok && __ldcg(&C->active);
      s_dt = __ldcg(&C->dt);
      s_nsrc = __ldcg(&C->nsrc);
    }
    __syncthreads();
    if (s_run) {
      const int X = (p.cur + 2 * step) % 3, Y = (X + 1) % 3, Z = (X + 2) % 3;
      StageArgs a = p.a;
      a.X = p.buf[X];
      a.Y = stage == 0 ? nullptr : p.buf[Y];
      a.out = stage == 0 ? p.buf[Y] : p.buf[Z];
      persistent_tile<S, PM, THREED>(stage, a, t, sg, C, s_dt, s_nsrc, sm, red_rate, red_flags);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      // the block's writes (planes, the box's flags and Courant rate) before the count
      __threadfence();
      if (stage == 0) {
        atomicAdd(p.done0 + t.box, 1u);
      } else if (atomicAdd(p.done1 + t.box, 1u) + 1u == ((unsigned)step + 1u) * ntb) {
        // the box's last stage-1 tile of the step: its clock advances
        // (k_end_batch) and, unless the run ends here, the next dt is set
        // (k_dt_batch); then the box's next step may start
        __threadfence();
        Ctrl c = ctrl_load_cg(C);
        box_end_step(c);
        if (step + 1 < p.nsteps) box_begin_step(c);
        ctrl_store_cg(C, c);
        __threadfence();
        atomicExch(p.ready + t.box, (unsigned)step + 2u);
      }
    }
  }
}

__global__ void k_persist_init(PersistArgs p, int nbox) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b == 0) {
    *p.head = 0ull;
    *p.status = 0;
  }
  if (b >= nbox) return;
  p.done0[b] = 0u;
  p.done1[b] = 0u;
  p.ready[b] = 1u;  // the first step's dt was set by k_dt_batch
}

__global__ void k_wait_selftest(unsigned* never, long long limit, int* status) {
  if (!wait_at_least(never, 1u, limit)) atomicOr(status, 1);
}

template <int PM, bool THREED, int SH>
static cudaError_t launch_persistent_t(const PersistArgs& p, int nbox, cudaStream_t s,
                                       int* blocks_out) {
  const size_t smem = ShapeSel<SH>::type::SMEM_DOUBLES * sizeof(double);
  const void* fn = (const void*)k_batch_persistent<PM, THREED, SH>;
  cudaError_t e = ensure_dyn_smem(fn, smem);
  if (e != cudaSuccess) return e;
  int dev = 0, sms = 0, per_sm = 0;
  if ((e = cudaGetDevice(&dev)) != cudaSuccess) return e;
  if ((e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess)
    return e;
  if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, NT, smem)) != cudaSuccess)
    return e;
  const int blocks = std::max(1, per_sm) * sms;
  k_persist_init<<<(nbox + 127) / 128, 128, 0, s>>>(p, nbox);
  k_batch_persistent<PM, THREED, SH><<<blocks, NT, smem, s>>>(p);
  if (blocks_out) *blocks_out = blocks;
  return cudaGetLastError();
}

template <int SH>
static cudaError_t launch_persistent_s(const PersistArgs& p, int pm, bool threed, int nbox,
                                       cudaStream_t s, int* blocks_out) {
  if (pm == 1)
    return threed ? launch_persistent_t<1, true, SH>(p, nbox, s, blocks_out)
                  : launch_persistent_t<1, false, SH>(p, nbox, s, blocks_out);
  return threed ? launch_persistent_t<0, true, SH>(p, nbox, s, blocks_out)
                : launch_persistent_t<0, false, SH>(p, nbox, s, blocks_out);
}

cudaError_t launch_batch_persistent(const PersistArgs& p, int pm, bool threed, int nbox,
                                    cudaStream_t s, int* blocks_out, int shape) {
  return shape == 1 ? launch_persistent_s<1>(p, pm, threed, nbox, s, blocks_out)
                    : launch_persistent_s<0>(p, pm, threed, nbox, s, blocks_out);
}

cudaError_t persistent_wait_selftest(long long poll_limit, int* gave_up, float* ms) {
  unsigned* never = nullptr;
  int* status = nullptr;
  cudaError_t e = cudaMalloc(&never, sizeof(unsigned));
  if (e != cudaSuccess) return e;
  if ((e = cudaMalloc(&status, sizeof(int))) != cudaSuccess) {
    cudaFree(never);
    return e;
  }
  cudaMemset(never, 0, sizeof(unsigned));
  cudaMemset(status, 0, sizeof(int));
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  cudaEventRecord(e0);
  k_wait_selftest<<<1, 1>>>(never, poll_limit, status);
  cudaEventRecord(e1);
  e = cudaEventSynchronize(e1);
  if (e == cudaSuccess && ms) cudaEventElapsedTime(ms, e0, e1);
  int h = 0;
  if (e == cudaSuccess) e = cudaMemcpy(&h, status, sizeof(int), cudaMemcpyDeviceToHost);
  if (gave_up) *gave_up = h;
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(never);
  cudaFree(status);
  return e;
}

template <int STAGE, int PM, bool THREED, bool GRAV, int SH>
static cudaError_t launch_stage_t(const StageArgs& a, int ntiles, cudaStream_t s) {
  const size_t smem = ShapeSel<SH>::type::SMEM_DOUBLES * sizeof(double);
  cudaError_t e = ensure_dyn_smem((const void*)k_stage<STAGE, PM, THREED, GRAV, SH>, smem);
  if (e != cudaSuccess) return e;
  if (ntiles <= 0) return cudaSuccess;
  k_stage<STAGE, PM, THREED, GRAV, SH><<<ntiles, NT, smem, s>>>(a);
  return cudaGetLastError();
}

template <int STAGE, bool GRAV, int SH>
static cudaError_t launch_stage_g(int pm, bool threed, const StageArgs& a, int ntiles,
                                  cudaStream_t s) {
  if (pm == 1) return threed ? launch_stage_t<STAGE, 1, true, GRAV, SH>(a, ntiles, s)
                             : launch_stage_t<STAGE, 1, false, GRAV, SH>(a, ntiles, s);
  return threed ? launch_stage_t<STAGE, 0, true, GRAV, SH>(a, ntiles, s)
                : launch_stage_t<STAGE, 0, false, GRAV, SH>(a, ntiles, s);
}

// a.G set: the step has a gravitational force (instances with the force terms,
// tile shape 0 only: the batched path, the one that tunes the shape, has no
// force, and a grid with the tabulated EOS or flux_ang and a force runs the
// per-phase kernels).  Shape 2: the tabulated EOS; shape 3: flux_ang.
template <int STAGE>
static cudaError_t launch_stage_s(int pm, bool threed, const StageArgs& a, int ntiles,
                                  cudaStream_t s, int shape) {
  if (a.G) {
    if (shape != 0) return cudaErrorInvalidValue;
    return launch_stage_g<STAGE, true, 0>(pm, threed, a, ntiles, s);
  }
  if (shape == 2) return launch_stage_g<STAGE, false, 2>(pm, threed, a, ntiles, s);
  if (shape == 3) return launch_stage_g<STAGE, false, 3>(pm, threed, a, ntiles, s);
  return shape == 1 ? launch_stage_g<STAGE, false, 1>(pm, threed, a, ntiles, s)
                    : launch_stage_g<STAGE, false, 0>(pm, threed, a, ntiles, s);
}

// pm: 1 every box has power-of-two spacings, 0 otherwise
cudaError_t launch_stage(int stage, int pm, bool threed, const StageArgs& a, int ntiles,
                         cudaStream_t s, int shape) {
  return stage == 0 ? launch_stage_s<0>(pm, threed, a, ntiles, s, shape)
                    : launch_stage_s<1>(pm, threed, a, ntiles, s, shape);
}

size_t stage_smem_bytes(int shape) {
  return (shape == 3   ? Shape3::SMEM_DOUBLES
          : shape == 2 ? Shape2::SMEM_DOUBLES
          : shape == 1 ? Shape1::SMEM_DOUBLES
                       : Shape0::SMEM_DOUBLES) *
         sizeof(double);
}

// ------------------------------------------------------------------ clock kernels
// dt control of main.f90:266-281 and 342, per box
__global__ void k_dt(Ctrl* ctrl, int n) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= n) return;
  Ctrl& c = ctrl[b];
  if (!(c.time < c.endtime) || c.step >= 1000000 || c.step >= c.max_step) {
    c.active = 0;
    return;
  }
  c.step = c.step + 1;
  const double rate = __longlong_as_double((long long)c.rate_bits);
  c.rate = rate;
  c.rate_bits = 0ull;
  double dt = c.cfl / rate;            // courant.f90:28
  dt = dt * 1.0;                       // dt*f1, f1=one
  if (c.step > 1 && c.dtold > 0.0) dt = fmin(dt, c.dtold * 1.1);
  c.dtold = dt;
  if (dt + c.time > c.endtime) dt = c.endtime - c.time;
  dt = dt * kHalf;                     // source(time,0) runs with dt/2
  dt = dt * 2.0;                       // flux stages run with the full dt
  c.dt = dt;
  c.active = 1;
}

// main.f90:471,544-545
__global__ void k_end(Ctrl* ctrl, int n) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= n) return;
  Ctrl& c = ctrl[b];
  if (!c.active) return;
  double dt = kHalf * c.dt;
  dt = dt * 2.0;
  c.time = c.time + dt;
}

// batched boxes: as k_dt/k_end, plus the saved clock and the trip of a box
// whose step raised a guard (its planes then keep the step's input)
__global__ void k_dt_batch(Ctrl* ctrl, int n) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= n) return;
  box_begin_step(ctrl[b]);
}
__global__ void k_end_batch(Ctrl* ctrl, int n) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= n) return;
  box_end_step(ctrl[b]);
}
cudaError_t launch_dt_batch(Ctrl* ctrl, int nbox, cudaStream_t s) {
  k_dt_batch<<<(nbox + 127) / 128, 128, 0, s>>>(ctrl, nbox);
  return cudaGetLastError();
}
cudaError_t launch_end_batch(Ctrl* ctrl, int nbox, cudaStream_t s) {
  k_end_batch<<<(nbox + 127) / 128, 128, 0, s>>>(ctrl, nbox);
  return cudaGetLastError();
}

cudaError_t launch_dt(Ctrl* ctrl, int nbox, cudaStream_t s) {
  k_dt<<<(nbox + 127) / 128, 128, 0, s>>>(ctrl, nbox);
  return cudaGetLastError();
}
cudaError_t launch_end(Ctrl* ctrl, int nbox, cudaStream_t s) {
  k_end<<<(nbox + 127) / 128, 128, 0, s>>>(ctrl, nbox);
  return cudaGetLastError();
}

// ------------------------------------------------------------------ phase kernels
namespace {

constexpr int PB = 256;
inline int nblk(long long n) { return (int)((n + PB - 1) / PB); }

__device__ __forceinline__ bool is_ghost(const Geom& g, int x, int y, int z) {
  return x < g.ax0 || x >= g.ax1 || y < g.ay0 || y >= g.ay1 ||
         (g.threed && (z < g.az0 || z >= g.az1));
}

// state.f90:29-87, fixed gamma
__global__ void k_phase_state(Geom g, PhaseArrays a, Ctrl* ctrl) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= g.ng) return;
  const long long n = g.ng;
  const double d = a.cons[i];
  const double u1 = a.u[i], u2 = a.u[n + i], u3 = a.u[2 * n + i];
  const double ekin = kin_rho_u(d, u1, u2, u3);
  double eps = fmax(a.cons[4 * n + i] - ekin, g.small_eps);
  if (g.tab) {
    // state.f90:60-79
    double tk, m, gam;
    if (g.nz == 1) {
      // disk: surface density over twice the scale height
      const int ix = (int)(i % g.nx), iy = (int)((i / g.nx) % g.ny);
      const double x = g.dx * ((double)(ix + 1) - ((double)g.nx + 1.0) / 2.0);
      const double y = g.dy * ((double)(iy + 1) - ((double)g.ny + 1.0) / 2.0);
      const double hscale = sqrt((a.adindx[i] - 1.0) * eps / (2.0 * ekin) * (x * x + y * y));
      eps = eps / (2.0 * hscale);
      const double rho = d / (2.0 * hscale);
      get_gamma2(a.eos, eps, rho, tk, m, gam);
    } else {
      get_gamma2(a.eos, eps, d, tk, m, gam);
    }
    a.muc[i] = m;
    a.adindx[i] = gam;
    double p = (d * tk * g.rgas / m);
    if (d < kLowRho) {
      p = g.rgas * a.eos.tk_bgrnd / g.muc * d;
      eps = p / (g.gam - 1.0);
      a.cons[4 * n + i] = eps + ekin;
      atomicOr(&ctrl->flags, (unsigned)kFlagLowRho);
    }
    a.p[i] = p;
    return;
  }
  a.adindx[i] = g.gam;
  if (d < kLowRho) {
    const double tk = fmin(5e3, a.p[i] / (d * g.rgas) * g.muc);
    const double p = (d * tk * g.rgas / g.muc);
    a.p[i] = p;
    eps = p / (g.gam - 1.0);
    a.cons[4 * n + i] = eps + ekin;
    atomicOr(&ctrl->flags, (unsigned)kFlagLowRho);
  } else {
    a.p[i] = eps * (g.gam - 1.0);
  }
}

// velocity.f90:18-53
__global__ void k_phase_velocity(Geom g, PhaseArrays a, Ctrl* ctrl) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= g.ng) return;
  const long long n = g.ng;
  double* c = a.cons;
  const double d = c[i];
  double u[3];
  for (int k = 0; k < 3; ++k) u[k] = c[(k + 1) * n + i] / d;
  int flag = 0;
  for (int k = 0; k < 3; ++k)
    if (fabs(u[k]) > g.vlimit) flag = 1;
  if (flag) {
    double ekin = kin_mom(d, c[n + i], c[2 * n + i], c[3 * n + i]);
    double speed = 0.0;
    for (int k = 0; k < 3; ++k) speed = speed + u[k] * u[k];
    speed = sqrt(speed);
    for (int k = 0; k < 3; ++k) {
      u[k] = u[k] * g.vlimit / speed;
      c[(k + 1) * n + i] = u[k] * d;
    }
    double E = c[4 * n + i] - ekin;
    ekin = kin_mom(d, c[n + i], c[2 * n + i], c[3 * n + i]);
    c[4 * n + i] = fmax(E, g.small_eps) + ekin;
    atomicOr(&ctrl->flags, (unsigned)kFlagVlimit);
  }
  for (int k = 0; k < 3; ++k) a.u[k * n + i] = u[k];
}

// courant.f90:19-23 (max over every cell, ghosts included)
__global__ void k_phase_courant(Geom g, PhaseArrays a, Ctrl* ctrl) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  const long long n = g.ng;
  double r = 0.0;
  bool bad = false;
  if (i < n) {
    const double sound = sqrt(a.adindx[i] * a.p[i] / a.cons[i]);
    const double r0 = (sound + fabs(a.u[i])) / g.dx + (sound + fabs(a.u[n + i])) / g.dy +
                      (sound + fabs(a.u[2 * n + i])) / g.dz;
    if (!(r0 >= 0.0)) bad = true;
    r = fmax(r, r0);
  }
  __shared__ double wm[PB / 32];
  r = warp_max(r);
  if ((threadIdx.x & 31) == 0) wm[threadIdx.x >> 5] = r;
  __syncthreads();
  if (threadIdx.x == 0) {
    double m = 0.0;
    for (int k = 0; k < PB / 32; ++k) m = fmax(m, wm[k]);
    atomicMax(&ctrl->rate_bits, (unsigned long long)__double_as_longlong(m));
  }
  if (bad) atomicOr(&ctrl->flags, (unsigned)kFlagNonFinite);
}

// avisc (avisc.f90:13-23): qq(d) = avmag_d*min(0, u_d(b+) - u_d(b-))**2 on the
// cells with boundary > 0 (the ghost layers -- the reference's test, kept as
// written), zero elsewhere.  b are the cell's neighbours through get_boundary
// (utils.f90:62-73): a neighbour in a ghost layer becomes the cell itself.  The
// neighbour table is init_grid.f90:178-261: the outer layer (boundary 1) stores
// only its donor, two cells inward, in ineigh(1) (the +y slot) and leaves the
// other five at 0, an index outside grid(1:ngrid) that the reference reads
// anyway; here such an entry resolves to the cell itself, like a ghost
// neighbour.  The inner layer (boundary 2) has the six neighbours, with the z
// pair set to the cell itself when nz < 6.
__global__ void k_phase_avisc(Geom g, const double* u, double ax, double ay, double az,
                              double* qq) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  const long long n = g.ng;
  if (i >= n) return;
  const int x = (int)(i % g.nx), y = (int)((i / g.nx) % g.ny), z = (int)(i / g.sz);
  // boundary flag of a cell (init_grid.f90:82-105), 0-based coordinates
  auto flag = [&](int cx, int cy, int cz) -> int {
    const bool zl = g.nz >= 6;
    if (cx == 0 || cx == g.nx - 1 || cy == 0 || cy == g.ny - 1 ||
        (zl && (cz == 0 || cz == g.nz - 1)))
      return 1;
    if (cx == 1 || cx == g.nx - 2 || cy == 1 || cy == g.ny - 2 ||
        (zl && (cz == 1 || cz == g.nz - 2)))
      return 2;
    return 0;
  };
  const int b = flag(x, y, z);
  double q1 = 0.0, q2 = 0.0, q3 = 0.0;
  if (b > 0) {
    // neighbours (+y, -y, +x, -x, +z, -z) as cell offsets, -1 = the cell itself
    long long nb[6];
    int cx[6], cy[6], cz[6];
    for (int k = 0; k < 6; ++k) { nb[k] = -1; cx[k] = x; cy[k] = y; cz[k] = z; }
    if (b == 1) {
      // init_grid.f90:180-203: the donor, two cells inward, in ineigh(1)
      if (x == 0) cx[0] = x + 2;
      else if (x == g.nx - 1) cx[0] = x - 2;
      else if (y == 0) cy[0] = y + 2;
      else if (y == g.ny - 1) cy[0] = y - 2;
      else if (z == 0) cz[0] = g.nz < 6 ? z : z + 2;
      else cz[0] = g.nz < 6 ? z : z - 2;
      nb[0] = 0;
    } else {
      cy[0] = y + 1; cy[1] = y - 1; cx[2] = x + 1; cx[3] = x - 1;
      if (g.nz >= 6) { cz[4] = z + 1; cz[5] = z - 1; }
      for (int k = 0; k < 6; ++k) nb[k] = 0;
    }
    long long bi[6];
    for (int k = 0; k < 6; ++k) {
      const long long j = cx[k] + cy[k] * g.sy + cz[k] * g.sz;
      bi[k] = (nb[k] < 0 || flag(cx[k], cy[k], cz[k]) > 0) ? i : j;
    }
    const double m1 = fmin(0.0, u[bi[2]] - u[bi[3]]);
    const double m2 = fmin(0.0, u[n + bi[0]] - u[n + bi[1]]);
    const double m3 = fmin(0.0, u[2 * n + bi[4]] - u[2 * n + bi[5]]);
    q1 = ax * (m1 * m1);
    q2 = ay * (m2 * m2);
    q3 = az * (m3 * m3);
  }
  qq[i] = q1;
  qq[n + i] = q2;
  qq[2 * n + i] = q3;
}

__global__ void k_phase_courant_finish(Ctrl* ctrl) {
  Ctrl& c = *ctrl;
  c.rate = __longlong_as_double((long long)c.rate_bits);
  c.dt = c.cfl / c.rate;
}

// source.f90:148-191 (interior cells)
__global__ void k_phase_source(Geom g, PhaseArrays a, Ctrl* ctrl, double mult) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= g.ng) return;
  const int x = (int)(i % g.nx), y = (int)((i / g.nx) % g.ny), z = (int)(i / g.sz);
  if (is_ghost(g, x, y, z)) return;
  const long long n = g.ng;
  const double dt = mult * ctrl->dt;
  double d = a.cons[i], m1 = a.cons[n + i], m2 = a.cons[2 * n + i], m3 = a.cons[3 * n + i],
         E = a.cons[4 * n + i];
  double g1 = 0.0, g2 = 0.0, g3 = 0.0;
  if (a.gforce) {
    g1 = a.gforce[i];
    g2 = a.gforce[n + i];
    g3 = a.gforce[2 * n + i];
  }
  source_gravity(d, m1, m2, m3, E, g1, g2, g3, a.u[i], a.u[n + i], a.u[2 * n + i], dt,
                 g.small_eps);
  a.cons[n + i] = m1;
  a.cons[2 * n + i] = m2;
  a.cons[3 * n + i] = m3;
  a.cons[4 * n + i] = E;
}

// set_ghost_cells as gather (values before the sweep) + scatter
__global__ void k_ghost_gather(int nghost, const int32_t* src, const uint8_t* sgn,
                               const double* cons, long long n, double* tmp) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= nghost) return;
  const long long s = src[k];
  const unsigned m = sgn[k];
  tmp[k] = cons[s];
  tmp[nghost + k] = (m & 1) ? -cons[n + s] : cons[n + s];
  tmp[2 * nghost + k] = (m & 2) ? -cons[2 * n + s] : cons[2 * n + s];
  tmp[3 * nghost + k] = (m & 4) ? -cons[3 * n + s] : cons[3 * n + s];
  tmp[4 * nghost + k] = cons[4 * n + s];
}
__global__ void k_ghost_scatter(int nghost, const int32_t* dst, const double* tmp, double* cons,
                                long long n) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= nghost) return;
  const long long d = dst[k];
  for (int q = 0; q < 5; ++q) cons[q * n + d] = tmp[q * nghost + k];
}

// flux.f90:47-116: slopes and interface states of every cell.
// states layout: [(dir*2+side)*7 + q][cell], side 0 = minus, 1 = plus,
// q = rho, u1, u2, u3, p, eps, gamma.
// cell centre of cell i (init_grid.f90:84-92)
__device__ __forceinline__ void cell_xy(const Geom& g, long long i, double& x, double& y) {
  const int ix = (int)(i % g.nx), iy = (int)((i / g.nx) % g.ny);
  x = g.dx * ((double)(ix + 1) - ((double)g.nx + 1.0) / 2.0);
  y = g.dy * ((double)(iy + 1) - ((double)g.ny + 1.0) / 2.0);
}

// flux_ang.f90:44-62: (m1, m2) -> (radial momentum, angular momentum) about the
// z axis through (0, -yoffset), on cons and (stage 1) cons_old
__global__ void k_ang_to(Geom g, PhaseArrays a, int avg) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= g.ng) return;
  const long long n = g.ng;
  double x, y;
  cell_xy(g, i, x, y);
  y = y + g.yoff;
  const double r = sqrt(x * x + y * y);
  double m1 = a.cons[n + i], m2 = a.cons[2 * n + i];
  a.cons[n + i] = (m1 * x + m2 * y) / r;
  a.cons[2 * n + i] = x * m2 - y * m1;
  if (avg > 0) {
    m1 = a.cons_old[n + i];
    m2 = a.cons_old[2 * n + i];
    a.cons_old[n + i] = (m1 * x + m2 * y) / r;
    a.cons_old[2 * n + i] = x * m2 - y * m1;
  }
}

// flux.f90:253-482 (and flux_ang.f90:301-518 when ANG): slopes and face states
// of every cell.  States: [(dir*2 + side)*NQ + k] planes, side 0 minus, 1 plus;
// k = rho, u1, u2, u3, p, eps, gamma (and, with ANG, the radial and angular
// momenta of the transformed cons(2), cons(3)).
template <bool ANG>
__global__ void k_phase_states(Geom g, PhaseArrays a, Ctrl* ctrl) {
  constexpr int NQ = ANG ? 9 : 7;
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= g.ng) return;
  const long long n = g.ng;
  const int x = (int)(i % g.nx), y = (int)((i / g.nx) % g.ny), z = (int)(i / g.sz);
  const bool ghost = is_ghost(g, x, y, z);
  const double dt = ctrl->dt;
  const double* c = a.cons;
  const double* u = a.u;
  const double ds[3] = {g.dx, g.dy, g.dz};
  const long long st[3] = {1, g.sy, g.threed ? g.sz : 0};
  const double d0 = c[i];
  const double sound = sqrt(a.p[i] * a.adindx[i] / d0);
  const double eps0 = recon_eps(d0, c[4 * n + i], u[i], u[n + i], u[2 * n + i], g.small_eps);
  // unrolled: the per-direction constants stay in registers, not on the stack
#pragma unroll
  for (int dir = 0; dir < 3; ++dir) {
    const long long im = ghost ? i : i - st[dir], ip = ghost ? i : i + st[dir];
    const long long idx3[3] = {im, i, ip};
    double sl[NQ];
    for (int k = 0; k < 3; ++k)
      sl[1 + k] = slope3(u[k * n + im], u[k * n + i], u[k * n + ip]);
    double eps[3];
    for (int k = 0; k < 3; ++k) {
      const long long j = idx3[k];
      eps[k] = recon_eps(c[j], c[4 * n + j], u[j], u[n + j], u[2 * n + j], g.small_eps);
    }
    sl[4] = slope3(a.p[im], a.p[i], a.p[ip]);
    sl[0] = slope3(c[im], c[i], c[ip]);
    sl[5] = slope3(eps[0], eps[1], eps[2]);
    sl[6] = slope3(a.adindx[im], a.adindx[i], a.adindx[ip]);
    if (ANG) {
      sl[7] = slope3(c[n + im], c[n + i], c[n + ip]);
      sl[NQ - 1] = slope3(c[2 * n + im], c[2 * n + i], c[2 * n + ip]);
    }
    const double ud = u[dir * n + i];
    const double lp = fmax(ud + sound, 0.0) * dt / ds[dir];
    const double lm = fmin(ud - sound, 0.0) * dt / ds[dir];
    double q[NQ];
    q[0] = d0; q[1] = u[i]; q[2] = u[n + i]; q[3] = u[2 * n + i];
    q[4] = a.p[i]; q[5] = eps0; q[6] = a.adindx[i];
    if (ANG) {
      q[7] = c[n + i];
      q[NQ - 1] = c[2 * n + i];
    }
#pragma unroll
    for (int k = 0; k < NQ; ++k) {
      const double mi = q[k] + kHalf * (-1.0 - lm) * sl[k];
      const double pl = q[k] + kHalf * (1.0 - lp) * sl[k];
      // the zero transverse terms of flux.f90:391-479 (not applied to the
      // momenta of flux_ang)
      const bool tr = k < 7;
      a.states[((dir * 2 + 0) * NQ + k) * n + i] = tr ? mi + 0.0 * (dt * kHalf / ds[dir]) : mi;
      a.states[((dir * 2 + 1) * NQ + k) * n + i] = tr ? pl + 0.0 * (dt * kHalf / ds[dir]) : pl;
    }
  }
}

// HLL flux through the face between cells lc and rc in direction dir
// (flux.f90:487-590); with ANG the momenta are the transformed ones and the
// pressure terms follow flux_ang.f90:523-618 at the updated cell's centre (x, y,
// r, without yoffset)
template <bool ANG>
__device__ __forceinline__ void phase_face(const double* S, long long n, int dir, long long lc,
                                           long long rc, double x, double y, double r,
                                           double F[5]) {
  constexpr int NQ = ANG ? 9 : 7;
  // plus state of the low cell, minus state of the high cell (flux.f90:504-530)
  const double* Lp = S + ((dir * 2 + 1) * NQ) * n;
  const double* Rm = S + ((dir * 2 + 0) * NQ) * n;
  const double dl = Lp[lc], vxl = Lp[n + lc], vyl = Lp[2 * n + lc], vzl = Lp[3 * n + lc],
               pl = Lp[4 * n + lc], el = Lp[5 * n + lc], gl = Lp[6 * n + lc];
  const double dr = Rm[rc], vxr = Rm[n + rc], vyr = Rm[2 * n + rc], vzr = Rm[3 * n + rc],
               pr = Rm[4 * n + rc], er = Rm[5 * n + rc], gr = Rm[6 * n + rc];
  double sl[5], sr[5], fl[5], fr[5];
  sl[0] = dl;
  sr[0] = dr;
  if (ANG) {
    sl[1] = Lp[7 * n + lc]; sl[2] = Lp[(NQ - 1) * n + lc];
    sr[1] = Rm[7 * n + rc]; sr[2] = Rm[(NQ - 1) * n + rc];
  } else {
    sl[1] = dl * vxl; sl[2] = dl * vyl;
    sr[1] = dr * vxr; sr[2] = dr * vyr;
  }
  sl[3] = dl * vzl;
  sl[4] = el + kHalf * dl * (vxl * vxl + vyl * vyl + vzl * vzl);
  sr[3] = dr * vzr;
  sr[4] = er + kHalf * dr * (vxr * vxr + vyr * vyr + vzr * vzr);
  for (int k = 0; k < 5; ++k) { fl[k] = 0.0; fr[k] = 0.0; }
  double vl, vr;
  if (ANG) {
    if (dir == 0) {
      vr = vxr; vl = vxl;
      fl[1] = pl * x / r; fr[1] = pr * x / r;
      fl[2] = -(pl * y); fr[2] = -(pr * y);
    } else if (dir == 1) {
      vr = vyr; vl = vyl;
      fl[1] = pl * y / r; fr[1] = pr * y / r;
      fl[2] = pl * x; fr[2] = pr * x;
    } else {
      vr = vzr; vl = vzl; fl[3] = pl; fr[3] = pr;
    }
  } else {
    if (dir == 0) { vr = vxr; vl = vxl; fl[1] = pl; fr[1] = pr; }
    else if (dir == 1) { vr = vyr; vl = vyl; fl[2] = pl; fr[2] = pr; }
    else { vr = vzr; vl = vzl; fl[3] = pl; fr[3] = pr; }
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
  const double cr = sqrt(gr * pr / dr);
  const double cl = sqrt(gl * pl / dl);
  const double ap = fmax(fmax(0.0, vr + cr), vl + cl);
  const double am = fmax(fmax(0.0, -(vr - cr)), -(vl - cl));
  for (int k = 0; k < 5; ++k) F[k] = (ap * fl[k] + am * fr[k] - ap * am * (sr[k] - sl[k])) / (ap + am);
}

// flux.f90:121-230 (flux_ang.f90:149-276 with ANG): face fluxes of interior
// cells, update of every cell, (ANG) momenta back to (m1, m2), floors
template <bool ANG>
__global__ void k_phase_update(Geom g, PhaseArrays a, Ctrl* ctrl, int avg) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= g.ng) return;
  const long long n = g.ng;
  const int x = (int)(i % g.nx), y = (int)((i / g.nx) % g.ny), z = (int)(i / g.sz);
  const double dt = ctrl->dt;
  double cx = 0.0, cy = 0.0, cr = 0.0;
  if (ANG) {
    cell_xy(g, i, cx, cy);
    cr = sqrt(cx * cx + cy * cy);
  }
  double ft[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
  if (!is_ghost(g, x, y, z)) {
    const long long st[3] = {1, g.sy, g.threed ? g.sz : 0};
    double fm[3][5], fp[3][5];
    for (int dir = 0; dir < 3; ++dir) {
      if (ANG) {
        // the pressure terms depend on the updated cell: both faces here
        phase_face<ANG>(a.states, n, dir, i - st[dir], i, cx, cy, cr, fm[dir]);
        phase_face<ANG>(a.states, n, dir, i, i + st[dir], cx, cy, cr, fp[dir]);
      } else {
        const double* F = a.states + 42 * n;  // k_phase_faces
        for (int k = 0; k < 5; ++k) {
          fm[dir][k] = F[(dir * 5 + k) * n + i - st[dir]];
          fp[dir][k] = F[(dir * 5 + k) * n + i];
        }
      }
    }
    for (int k = 0; k < 5; ++k)
      ft[k] = -(g.ayz * (fp[0][k] - fm[0][k]) + g.axz * (fp[1][k] - fm[1][k]) +
                g.axy * (fp[2][k] - fm[2][k])) * dt / g.vol;
  }
  double v[5];
  for (int k = 0; k < 5; ++k) {
    const double c = a.cons[k * n + i];
    v[k] = avg == 0 ? c + ft[k] : kHalf * (a.cons_old[k * n + i] + c + ft[k]);
  }
  if (ANG) {
    // flux_ang.f90:247-270, about the axis through (0, -yoffset)
    const double ty = cy + g.yoff, tr = sqrt(cx * cx + ty * ty);
    const double rmom = v[1], angmom = v[2];
    v[1] = (rmom * cx - angmom * ty / tr) / tr;
    v[2] = (rmom * ty + angmom * cx / tr) / tr;
    if (avg > 0) {
      const double ro = a.cons_old[n + i], ao = a.cons_old[2 * n + i];
      a.cons_old[n + i] = (ro * cx - ao * ty / tr) / tr;
      a.cons_old[2 * n + i] = (ro * ty + ao * cx / tr) / tr;
    }
  }
  floors(v[0], v[1], v[2], v[3], v[4], g.small_rho, g.small_eps);
  bool bad = false;
  for (int k = 0; k < 5; ++k) {
    a.cons[k * n + i] = v[k];
    if (!isfinite(v[k])) bad = true;
  }
  if (bad) atomicOr(&ctrl->flags, (unsigned)kFlagNonFinite);
}

// HLL flux of every face once (fixed frame): F[dir][i] = flux through the face
// between cells i and i + stride(dir), from the face states; without z ghosts
// (nz < 6) the z "face" is the cell with itself, as the update reads it
__global__ void k_phase_faces(Geom g, PhaseArrays a, double* F) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= g.ng) return;
  const long long n = g.ng;
  const long long st[3] = {1, g.sy, g.threed ? g.sz : 0};
  for (int dir = 0; dir < 3; ++dir) {
    if (i + st[dir] >= n) continue;
    double f[5];
    phase_face<false>(a.states, n, dir, i, i + st[dir], 0.0, 0.0, 0.0, f);
    for (int k = 0; k < 5; ++k) F[(dir * 5 + k) * n + i] = f[k];
  }
}

__global__ void k_copy5(const double* src, double* dst, long long n) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= 5 * n) return;
  dst[i] = src[i];
}

// fused state (X planes) -> reference arrays: interior cons = src^(nsrc-1)(X)
__global__ void k_f2p_interior(Geom g, const double* X, long long xps, int nsrc, PhaseArrays a) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= g.ng) return;
  const int x = (int)(i % g.nx), y = (int)((i / g.nx) % g.ny), z = (int)(i / g.sz);
  if (is_ghost(g, x, y, z)) return;
  const long long n = g.ng;
  Cons c{X[i], X[xps + i], X[2 * xps + i], X[3 * xps + i], X[4 * xps + i]};
  apply_sources(c, nsrc - 1, g.small_eps);
  a.cons[i] = c.d;
  a.cons[n + i] = c.m1;
  a.cons[2 * n + i] = c.m2;
  a.cons[3 * n + i] = c.m3;
  a.cons[4 * n + i] = c.E;
}
__global__ void k_fill_resolved(int nghost, const int32_t* dst, const int32_t* src,
                                const uint8_t* sgn, double* cons, long long n) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= nghost) return;
  const long long s = src[k], d = dst[k];
  const unsigned m = sgn[k];
  cons[d] = cons[s];
  cons[n + d] = (m & 1) ? -cons[n + s] : cons[n + s];
  cons[2 * n + d] = (m & 2) ? -cons[2 * n + s] : cons[2 * n + s];
  cons[3 * n + d] = (m & 4) ? -cons[3 * n + s] : cons[3 * n + s];
  cons[4 * n + d] = cons[4 * n + s];
}
// the pressure state() leaves at the end of a step with a force (main.f90:513):
// from the cons after source(1) and the velocity array of before it (UC, the
// velocity after flux(1)), a ghost's as its donor's (|u| is the same)
__global__ void k_p_from_uc(Geom g, PhaseArrays a, const double* uc) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= g.ng) return;
  const int x = (int)(i % g.nx), y = (int)((i / g.nx) % g.ny), z = (int)(i / g.sz);
  if (is_ghost(g, x, y, z)) return;
  const long long n = g.ng;
  a.p[i] = eos_pressure(a.cons[i], a.cons[4 * n + i], uc[i], uc[n + i], uc[2 * n + i], g.gm1,
                        g.small_eps);
}
__global__ void k_p_ghosts(int nghost, const int32_t* dst, const int32_t* src, double* p) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k < nghost) p[dst[k]] = p[src[k]];
}

// Host-overlapped step: z slabs of a cell range [i0, i1) between the reference's
// AoS layout (5 doubles per cell, as on the host) and the fused planes X.
__global__ void k_slab_in(const double* aos, double* X, long long ps, long long i0, long long i1) {
  const long long i = i0 + blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= i1) return;
  for (int q = 0; q < 5; ++q) X[q * ps + i] = aos[5 * i + q];
}
// the reference cons of the interior cells of the slab (as k_f2p_interior)
__global__ void k_slab_out(Geom g, const double* X, long long ps, int nsrc, double* aos,
                           long long i0, long long i1) {
  const long long i = i0 + blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= i1) return;
  const int x = (int)(i % g.nx), y = (int)((i / g.nx) % g.ny), z = (int)(i / g.sz);
  if (is_ghost(g, x, y, z)) return;
  Cons c{X[i], X[ps + i], X[2 * ps + i], X[3 * ps + i], X[4 * ps + i]};
  apply_sources(c, nsrc - 1, g.small_eps);
  aos[5 * i] = c.d;
  aos[5 * i + 1] = c.m1;
  aos[5 * i + 2] = c.m2;
  aos[5 * i + 3] = c.m3;
  aos[5 * i + 4] = c.E;
}
// the ghosts [g0, g1) of the resolved plan (as k_fill_resolved; donors already written)
__global__ void k_slab_ghosts(const int32_t* dst, const int32_t* src, const uint8_t* sgn,
                              double* aos, int g0, int g1) {
  const int k = g0 + blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= g1) return;
  const long long s = src[k], d = dst[k];
  const unsigned m = sgn[k];
  aos[5 * d] = aos[5 * s];
  aos[5 * d + 1] = (m & 1) ? -aos[5 * s + 1] : aos[5 * s + 1];
  aos[5 * d + 2] = (m & 2) ? -aos[5 * s + 2] : aos[5 * s + 2];
  aos[5 * d + 3] = (m & 4) ? -aos[5 * s + 3] : aos[5 * s + 3];
  aos[5 * d + 4] = aos[5 * s + 4];
}
// velocity and pressure arrays of the reference after the last state()/velocity()
__global__ void k_f2p_prims(Geom g, PhaseArrays a) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= g.ng) return;
  const long long n = g.ng;
  const double d = a.cons[i];
  const double u1 = a.cons[n + i] / d, u2 = a.cons[2 * n + i] / d, u3 = a.cons[3 * n + i] / d;
  a.u[i] = u1;
  a.u[n + i] = u2;
  a.u[2 * n + i] = u3;
  a.p[i] = eos_pressure(d, a.cons[4 * n + i], u1, u2, u3, g.gm1, g.small_eps);
  a.adindx[i] = g.gam;
}

__global__ void k_check_cells(Geom g, PhaseArrays a, Ctrl* ctrl) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= g.ng) return;
  const long long n = g.ng;
  const double d = a.cons[i];
  bool ok = d >= kLowRho;
  for (int k = 0; k < 3; ++k) ok = ok && (a.u[k * n + i] == a.cons[(k + 1) * n + i] / d);
  if (!ok) atomicOr(&ctrl->flags, (unsigned)kFlagNotClean);
}
__global__ void k_check_ghosts(int nghost, const int32_t* dst, const int32_t* src,
                               const uint8_t* sgn, const double* cons, long long n, Ctrl* ctrl) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= nghost) return;
  const long long s = src[k], d = dst[k];
  const unsigned m = sgn[k];
  bool ok = cons[d] == cons[s] && cons[4 * n + d] == cons[4 * n + s];
  ok = ok && cons[n + d] == ((m & 1) ? -cons[n + s] : cons[n + s]);
  ok = ok && cons[2 * n + d] == ((m & 2) ? -cons[2 * n + s] : cons[2 * n + s]);
  ok = ok && cons[3 * n + d] == ((m & 4) ? -cons[3 * n + s] : cons[3 * n + s]);
  if (!ok) atomicOr(&ctrl->flags, (unsigned)kFlagNotClean);
}

__global__ void k_aos_to_soa(const double* aos, double* soa, long long n, int k) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= n) return;
  for (int q = 0; q < k; ++q) soa[q * n + i] = aos[i * k + q];
}
__global__ void k_soa_to_aos(const double* soa, double* aos, long long n, int k) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= n) return;
  for (int q = 0; q < k; ++q) aos[i * k + q] = soa[q * n + i];
}

}  // namespace

cudaError_t phase_state(const Geom& g, PhaseArrays& a, Ctrl* ctrl, cudaStream_t s) {
  k_phase_state<<<nblk(g.ng), PB, 0, s>>>(g, a, ctrl);
  return cudaGetLastError();
}
cudaError_t phase_velocity(const Geom& g, PhaseArrays& a, Ctrl* ctrl, cudaStream_t s) {
  k_phase_velocity<<<nblk(g.ng), PB, 0, s>>>(g, a, ctrl);
  return cudaGetLastError();
}
cudaError_t phase_courant(const Geom& g, PhaseArrays& a, Ctrl* ctrl, cudaStream_t s) {
  k_phase_courant<<<nblk(g.ng), PB, 0, s>>>(g, a, ctrl);
  return cudaGetLastError();
}
cudaError_t phase_avisc(const Geom& g, const double* u, const double avmag[3], double* qq,
                        cudaStream_t s) {
  k_phase_avisc<<<nblk(g.ng), PB, 0, s>>>(g, u, avmag[0], avmag[1], avmag[2], qq);
  return cudaGetLastError();
}
cudaError_t phase_courant_finish(Ctrl* ctrl, cudaStream_t s) {
  k_phase_courant_finish<<<1, 1, 0, s>>>(ctrl);
  return cudaGetLastError();
}
// calc_gforce (utils.f90:549-571): central differences of the potential on
// interior cells, g = -(phi(+) - phi(-))/(2 d) per axis; the z neighbours of a
// grid without z ghost layers are the cell itself.  Ghost rows are set to zero
// (source() reads interior cells only).
__global__ void k_calc_gforce(Geom g, const double* phi, double* gf) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= g.ng) return;
  const long long n = g.ng;
  const int x = (int)(i % g.nx), y = (int)((i / g.nx) % g.ny), z = (int)(i / g.sz);
  if (is_ghost(g, x, y, z)) {
    gf[i] = 0.0;
    gf[n + i] = 0.0;
    gf[2 * n + i] = 0.0;
    return;
  }
  const long long sz = g.threed ? g.sz : 0;
  gf[i] = -(phi[i + 1] - phi[i - 1]) / (2.0 * g.dx);
  gf[n + i] = -(phi[i + g.sy] - phi[i - g.sy]) / (2.0 * g.dy);
  gf[2 * n + i] = -(phi[i + sz] - phi[i - sz]) / (2.0 * g.dz);
}

cudaError_t phase_calc_gforce(const Geom& g, const double* phi, double* gforce, cudaStream_t s) {
  k_calc_gforce<<<nblk(g.ng), PB, 0, s>>>(g, phi, gforce);
  return cudaGetLastError();
}

cudaError_t phase_source(const Geom& g, PhaseArrays& a, Ctrl* ctrl, double mult, cudaStream_t s) {
  k_phase_source<<<nblk(g.ng), PB, 0, s>>>(g, a, ctrl, mult);
  return cudaGetLastError();
}
cudaError_t phase_ghost(int nghost, const int32_t* dst, const int32_t* src, const uint8_t* sgn,
                        PhaseArrays& a, long long ng, cudaStream_t s) {
  if (nghost <= 0) return cudaSuccess;
  k_ghost_gather<<<nblk(nghost), PB, 0, s>>>(nghost, src, sgn, a.cons, ng, a.gtmp);
  k_ghost_scatter<<<nblk(nghost), PB, 0, s>>>(nghost, dst, a.gtmp, a.cons, ng);
  return cudaGetLastError();
}
cudaError_t phase_flux(const Geom& g, PhaseArrays& a, Ctrl* ctrl, int avg, cudaStream_t s) {
  if (g.ang) {
    k_ang_to<<<nblk(g.ng), PB, 0, s>>>(g, a, avg);
    k_phase_states<true><<<nblk(g.ng), PB, 0, s>>>(g, a, ctrl);
    k_phase_update<true><<<nblk(g.ng), PB, 0, s>>>(g, a, ctrl, avg);
  } else {
    k_phase_states<false><<<nblk(g.ng), PB, 0, s>>>(g, a, ctrl);
    k_phase_faces<<<nblk(g.ng), PB, 0, s>>>(g, a, a.states + 42 * g.ng);
    k_phase_update<false><<<nblk(g.ng), PB, 0, s>>>(g, a, ctrl, avg);
  }
  return cudaGetLastError();
}
cudaError_t phase_copy_old(const Geom& g, PhaseArrays& a, cudaStream_t s) {
  k_copy5<<<nblk(5 * g.ng), PB, 0, s>>>(a.cons, a.cons_old, g.ng);
  return cudaGetLastError();
}
cudaError_t fused_to_phase(const Geom& g, const double* X, int nsrc, PhaseArrays& a, int nghost,
                           const int32_t* dst, const int32_t* src2, const uint8_t* sgn2,
                           cudaStream_t s, long long xps) {
  k_f2p_interior<<<nblk(g.ng), PB, 0, s>>>(g, X, xps > 0 ? xps : g.ng, nsrc, a);
  if (nghost > 0)
    k_fill_resolved<<<nblk(nghost), PB, 0, s>>>(nghost, dst, src2, sgn2, a.cons, g.ng);
  k_f2p_prims<<<nblk(g.ng), PB, 0, s>>>(g, a);
  return cudaGetLastError();
}
__global__ void k_log10_rows(const double* eng2, long long neos, int nr, double* out) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r < nr) out[r] = log10(eng2[(long long)r * neos]);
}
cudaError_t eos_log_rows(const double* eng2, long long neos, int nr, double* out,
                         cudaStream_t s) {
  k_log10_rows<<<(nr + 127) / 128, 128, 0, s>>>(eng2, neos, nr, out);
  return cudaGetLastError();
}
__global__ void k_fill_const(double* a, long long n, double v) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i < n) a[i] = v;
}
cudaError_t p_after_force(const Geom& g, PhaseArrays& a, const double* uc, int nghost,
                          const int32_t* dst, const int32_t* src2, cudaStream_t s) {
  k_p_from_uc<<<nblk(g.ng), PB, 0, s>>>(g, a, uc);
  if (nghost > 0) k_p_ghosts<<<nblk(nghost), PB, 0, s>>>(nghost, dst, src2, a.p);
  return cudaGetLastError();
}
cudaError_t slab_in(const double* aos, double* X, long long ps, long long i0, long long i1,
                    cudaStream_t s) {
  if (i1 > i0) k_slab_in<<<nblk(i1 - i0), PB, 0, s>>>(aos, X, ps, i0, i1);
  return cudaGetLastError();
}
cudaError_t slab_out(const Geom& g, const double* X, long long ps, int nsrc, double* aos,
                     long long i0, long long i1, const int32_t* dst, const int32_t* src2,
                     const uint8_t* sgn2, int g0, int g1, cudaStream_t s) {
  if (i1 > i0) k_slab_out<<<nblk(i1 - i0), PB, 0, s>>>(g, X, ps, nsrc, aos, i0, i1);
  if (g1 > g0) k_slab_ghosts<<<nblk(g1 - g0), PB, 0, s>>>(dst, src2, sgn2, aos, g0, g1);
  return cudaGetLastError();
}
cudaError_t fill_const(double* a, long long n, double v, cudaStream_t s) {
  k_fill_const<<<nblk(n), PB, 0, s>>>(a, n, v);
  return cudaGetLastError();
}

// velocity and pressure arrays from the conserved variables alone
cudaError_t prims_from_cons(const Geom& g, PhaseArrays& a, cudaStream_t s) {
  k_f2p_prims<<<nblk(g.ng), PB, 0, s>>>(g, a);
  return cudaGetLastError();
}

// the reference cons only (no primitives) of the fused state X into cons
cudaError_t fused_to_cons(const Geom& g, const double* X, int nsrc, double* cons, int nghost,
                          const int32_t* dst, const int32_t* src2, const uint8_t* sgn2,
                          cudaStream_t s) {
  PhaseArrays a{};
  a.cons = cons;
  k_f2p_interior<<<nblk(g.ng), PB, 0, s>>>(g, X, g.ng, nsrc, a);
  if (nghost > 0) k_fill_resolved<<<nblk(nghost), PB, 0, s>>>(nghost, dst, src2, sgn2, cons, g.ng);
  return cudaGetLastError();
}
// does a box's plane set hold a state the fused stages start from
// (interior rho >= 1e-4 and finite, ghosts = two-sweep fill of the interior)?
__global__ void k_box_check_cells(Geom g, const double* X, long long ps, Ctrl* ctrl) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= g.ng) return;
  const int x = (int)(i % g.nx), y = (int)((i / g.nx) % g.ny), z = (int)(i / g.sz);
  if (is_ghost(g, x, y, z)) return;
  bool ok = X[i] >= kLowRho;
  for (int q = 0; q < 5; ++q) ok = ok && isfinite(X[q * ps + i]);
  if (!ok) atomicOr(&ctrl->flags, (unsigned)kFlagNotClean);
}
__global__ void k_box_check_ghosts(int nghost, const int32_t* dst, const int32_t* src,
                                   const uint8_t* sgn, const double* X, long long ps,
                                   Ctrl* ctrl) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= nghost) return;
  const long long s = src[k], d = dst[k];
  const unsigned m = sgn[k];
  bool ok = X[d] == X[s] && X[4 * ps + d] == X[4 * ps + s];
  ok = ok && X[ps + d] == ((m & 1) ? -X[ps + s] : X[ps + s]);
  ok = ok && X[2 * ps + d] == ((m & 2) ? -X[2 * ps + s] : X[2 * ps + s]);
  ok = ok && X[3 * ps + d] == ((m & 4) ? -X[3 * ps + s] : X[3 * ps + s]);
  if (!ok) atomicOr(&ctrl->flags, (unsigned)kFlagNotClean);
}
// Courant rate (courant.f90:19-23) of a box whose planes hold the reference
// cons with u == m/rho: the max over interior cells (ghosts repeat them)
__global__ void k_box_rate(Geom g, const double* X, long long ps, Ctrl* ctrl) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  double r = 0.0;
  if (i < g.ng) {
    const int x = (int)(i % g.nx), y = (int)((i / g.nx) % g.ny), z = (int)(i / g.sz);
    if (!is_ghost(g, x, y, z)) {
      const double d = X[i];
      const double u1 = X[ps + i] / d, u2 = X[2 * ps + i] / d, u3 = X[3 * ps + i] / d;
      const double p = eos_pressure(d, X[4 * ps + i], u1, u2, u3, g.gm1, g.small_eps);
      r = g.pow2 ? courant_rate<true>(d, p, g.gam, u1, u2, u3, g.dx, g.dy, g.dz, g.idx, g.idy, g.idz)
                 : courant_rate<false>(d, p, g.gam, u1, u2, u3, g.dx, g.dy, g.dz, g.idx, g.idy, g.idz);
    }
  }
  __shared__ double wm[PB / 32];
  r = warp_max(r);
  if ((threadIdx.x & 31) == 0) wm[threadIdx.x >> 5] = r;
  __syncthreads();
  if (threadIdx.x == 0) {
    double m = 0.0;
    for (int k = 0; k < PB / 32; ++k) m = fmax(m, wm[k]);
    atomicMax(&ctrl->rate_bits, (unsigned long long)__double_as_longlong(m));
  }
}

cudaError_t box_check_clean(const Geom& g, const double* X, long long ps, int nghost,
                            const int32_t* dst, const int32_t* src2, const uint8_t* sgn2,
                            Ctrl* ctrl, cudaStream_t s) {
  k_box_check_cells<<<nblk(g.ng), PB, 0, s>>>(g, X, ps, ctrl);
  if (nghost > 0)
    k_box_check_ghosts<<<nblk(nghost), PB, 0, s>>>(nghost, dst, src2, sgn2, X, ps, ctrl);
  return cudaGetLastError();
}
// the same over the interior cells of [i0, i1), into *bits
__global__ void k_slab_rate(Geom g, const double* X, long long ps, long long i0, long long i1,
                            unsigned long long* bits) {
  const long long i = i0 + blockIdx.x * (long long)blockDim.x + threadIdx.x;
  double r = 0.0;
  if (i < i1) {
    const int x = (int)(i % g.nx), y = (int)((i / g.nx) % g.ny), z = (int)(i / g.sz);
    if (!is_ghost(g, x, y, z)) {
      const double d = X[i];
      const double u1 = X[ps + i] / d, u2 = X[2 * ps + i] / d, u3 = X[3 * ps + i] / d;
      const double p = eos_pressure(d, X[4 * ps + i], u1, u2, u3, g.gm1, g.small_eps);
      r = g.pow2 ? courant_rate<true>(d, p, g.gam, u1, u2, u3, g.dx, g.dy, g.dz, g.idx, g.idy, g.idz)
                 : courant_rate<false>(d, p, g.gam, u1, u2, u3, g.dx, g.dy, g.dz, g.idx, g.idy, g.idz);
    }
  }
  __shared__ double wm[PB / 32];
  r = warp_max(r);
  if ((threadIdx.x & 31) == 0) wm[threadIdx.x >> 5] = r;
  __syncthreads();
  if (threadIdx.x == 0) {
    double m = 0.0;
    for (int k = 0; k < PB / 32; ++k) m = fmax(m, wm[k]);
    atomicMax(bits, (unsigned long long)__double_as_longlong(m));
  }
}
cudaError_t slab_rate(const Geom& g, const double* X, long long ps, long long i0, long long i1,
                      unsigned long long* bits, cudaStream_t s) {
  if (i1 > i0) k_slab_rate<<<nblk(i1 - i0), PB, 0, s>>>(g, X, ps, i0, i1, bits);
  return cudaGetLastError();
}
cudaError_t box_rate(const Geom& g, const double* X, long long ps, Ctrl* ctrl, cudaStream_t s) {
  k_box_rate<<<nblk(g.ng), PB, 0, s>>>(g, X, ps, ctrl);
  return cudaGetLastError();
}

cudaError_t check_clean(const Geom& g, const PhaseArrays& a, int nghost, const int32_t* dst,
                        const int32_t* src2, const uint8_t* sgn2, Ctrl* ctrl, cudaStream_t s) {
  k_check_cells<<<nblk(g.ng), PB, 0, s>>>(g, a, ctrl);
  if (nghost > 0) k_check_ghosts<<<nblk(nghost), PB, 0, s>>>(nghost, dst, src2, sgn2, a.cons, g.ng, ctrl);
  return cudaGetLastError();
}
cudaError_t aos_to_soa(const double* aos, double* soa, long long n, int k, cudaStream_t s) {
  k_aos_to_soa<<<nblk(n), PB, 0, s>>>(aos, soa, n, k);
  return cudaGetLastError();
}
cudaError_t soa_to_aos(const double* soa, double* aos, long long n, int k, cudaStream_t s) {
  k_soa_to_aos<<<nblk(n), PB, 0, s>>>(soa, aos, n, k);
  return cudaGetLastError();
}

}  // namespace bx

namespace bx {
int stage_blocks_per_sm(int stage, int pm, bool threed, int shape) {
  int nb = 0;
  const size_t smem = stage_smem_bytes(shape);
  const void* fn;
  if (shape == 3) {
    if (stage == 0)
      fn = pm == 1 ? (threed ? (const void*)k_stage<0, 1, true, false, 3>
                             : (const void*)k_stage<0, 1, false, false, 3>)
                   : (threed ? (const void*)k_stage<0, 0, true, false, 3>
                             : (const void*)k_stage<0, 0, false, false, 3>);
    else
      fn = pm == 1 ? (threed ? (const void*)k_stage<1, 1, true, false, 3>
                             : (const void*)k_stage<1, 1, false, false, 3>)
                   : (threed ? (const void*)k_stage<1, 0, true, false, 3>
                             : (const void*)k_stage<1, 0, false, false, 3>);
  } else if (shape == 2) {
    if (stage == 0)
      fn = pm == 1 ? (threed ? (const void*)k_stage<0, 1, true, false, 2>
                             : (const void*)k_stage<0, 1, false, false, 2>)
                   : (threed ? (const void*)k_stage<0, 0, true, false, 2>
                             : (const void*)k_stage<0, 0, false, false, 2>);
    else
      fn = pm == 1 ? (threed ? (const void*)k_stage<1, 1, true, false, 2>
                             : (const void*)k_stage<1, 1, false, false, 2>)
                   : (threed ? (const void*)k_stage<1, 0, true, false, 2>
                             : (const void*)k_stage<1, 0, false, false, 2>);
  } else if (shape == 1) {
    if (stage == 0)
      fn = pm == 1 ? (threed ? (const void*)k_stage<0, 1, true, false, 1>
                             : (const void*)k_stage<0, 1, false, false, 1>)
                   : (threed ? (const void*)k_stage<0, 0, true, false, 1>
                             : (const void*)k_stage<0, 0, false, false, 1>);
    else
      fn = pm == 1 ? (threed ? (const void*)k_stage<1, 1, true, false, 1>
                             : (const void*)k_stage<1, 1, false, false, 1>)
                   : (threed ? (const void*)k_stage<1, 0, true, false, 1>
                             : (const void*)k_stage<1, 0, false, false, 1>);
  } else {
    if (stage == 0)
      fn = pm == 1 ? (threed ? (const void*)k_stage<0, 1, true> : (const void*)k_stage<0, 1, false>)
                   : (threed ? (const void*)k_stage<0, 0, true> : (const void*)k_stage<0, 0, false>);
    else
      fn = pm == 1 ? (threed ? (const void*)k_stage<1, 1, true> : (const void*)k_stage<1, 1, false>)
                   : (threed ? (const void*)k_stage<1, 0, true> : (const void*)k_stage<1, 0, false>);
  }
  if (ensure_dyn_smem(fn, smem) != cudaSuccess ||
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, fn, NT, smem) != cudaSuccess) {
    cudaGetLastError();
    return 1;
  }
  return nb;
}
}  // namespace bx

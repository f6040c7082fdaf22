// bx_math.cuh -- per-cell and per-face arithmetic of the hydro step, FP64.
//
// Every formula is written in the evaluation order of the reference Fortran
// (left-to-right association, x**2 as x*x).  The library is compiled with
// -fmad=false so no multiply-add is contracted, and uses IEEE division and
// square root, which makes each result bit-identical to gfortran -O3 on x86-64
// (SSE2, no FMA) for the same inputs -- up to the sign of zero and NaN payloads.
#pragma once
#include <cstdint>

#define BX_HD __host__ __device__ __forceinline__

namespace bx {

constexpr double kHalf = 0.5;      // half = one/two, parameters.f90:143
constexpr double kTheta = 1.25;    // SLOPE_THETA, Makefile:20 / utils.f90:739
constexpr double kLowRho = 1e-4;   // low-density EOS branch, state.f90:52

// Primitive set used by reconstruction: rho, u1..3, p, eps (internal energy
// per volume), plus the sound speed c = sqrt(p*gamma/rho) of the cell and, with
// the tabulated EOS, the cell's gamma (adindx), with angular-momentum fluxing
// the radial and angular momenta (rm, am), reconstructed like the others.
struct Prim {
  double d, u1, u2, u3, p, e, c, g, rm, am;
};

// Reconstructed face state (one side of one face); g: gamma, with the
// tabulated EOS only (fixed gamma: the grid's); rm, am: with flux_ang only.
struct FaceState {
  double d, u1, u2, u3, p, e, g, rm, am;
};

// genminmod (utils.f90:696-707) of (theta*d1, half*d2, theta*d3) where
// d1=c1-c0, d2=c2-c0, d3=c2-c1 (slope, utils.f90:738-741).  When d1 and d3
// share a strict sign, d2 has it too (c2-c0 is a rounded nonzero difference
// of the same sign), so the branch test needs d1 and d3 only; the minimum of
// magnitudes equals min(x1,x2,x3) (all positive) or -max(x1,x2,x3) (all
// negative) exactly.
BX_HD double slope3(double c0, double c1, double c2) {
  const double d1 = c1 - c0, d2 = c2 - c0, d3 = c2 - c1;
  const double x1 = kTheta * d1, x2 = kHalf * d2, x3 = kTheta * d3;
#ifdef __CUDA_ARCH__
  // The argument of least magnitude, with its own sign, by two compares of
  // magnitudes (a NaN compares false; the guards flag it).  When d1 and d3
  // share a strict sign (their sign bits agree and neither is zero, so m is
  // not zero), all three arguments carry it and the result is m; anything else
  // gives the reference's +0.  Ties of magnitude pick arguments of equal value.
  const double t = fabs(x1) < fabs(x2) ? x1 : x2;
  const double m = fabs(t) < fabs(x3) ? t : x3;
  const int h1 = __double2hiint(d1), h3 = __double2hiint(d3);
  const bool take = ((h1 ^ h3) >= 0) && (m != 0.0);
  return take ? m : 0.0;
#else
  const double m = fmin(fabs(x1), fmin(fabs(x2), fabs(x3)));
  const bool pos = (d1 > 0.0) && (d3 > 0.0);
  const bool neg = (d1 < 0.0) && (d3 < 0.0);
  return pos ? m : (neg ? -m : 0.0);
#endif
}

// K = rho*half*(u1^2+u2^2+u3^2) (state.f90:32,47) and the same value written
// half*rho*(...) in flux.f90:282-286,342 (multiplication commutes exactly).
BX_HD double kin_rho_u(double d, double u1, double u2, double u3) {
  return d * kHalf * (u1 * u1 + u2 * u2 + u3 * u3);
}

// half*(m1^2+m2^2+m3^2)/rho (velocity.f90:37, source.f90:176, flux.f90:227)
BX_HD double kin_mom(double d, double m1, double m2, double m3) {
  return kHalf * (m1 * m1 + m2 * m2 + m3 * m3) / d;
}

// source() energy update with zero gravitational force (source.f90:161-182):
// momenta gain (rho*0)*dt = 0 and E = max(E - K + 0, small_eps) + K.
BX_HD double source_energy(double d, double m1, double m2, double m3, double E,
                           double small_eps) {
  const double ek = kin_mom(d, m1, m2, m3);
  return fmax(E - ek, small_eps) + ek;
}

// source() with a gravitational acceleration g (source.f90:161-182); u is the
// velocity array the reference holds at that moment.
BX_HD void source_gravity(double& d, double& m1, double& m2, double& m3, double& E,
                          double g1, double g2, double g3, double u1, double u2, double u3,
                          double dt, double small_eps) {
  m2 = m2 + (d * (g2)) * dt;
  m1 = m1 + (d * (g1)) * dt;
  m3 = m3 + ((g3) * d) * dt;
  const double ek = kin_mom(d, m1, m2, m3);
  E = fmax(E - ek + dt * d * (((u1) * (g1) + (u2) * (g2) + (u3) * (g3))), small_eps) + ek;
}

// fixed-gamma pressure for rho >= 1e-4 (state.f90:47-48,58)
BX_HD double eos_pressure(double d, double E, double u1, double u2, double u3, double gm1,
                          double small_eps) {
  const double ek = kin_rho_u(d, u1, u2, u3);
  return fmax(E - ek, small_eps) * gm1;
}

// internal energy per volume used by reconstruction (flux.f90:282-286,342)
BX_HD double recon_eps(double d, double E, double u1, double u2, double u3, double small_eps) {
  return fmax(E - kHalf * d * (u1 * u1 + u2 * u2 + u3 * u3), small_eps);
}

// x/d for a grid constant d (a cell size or the cell volume) given its
// correctly rounded reciprocal r, computed on the host.  With q0 = RN(x*r) the
// residual x - d*q0 is exact under a fused multiply-add and RN(q0 + (x-d*q0)*r)
// is the IEEE quotient (Markstein's theorem) while |x| and d lie in
// [2^-450, 2^450] (bx_create keeps d there); zero gives x*r, a signed zero like
// x/d; other x take the IEEE division.
BX_HD double cdiv(double x, double d, double r) {
#ifdef __CUDA_ARCH__
  const double ax = fabs(x);
  if (ax >= 0x1p-450 && ax <= 0x1p+450) {
    const double q0 = x * r;
    return fma(fma(-d, q0, x), r, q0);
  }
  if (ax == 0.0) return x * r;
#endif
  return x / d;
}

// Courant rate of one cell (courant.f90:20-21); idx etc. are 1/dx etc.: when
// the spacing is a power of two x/2^k and x*2^-k round identically, otherwise
// cdiv gives the IEEE quotient.
template <bool POW2>
BX_HD double courant_rate(double d, double p, double gam, double u1, double u2, double u3,
                          double dx, double dy, double dz, double idx, double idy,
                          double idz) {
  const double sound = sqrt(gam * p / d);
  if (POW2)
    return (sound + fabs(u1)) * idx + (sound + fabs(u2)) * idy + (sound + fabs(u3)) * idz;
  return cdiv(sound + fabs(u1), dx, idx) + cdiv(sound + fabs(u2), dy, idy) +
         cdiv(sound + fabs(u3), dz, idz);
}

#ifdef __CUDACC__
// courant_rate with the division by rho through a SharedDiv of rho
template <bool POW2>
__device__ __forceinline__ double courant_rate_q(const struct SharedDiv& qd, double p, double gam,
                                                 double u1, double u2, double u3, double dx,
                                                 double dy, double dz, double idx, double idy,
                                                 double idz);
#endif

// calculate_states for one cell and one direction (flux.f90:327-351):
// lambda_p = max(u_d+c,0)*dt/ds, lambda_m = min(u_d-c,0)*dt/ds,
// q- = q + half*(-1-lambda_m)*s, q+ = q + half*(1-lambda_p)*s.
// The transverse terms of flux.f90:391-479 add zero and are omitted.
template <bool POW2, bool TAB = false, bool ANG = false>
BX_HD void muscl_states(const Prim& q, double ud, double sd, double su1, double su2,
                        double su3, double sp, double se, double dt, double ds, double ids,
                        FaceState& mi, FaceState& pl, double sg = 0.0, double srm = 0.0,
                        double sam = 0.0) {
  double lp = fmax(ud + q.c, 0.0) * dt;
  double lm = fmin(ud - q.c, 0.0) * dt;
  if (POW2) {
    lp = lp * ids;
    lm = lm * ids;
  } else {
    lp = cdiv(lp, ds, ids);
    lm = cdiv(lm, ds, ids);
  }
  const double hm = kHalf * (-1.0 - lm);
  const double hp = kHalf * (1.0 - lp);
  mi.u1 = q.u1 + hm * su1;
  pl.u1 = q.u1 + hp * su1;
  mi.u2 = q.u2 + hm * su2;
  pl.u2 = q.u2 + hp * su2;
  mi.u3 = q.u3 + hm * su3;
  pl.u3 = q.u3 + hp * su3;
  mi.p = q.p + hm * sp;
  pl.p = q.p + hp * sp;
  mi.d = q.d + hm * sd;
  pl.d = q.d + hp * sd;
  mi.e = q.e + hm * se;
  pl.e = q.e + hp * se;
  if (TAB) {
    mi.g = q.g + hm * sg;
    pl.g = q.g + hp * sg;
  }
  if (ANG) {
    // flux_ang.f90:349-518: the transformed momenta, without transverse terms
    mi.rm = q.rm + hm * srm;
    pl.rm = q.rm + hp * srm;
    mi.am = q.am + hm * sam;
    pl.am = q.am + hp * sam;
  }
}

// Face state of a ghost cell: its slopes are zero (flux.f90:53-54), so both
// sides equal the cell values.
BX_HD void ghost_states(const Prim& q, FaceState& mi, FaceState& pl) {
  mi.d = q.d; mi.u1 = q.u1; mi.u2 = q.u2; mi.u3 = q.u3; mi.p = q.p; mi.e = q.e; mi.g = q.g;
  mi.rm = q.rm; mi.am = q.am;
  pl = mi;
}

// The shared-denominator quotient below is exact for a numerator a when a = +-0
// or |a| lies in [2^-450, 2^451) (NaN and infinities fail): three compares,
// which the compiler chains on one predicate.
__device__ __forceinline__ bool quot_fast_ok(double a) {
  const double m = fabs(a);
  return (m >= 0x1p-450 && m < 0x1p+451) || a == 0.0;
}

// q = a/d for five numerators over one denominator d, given r = RN(1/d) with d
// in [2^-450, 2^450] and every a passing quot_fast_ok: q0 = RN(a r) and the
// residual e = RN(a - d q0), exact under a fused multiply-add, give the
// correctly rounded quotient RN(q0 + e r) (Markstein's theorem).  The residual
// is formed as -RN(d q0 - a), the same value for every nonzero a, so that a = -0
// yields -0 like a/d (q0 = -0 and e = -0).
__device__ __forceinline__ double quot_fast(double a, double d, double r) {
  const double q0 = a * r;
  const double e = -fma(d, q0, -a);
  return fma(e, r, q0);
}

// IEEE a/d out of line: the fallback of the shortened divisions below, taken
// only outside their exponent window, so its code is not repeated at every
// division of the stage kernels
static __device__ __noinline__ double div_ieee(double a, double d) { return a / d; }

// a/d for several numerators sharing one denominator d > 0.  With r the
// correctly rounded reciprocal of d, q0 = RN(a*r) is within one ulp of a/d and
// the residual a - d*q0 is exact under a fused multiply-add, so
// RN(q0 + (a - d*q0)*r) is the correctly rounded quotient (Markstein's
// theorem, as used for IEEE division on FMA hardware).  The theorem needs the
// quotient and the residual away from the overflow and subnormal ranges:
// with d and |a| in [2^-450, 2^450] the quotient lies in [2^-900, 2^900] and
// the residual (about |a|*2^-53) stays normal.  quot_fast computes it (signed
// zeros included) wherever quot_fast_ok admits a; outside that window the IEEE
// division is taken instead.
struct SharedDiv {
  double d, r;
  bool ok;
  __device__ __forceinline__ explicit SharedDiv(double den) : d(den) {
    ok = den >= 0x1p-450 && den <= 0x1p+450;
    r = ok ? __drcp_rn(den) : 0.0;
  }
  __device__ __forceinline__ double operator()(double a) const {
    if (ok && quot_fast_ok(a)) return quot_fast(a, d, r);
    return div_ieee(a, d);
  }
};

template <bool POW2>
__device__ __forceinline__ double courant_rate_q(const SharedDiv& qd, double p, double gam,
                                                 double u1, double u2, double u3, double dx,
                                                 double dy, double dz, double idx, double idy,
                                                 double idz) {
  const double sound = sqrt(qd(gam * p));
  if (POW2)
    return (sound + fabs(u1)) * idx + (sound + fabs(u2)) * idy + (sound + fabs(u3)) * idz;
  return cdiv(sound + fabs(u1), dx, idx) + cdiv(sound + fabs(u2), dy, idy) +
         cdiv(sound + fabs(u3), dz, idz);
}

// half*(m1^2+m2^2+m3^2)/rho and the zero-force source() energy update with the
// division by rho through a SharedDiv of rho
__device__ __forceinline__ double kin_mom_q(const SharedDiv& qd, double m1, double m2,
                                            double m3) {
  return qd(kHalf * (m1 * m1 + m2 * m2 + m3 * m3));
}
__device__ __forceinline__ double source_energy_q(const SharedDiv& qd, double m1, double m2,
                                                  double m3, double E, double small_eps) {
  const double ek = kin_mom_q(qd, m1, m2, m3);
  return fmax(E - ek, small_eps) + ek;
}

// HLL flux through one face normal to axis DIR (0,1,2) from the plus state of
// the cell on the low side (L) and the minus state of the cell on the high side
// (R): get_fluxes + flux_hll, flux.f90:504-590.  gl=gr=gamma.
// Returns a nonzero code when ap+am == 0 (the reference divides by zero).
template <int DIR, bool TAB = false>
BX_HD void hll_flux(const FaceState& L, const FaceState& R, double gam, double F[5]) {
  // The wave speeds come first, then each component from its own state and
  // flux terms, so only the two face states and the speeds stay live across
  // the components (every expression is the reference's, in its order).
  const double vl = DIR == 0 ? L.u1 : (DIR == 1 ? L.u2 : L.u3);
  const double vr = DIR == 0 ? R.u1 : (DIR == 1 ? R.u2 : R.u3);
  // gl, gr: the reconstructed gammas with the tabulated EOS (flux.f90:507,521)
  const double cr = sqrt((TAB ? R.g : gam) * R.p / R.d);
  const double cl = sqrt((TAB ? L.g : gam) * L.p / L.d);
  const double ap = fmax(fmax(0.0, vr + cr), vl + cl);
  const double am = fmax(fmax(0.0, -(vr - cr)), -(vl - cl));
  const double apam = ap * am;
  const double den = ap + am;
  // the numerators first; they all share the denominator ap+am
#define BX_HLL_Q(x) (x)
  // component 0: the mass flux
  {
    const double sl = L.d, sr = R.d;
    const double fl = sl * vl, fr = sr * vr;
    F[0] = BX_HLL_Q(ap * fl + am * fr - apam * (sr - sl));
  }
  // components 1-3: momenta, with the pressure on the normal component
  {
    const double sl = L.d * L.u1, sr = R.d * R.u1;
    const double fl = DIR == 0 ? L.p + sl * vl : sl * vl;
    const double fr = DIR == 0 ? R.p + sr * vr : sr * vr;
    F[1] = BX_HLL_Q(ap * fl + am * fr - apam * (sr - sl));
  }
  {
    const double sl = L.d * L.u2, sr = R.d * R.u2;
    const double fl = DIR == 1 ? L.p + sl * vl : sl * vl;
    const double fr = DIR == 1 ? R.p + sr * vr : sr * vr;
    F[2] = BX_HLL_Q(ap * fl + am * fr - apam * (sr - sl));
  }
  {
    const double sl = L.d * L.u3, sr = R.d * R.u3;
    const double fl = DIR == 2 ? L.p + sl * vl : sl * vl;
    const double fr = DIR == 2 ? R.p + sr * vr : sr * vr;
    F[3] = BX_HLL_Q(ap * fl + am * fr - apam * (sr - sl));
  }
  // component 4: the energy, states(5) = eps + half*rho*|u|^2
  {
    const double sl = L.e + kHalf * L.d * (L.u1 * L.u1 + L.u2 * L.u2 + L.u3 * L.u3);
    const double sr = R.e + kHalf * R.d * (R.u1 * R.u1 + R.u2 * R.u2 + R.u3 * R.u3);
    const double fl = (sl + L.p) * vl, fr = (sr + R.p) * vr;
    F[4] = BX_HLL_Q(ap * fl + am * fr - apam * (sr - sl));
  }
#undef BX_HLL_Q
#ifdef __CUDA_ARCH__
  const bool fast = den >= 0x1p-450 && den <= 0x1p+450 && quot_fast_ok(F[0]) &&
                    quot_fast_ok(F[1]) && quot_fast_ok(F[2]) && quot_fast_ok(F[3]) &&
                    quot_fast_ok(F[4]);
  if (fast) {
    const double r = __drcp_rn(den);
#pragma unroll
    for (int i = 0; i < 5; ++i) F[i] = quot_fast(F[i], den, r);
  } else {
    for (int i = 0; i < 5; ++i) F[i] = div_ieee(F[i], den);
  }
#else
  for (int i = 0; i < 5; ++i) F[i] = F[i] / den;
#endif
}

// HLL flux with angular-momentum fluxing (flux_ang.f90:523-618, gl = gr =
// gamma): components 1 and 2 are the radial and angular momenta, whose x and y
// face fluxes carry pressure terms at the centre of the cell being updated
// (x, y without yoffset, r = sqrt(x^2 + y^2), flux_ang.f90:571-573).  For
// DIR 0 and 1, F[1], F[2] are those of the high cell (xh, yh, rh: the face is
// its minus face) and F[5], F[6] of the low cell (xl, yl, rl); z faces have no
// such terms (F[5], F[6] unset).
template <int DIR>
__device__ __forceinline__ void hll_flux_ang(const FaceState& L, const FaceState& R, double gam,
                                             double xl, double yl, double rl, double xh,
                                             double yh, double rh, double F[7]) {
  const double vl = DIR == 0 ? L.u1 : (DIR == 1 ? L.u2 : L.u3);
  const double vr = DIR == 0 ? R.u1 : (DIR == 1 ? R.u2 : R.u3);
  const double cr = sqrt(gam * R.p / R.d);
  const double cl = sqrt(gam * L.p / L.d);
  const double ap = fmax(fmax(0.0, vr + cr), vl + cl);
  const double am = fmax(fmax(0.0, -(vr - cr)), -(vl - cl));
  const double apam = ap * am;
  const double den = ap + am;
  auto num = [&](double sl, double sr, double fl, double fr) {
    return ap * fl + am * fr - apam * (sr - sl);
  };
  // mass
  F[0] = num(L.d, R.d, L.d * vl, R.d * vr);
  // momentum 3: the pressure on the z faces only
  {
    const double sl = L.d * L.u3, sr = R.d * R.u3;
    F[3] = num(sl, sr, (DIR == 2 ? L.p : 0.0) + sl * vl, (DIR == 2 ? R.p : 0.0) + sr * vr);
  }
  // energy
  {
    const double sl = L.e + kHalf * L.d * (L.u1 * L.u1 + L.u2 * L.u2 + L.u3 * L.u3);
    const double sr = R.e + kHalf * R.d * (R.u1 * R.u1 + R.u2 * R.u2 + R.u3 * R.u3);
    F[4] = num(sl, sr, (sl + L.p) * vl, (sr + R.p) * vr);
  }
  // radial and angular momenta, with the pressure terms of the updated cell
  auto mom = [&](double x, double y, double r, double& f1, double& f2) {
    double al = 0.0, ar = 0.0, bl = 0.0, br = 0.0;
    if (DIR == 0) {
      al = L.p * x / r; ar = R.p * x / r;
      bl = -(L.p * y); br = -(R.p * y);
    } else if (DIR == 1) {
      al = L.p * y / r; ar = R.p * y / r;
      bl = L.p * x; br = R.p * x;
    }
    f1 = num(L.rm, R.rm, al + L.rm * vl, ar + R.rm * vr);
    f2 = num(L.am, R.am, bl + L.am * vl, br + R.am * vr);
  };
  mom(xh, yh, rh, F[1], F[2]);
  constexpr int NQ = DIR == 2 ? 5 : 7;
  if (DIR != 2) mom(xl, yl, rl, F[5], F[6]);
  bool fast = den >= 0x1p-450 && den <= 0x1p+450;
#pragma unroll
  for (int i = 0; i < NQ; ++i) fast = fast && quot_fast_ok(F[i]);
  if (fast) {
    const double r = __drcp_rn(den);
#pragma unroll
    for (int i = 0; i < NQ; ++i) F[i] = quot_fast(F[i], den, r);
  } else {
    for (int i = 0; i < NQ; ++i) F[i] = div_ieee(F[i], den);
  }
}

// floors after the conservative update (flux.f90:223-230)
BX_HD void floors(double& d, double m1, double m2, double m3, double& E, double small_rho,
                  double small_eps) {
  d = fmax(d, small_rho);
  if (E < 0.0) E = kin_mom(d, m1, m2, m3) + small_eps;
}

}  // namespace bx

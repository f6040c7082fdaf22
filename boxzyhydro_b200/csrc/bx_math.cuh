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
// per volume), plus the sound speed c = sqrt(p*gamma/rho) of the cell.
struct Prim {
  double d, u1, u2, u3, p, e, c;
};

// Reconstructed face state (one side of one face); gamma is constant.
struct FaceState {
  double d, u1, u2, u3, p, e;
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
  const double m = fmin(fabs(x1), fmin(fabs(x2), fabs(x3)));
  const bool pos = (d1 > 0.0) && (d3 > 0.0);
  const bool neg = (d1 < 0.0) && (d3 < 0.0);
  return pos ? m : (neg ? -m : 0.0);
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

// calculate_states for one cell and one direction (flux.f90:327-351):
// lambda_p = max(u_d+c,0)*dt/ds, lambda_m = min(u_d-c,0)*dt/ds,
// q- = q + half*(-1-lambda_m)*s, q+ = q + half*(1-lambda_p)*s.
// The transverse terms of flux.f90:391-479 add zero and are omitted.
template <bool POW2>
BX_HD void muscl_states(const Prim& q, double ud, double sd, double su1, double su2,
                        double su3, double sp, double se, double dt, double ds, double ids,
                        FaceState& mi, FaceState& pl) {
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
}

// Face state of a ghost cell: its slopes are zero (flux.f90:53-54), so both
// sides equal the cell values.
BX_HD void ghost_states(const Prim& q, FaceState& mi, FaceState& pl) {
  mi.d = q.d; mi.u1 = q.u1; mi.u2 = q.u2; mi.u3 = q.u3; mi.p = q.p; mi.e = q.e;
  pl = mi;
}

// a/d for several numerators sharing one denominator d > 0.  With r the
// correctly rounded reciprocal of d, q0 = RN(a*r) is within one ulp of a/d and
// the residual a - d*q0 is exact under a fused multiply-add, so
// RN(q0 + (a - d*q0)*r) is the correctly rounded quotient (Markstein's
// theorem, as used for IEEE division on FMA hardware).  The theorem needs the
// quotient and the residual away from the overflow and subnormal ranges:
// with d and |a| in [2^-450, 2^450] the quotient lies in [2^-900, 2^900] and
// the residual (about |a|*2^-53) stays normal.  Outside that window (and for
// a = 0) the IEEE division is taken instead.
struct SharedDiv {
  double d, r;
  bool ok;
  __device__ __forceinline__ explicit SharedDiv(double den) : d(den) {
    ok = den >= 0x1p-450 && den <= 0x1p+450;
    r = ok ? __drcp_rn(den) : 0.0;
  }
  __device__ __forceinline__ double operator()(double a) const {
    const double aa = fabs(a);
    if (ok && aa >= 0x1p-450 && aa <= 0x1p+450) {
      const double q0 = a * r;
      const double e = fma(-d, q0, a);
      return fma(e, r, q0);
    }
    if (ok && aa == 0.0) return a * r;  // signed zero, as a/d
    return a / d;
  }
};

// HLL flux through one face normal to axis DIR (0,1,2) from the plus state of
// the cell on the low side (L) and the minus state of the cell on the high side
// (R): get_fluxes + flux_hll, flux.f90:504-590.  gl=gr=gamma.
// Returns a nonzero code when ap+am == 0 (the reference divides by zero).
template <int DIR>
BX_HD void hll_flux(const FaceState& L, const FaceState& R, double gam, double F[5]) {
  const double dl = L.d, pl = L.p, el = L.e, vxl = L.u1, vyl = L.u2, vzl = L.u3;
  const double dr = R.d, pr = R.p, er = R.e, vxr = R.u1, vyr = R.u2, vzr = R.u3;
  double sl[5], sr[5], fl[5], fr[5];
  sl[0] = dl;
  sl[1] = dl * vxl;
  sl[2] = dl * vyl;
  sl[3] = dl * vzl;
  sl[4] = el + kHalf * dl * (vxl * vxl + vyl * vyl + vzl * vzl);
  sr[0] = dr;
  sr[1] = dr * vxr;
  sr[2] = dr * vyr;
  sr[3] = dr * vzr;
  sr[4] = er + kHalf * dr * (vxr * vxr + vyr * vyr + vzr * vzr);
  const double vl = DIR == 0 ? vxl : (DIR == 1 ? vyl : vzl);
  const double vr = DIR == 0 ? vxr : (DIR == 1 ? vyr : vzr);
  fl[0] = sl[0] * vl;
  fr[0] = sr[0] * vr;
  // fluxes_l(2..4) = (p on the normal component, 0 elsewhere) + states*v
  fl[1] = DIR == 0 ? pl + sl[1] * vl : sl[1] * vl;
  fl[2] = DIR == 1 ? pl + sl[2] * vl : sl[2] * vl;
  fl[3] = DIR == 2 ? pl + sl[3] * vl : sl[3] * vl;
  fr[1] = DIR == 0 ? pr + sr[1] * vr : sr[1] * vr;
  fr[2] = DIR == 1 ? pr + sr[2] * vr : sr[2] * vr;
  fr[3] = DIR == 2 ? pr + sr[3] * vr : sr[3] * vr;
  fl[4] = (sl[4] + pl) * vl;
  fr[4] = (sr[4] + pr) * vr;
  const double cr = sqrt(gam * pr / dr);
  const double cl = sqrt(gam * pl / dl);
  const double ap = fmax(fmax(0.0, vr + cr), vl + cl);
  const double am = fmax(fmax(0.0, -(vr - cr)), -(vl - cl));
  const double apam = ap * am;
  const double den = ap + am;
#ifdef __CUDA_ARCH__
  const SharedDiv div(den);
#pragma unroll
  for (int i = 0; i < 5; ++i) F[i] = div(ap * fl[i] + am * fr[i] - apam * (sr[i] - sl[i]));
#else
  for (int i = 0; i < 5; ++i) F[i] = (ap * fl[i] + am * fr[i] - apam * (sr[i] - sl[i])) / den;
#endif
}

// floors after the conservative update (flux.f90:223-230)
BX_HD void floors(double& d, double m1, double m2, double m3, double& E, double small_rho,
                  double small_eps) {
  d = fmax(d, small_rho);
  if (E < 0.0) E = kin_mom(d, m1, m2, m3) + small_eps;
}

}  // namespace bx

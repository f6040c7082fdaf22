// bx_adjoint_math.cuh -- vector-Jacobian products of the per-face and per-cell
// arithmetic of the fused hydro step (bx_math.cuh), with every max/min/branch
// frozen at the choice the forward values make.  Derivatives need not round
// like the forward; they are written for clarity.
#pragma once
#include "bx_math.cuh"

namespace bx {

struct FS6 {  // a face state or its adjoint: rho, u1, u2, u3, p, eps
  double d, u1, u2, u3, p, e;
};

__device__ __forceinline__ FS6 fs_zero() { return FS6{0, 0, 0, 0, 0, 0}; }

// 1/x for the derivative terms (which need not round like the forward): the
// hardware's approximate reciprocal refined by two Newton steps,
// y <- y + y (1 - x y), each squaring the relative error; within a few ulps,
// with no branch.  Not for values the forward's branches depend on.
__device__ __forceinline__ double rcp_deriv(double x) {
  double y;
  asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(x));
  y = fma(y, fma(-x, y, 1.0), y);
  y = fma(y, fma(-x, y, 1.0), y);
  return y;
}

// --- HLL flux (flux.f90:504-590): adjoints of the two face states from gF.
template <int DIR>
__device__ __forceinline__ void hll_vjp(const FaceState& L, const FaceState& R, double gam,
                                        const double gF[5], FS6& gL, FS6& gR) {
  const double dl = L.d, pl = L.p, el = L.e;
  const double dr = R.d, pr = R.p, er = R.e;
  const double ul[3] = {L.u1, L.u2, L.u3}, ur[3] = {R.u1, R.u2, R.u3};
  const double vl = ul[DIR], vr = ur[DIR];
  const double Kl = ul[0] * ul[0] + ul[1] * ul[1] + ul[2] * ul[2];
  const double Kr = ur[0] * ur[0] + ur[1] * ur[1] + ur[2] * ur[2];
  double sl[5], sr[5], fl[5], fr[5];
  sl[0] = dl; sr[0] = dr;
  for (int j = 0; j < 3; ++j) { sl[1 + j] = dl * ul[j]; sr[1 + j] = dr * ur[j]; }
  sl[4] = el + kHalf * dl * Kl;
  sr[4] = er + kHalf * dr * Kr;
  fl[0] = sl[0] * vl; fr[0] = sr[0] * vr;
  for (int j = 0; j < 3; ++j) {
    fl[1 + j] = (j == DIR ? pl : 0.0) + sl[1 + j] * vl;
    fr[1 + j] = (j == DIR ? pr : 0.0) + sr[1 + j] * vr;
  }
  fl[4] = (sl[4] + pl) * vl;
  fr[4] = (sr[4] + pr) * vr;
  const double cr = sqrt(gam * pr / dr), cl = sqrt(gam * pl / dl);
  // ap = max(0, vr+cr, vl+cl), am = max(0, -(vr-cr), -(vl-cl)), evaluated as the forward
  const double a1 = vr + cr, a2 = vl + cl;
  const double b1 = -(vr - cr), b2 = -(vl - cl);
  const double t1 = fmax(0.0, a1);
  const double ap = fmax(t1, a2);
  const int sap = (a2 > t1) ? 2 : (a1 > 0.0 ? 1 : 0);
  const double t2 = fmax(0.0, b1);
  const double am = fmax(t2, b2);
  const int sam = (b2 > t2) ? 2 : (b1 > 0.0 ? 1 : 0);
  const double iD = rcp_deriv(ap + am);
  const double apm = ap * am;
  double gN[5], gD = 0.0, gap = 0.0, gam_ = 0.0;
  for (int k = 0; k < 5; ++k) {
    const double ds = sr[k] - sl[k];
    const double F = fma(ap, fl[k], fma(am, fr[k], -apm * ds)) * iD;
    gN[k] = gF[k] * iD;
    gD = fma(-gN[k], F, gD);
  }
  gap = gD;
  gam_ = gD;
  double gfl[5], gfr[5], gsl[5], gsr[5];
  for (int k = 0; k < 5; ++k) {
    const double ds = sr[k] - sl[k];
    gap = fma(gN[k], fma(-am, ds, fl[k]), gap);
    gam_ = fma(gN[k], fma(-ap, ds, fr[k]), gam_);
    gfl[k] = gN[k] * ap;
    gfr[k] = gN[k] * am;
    gsl[k] = gN[k] * apm;
    gsr[k] = -gsl[k];
  }
  double gvl = 0, gvr = 0, gcl = 0, gcr = 0;
  if (sap == 1) { gvr += gap; gcr += gap; }
  else if (sap == 2) { gvl += gap; gcl += gap; }
  if (sam == 1) { gcr += gam_; gvr -= gam_; }
  else if (sam == 2) { gcl += gam_; gvl -= gam_; }
  double gpl = 0, gpr = 0, gdl = 0, gdr = 0, gel = 0, ger = 0;
  double gul[3] = {0, 0, 0}, gur[3] = {0, 0, 0};
  // c = sqrt(gam p / d): dc/dp = c/(2p) = gam/(2 d c), dc/dd = -c/(2d) = -c^2/(2 d c)
  if (cl > 0.0) {
    const double t = kHalf * gcl * rcp_deriv(dl * cl);
    gpl += gam * t;
    gdl -= cl * cl * t;
  }
  if (cr > 0.0) {
    const double t = kHalf * gcr * rcp_deriv(dr * cr);
    gpr += gam * t;
    gdr -= cr * cr * t;
  }
  // fluxes: f0 = d v, f(1+j) = [j == DIR] p + s(1+j) v, f4 = (s4 + p) v
  gdl = fma(gfl[0], vl, gdl); gvl = fma(gfl[0], sl[0], gvl);
  gdr = fma(gfr[0], vr, gdr); gvr = fma(gfr[0], sr[0], gvr);
  for (int j = 0; j < 3; ++j) {
    if (j == DIR) { gpl += gfl[1 + j]; gpr += gfr[1 + j]; }
    gsl[1 + j] = fma(gfl[1 + j], vl, gsl[1 + j]); gvl = fma(gfl[1 + j], sl[1 + j], gvl);
    gsr[1 + j] = fma(gfr[1 + j], vr, gsr[1 + j]); gvr = fma(gfr[1 + j], sr[1 + j], gvr);
  }
  gsl[4] = fma(gfl[4], vl, gsl[4]); gpl = fma(gfl[4], vl, gpl); gvl = fma(gfl[4], sl[4] + pl, gvl);
  gsr[4] = fma(gfr[4], vr, gsr[4]); gpr = fma(gfr[4], vr, gpr); gvr = fma(gfr[4], sr[4] + pr, gvr);
  // conserved face variables s0 = d, s(1+j) = d u_j, s4 = e + d K/2
  gdl += gsl[0]; gdr += gsr[0];
  for (int j = 0; j < 3; ++j) {
    gdl = fma(gsl[1 + j], ul[j], gdl); gul[j] = fma(gsl[1 + j], dl, gul[j]);
    gdr = fma(gsr[1 + j], ur[j], gdr); gur[j] = fma(gsr[1 + j], dr, gur[j]);
  }
  gel += gsl[4]; gdl = fma(gsl[4], kHalf * Kl, gdl);
  ger += gsr[4]; gdr = fma(gsr[4], kHalf * Kr, gdr);
  const double hdl = gsl[4] * dl, hdr = gsr[4] * dr;
  for (int j = 0; j < 3; ++j) {
    gul[j] = fma(hdl, ul[j], gul[j]);
    gur[j] = fma(hdr, ur[j], gur[j]);
  }
  gul[DIR] += gvl;
  gur[DIR] += gvr;
  gL = FS6{gdl, gul[0], gul[1], gul[2], gpl, gel};
  gR = FS6{gdr, gur[0], gur[1], gur[2], gpr, ger};
}

// generalised minmod slope: slope3's value (bit for bit) and the index of the
// selected argument (1: theta*(c1-c0), 2: half*(c2-c0), 3: theta*(c2-c1); 0 when
// the slope is zero)
__device__ __forceinline__ double slope_and_sel(double c0, double c1, double c2, int& sel) {
  const double d1 = c1 - c0, d2 = c2 - c0, d3 = c2 - c1;
  const double x1 = fabs(kTheta * d1), x2 = fabs(kHalf * d2), x3 = fabs(kTheta * d3);
  const double m23 = fmin(x2, x3);
  const double m = fmin(x1, m23);
  const bool pos = (d1 > 0.0) && (d3 > 0.0), neg = (d1 < 0.0) && (d3 < 0.0);
  sel = !(pos || neg) ? 0 : (x1 <= m23 ? 1 : (x2 <= x3 ? 2 : 3));
  return pos ? m : (neg ? -m : 0.0);
}

}  // namespace bx

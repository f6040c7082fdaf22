// bx_adjoint.cu -- discrete adjoint of the fused hydro step (frozen dt and branches).
//
// The differentiated map is the step the fused stage kernels compute: from the
// conserved planes X (ghosts read through the donor rule) and n sources short
// of the reference state,
//   C0' = src^n(X),  C1 = C0' + L0(C0'),  C2 = (C0' + C1 + L1(C1, C0'))/2,
// with the next step starting from C2 (two sources short).  L0/L1 are the flux
// operators of stage 0/1 (stage 1 takes its pressure with the stage-0
// velocity, main.f90:351-355).  dt comes from the forward run and is held
// fixed; every max/min/limiter branch is taken where the forward values put it;
// the floors of flux.f90:223-230 must not fire in the forward (checked).
//
// The reverse of one stage runs five kernels over full-grid scratch planes:
//  R1 primitives of every cell;  R2 per face: recompute the two face states
//  and the HLL flux, and turn the flux adjoint into the adjoints of the plus
//  state of the low cell and the minus state of the high cell (each written by
//  exactly one face: no atomics);  R3 per cell: adjoint of the MUSCL states
//  into direct primitive adjoints and slope adjoints;  R4 per cell: gather the
//  slope adjoints of the (up to three) slopes that read this cell's
//  primitives, then primitives -> conserved variables;  R5 per interior cell:
//  add the adjoints that landed on face ghosts back onto their donor cells.
//
// Snapshots follow a binomial (revolve-style) schedule in a fixed pool of
// plane sets, so a run of any length is reversed in bounded memory.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <string>
#include <vector>

#include "bx_adjoint_math.cuh"
#include "bx_handle.h"
#include "bx_internal.h"

using namespace bx;

namespace {

constexpr int AB = 256;
inline int ablk(long long n) { return (int)((n + AB - 1) / AB); }

__device__ __forceinline__ int amap(int c, int a0, int a1, int wl, int wr, bool& flip) {
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

struct C5 {
  double d, m1, m2, m3, E;
};

// conserved values of cell (x,y,z) through the donor rule; returns the donor index
__device__ __forceinline__ C5 aload(const double* P, long long ps, const Geom& g, int x, int y, int z,
                                    long long* donor = nullptr, unsigned* sgn = nullptr) {
  bool fx = false, fy = false, fz = false;
  const int xx = amap(x, g.ax0, g.ax1, g.wall[0], g.wall[1], fx);
  const int yy = amap(y, g.ay0, g.ay1, g.wall[2], g.wall[3], fy);
  const int zz = g.threed ? amap(z, g.az0, g.az1, g.wall[4], g.wall[5], fz) : z;
  const long long c = xx + (long long)yy * g.sy + (long long)zz * g.sz;
  C5 r{P[c], P[ps + c], P[2 * ps + c], P[3 * ps + c], P[4 * ps + c]};
  if (fx) r.m1 = -r.m1;
  if (fy) r.m2 = -r.m2;
  if (fz) r.m3 = -r.m3;
  if (donor) *donor = c;
  if (sgn) *sgn = (fx ? 1u : 0u) | (fy ? 2u : 0u) | (fz ? 4u : 0u);
  return r;
}

__device__ __forceinline__ bool ainterior(const Geom& g, int x, int y, int z) {
  return x >= g.ax0 && x < g.ax1 && y >= g.ay0 && y < g.ay1 &&
         (!g.threed || (z >= g.az0 && z < g.az1));
}

__device__ __forceinline__ void decode(const Geom& g, long long i, int& x, int& y, int& z) {
  x = (int)(i % g.nx);
  y = (int)((i / g.nx) % g.ny);
  z = (int)(i / g.sz);
}

// ---- primitives of a stage (as load_prim of the stage kernels)
// P planes: 0 rho, 1-3 u, 4 p, 5 eps, 6 c
__global__ void k_r1_prims(Geom g, int stage, const double* A, const double* B, double* P) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= g.ng) return;
  int x, y, z;
  decode(g, i, x, y, z);
  const long long n = g.ng;
  const C5 a = aload(A, n, g, x, y, z);
  const double u1 = a.m1 / a.d, u2 = a.m2 / a.d, u3 = a.m3 / a.d;
  const double e = recon_eps(a.d, a.E, u1, u2, u3, g.small_eps);
  double p;
  if (stage == 0) {
    p = e * g.gm1;
  } else {
    const C5 b = aload(B, n, g, x, y, z);
    const double s1 = b.m1 / b.d, s2 = b.m2 / b.d, s3 = b.m3 / b.d;
    p = eos_pressure(a.d, a.E, s1, s2, s3, g.gm1, g.small_eps);
  }
  P[i] = a.d;
  P[n + i] = u1;
  P[2 * n + i] = u2;
  P[3 * n + i] = u3;
  P[4 * n + i] = p;
  P[5 * n + i] = e;
  P[6 * n + i] = sqrt(p * g.gam / a.d);
}

__device__ __forceinline__ Prim pget(const double* P, long long n, long long i) {
  return Prim{P[i], P[n + i], P[2 * n + i], P[3 * n + i], P[4 * n + i], P[5 * n + i],
              P[6 * n + i]};
}
__device__ __forceinline__ double pq(const Prim& q, int k) {
  return k == 0 ? q.d : k == 1 ? q.u1 : k == 2 ? q.u2 : k == 3 ? q.u3 : k == 4 ? q.p : q.e;
}
__device__ __forceinline__ double fq(const FS6& q, int k) {
  return k == 0 ? q.d : k == 1 ? q.u1 : k == 2 ? q.u2 : k == 3 ? q.u3 : k == 4 ? q.p : q.e;
}
__device__ __forceinline__ double ud_of(const Prim& q, int dir) {
  return dir == 0 ? q.u1 : dir == 1 ? q.u2 : q.u3;
}

// face states of cell i in direction dir (ghost cells: the cell values)
__device__ __forceinline__ void states_of(const Geom& g, const double* P, long long i, long long st,
                                          bool interior, int dir, double dt, FaceState& mi,
                                          FaceState& pl) {
  const long long n = g.ng;
  const Prim c = pget(P, n, i);
  if (!interior) {
    ghost_states(c, mi, pl);
    return;
  }
  const Prim m = pget(P, n, i - st), p = pget(P, n, i + st);
  const double ds = dir == 0 ? g.dx : dir == 1 ? g.dy : g.dz;
  const double ids = dir == 0 ? g.idx : dir == 1 ? g.idy : g.idz;
  const double sd = slope3(m.d, c.d, p.d), s1 = slope3(m.u1, c.u1, p.u1);
  const double s2 = slope3(m.u2, c.u2, p.u2), s3 = slope3(m.u3, c.u3, p.u3);
  const double sp = slope3(m.p, c.p, p.p), se = slope3(m.e, c.e, p.e);
  if (g.pow2)
    muscl_states<true>(c, ud_of(c, dir), sd, s1, s2, s3, sp, se, dt, ds, ids, mi, pl);
  else
    muscl_states<false>(c, ud_of(c, dir), sd, s1, s2, s3, sp, se, dt, ds, ids, mi, pl);
}

// G planes: [(dir*2 + side)*6 + q], side 0 = minus-state adjoint, 1 = plus-state adjoint
// R2: faces of direction DIR; thread per high-side cell (index along DIR in [a0, a1])
template <int DIR>
__global__ void k_r2_faces(Geom g, const double* P, const double* lamL, double dt, double* G) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= g.ng) return;
  int x, y, z;
  decode(g, i, x, y, z);
  const int c[3] = {x, y, z};
  const int lo[3] = {g.ax0, g.ay0, g.az0}, hi[3] = {g.ax1, g.ay1, g.az1};
  for (int k = 0; k < 3; ++k) {
    if (k == DIR) {
      if (c[k] < lo[k] || c[k] > hi[k]) return;
    } else if (k < 2 || g.threed) {
      if (c[k] < lo[k] || c[k] >= hi[k]) return;
    }
  }
  const long long n = g.ng;
  const long long st = DIR == 0 ? 1 : DIR == 1 ? g.sy : g.sz;
  const long long L = i - st, R = i;
  int lx = x, ly = y, lz = z;
  if (DIR == 0) lx -= 1; else if (DIR == 1) ly -= 1; else lz -= 1;
  const bool Lin = ainterior(g, lx, ly, lz), Rin = ainterior(g, x, y, z);
  FaceState Lm, Lp, Rm, Rp;
  states_of(g, P, L, st, Lin, DIR, dt, Lm, Lp);
  states_of(g, P, R, st, Rin, DIR, dt, Rm, Rp);
  const double area = DIR == 0 ? g.ayz : DIR == 1 ? g.axz : g.axy;
  const double coef = -(dt / g.vol) * area;
  double gF[5];
  for (int q = 0; q < 5; ++q) {
    const double lL = Lin ? lamL[q * n + L] : 0.0;
    const double lR = Rin ? lamL[q * n + R] : 0.0;
    gF[q] = coef * (lL - lR);
  }
  FS6 gL, gR;
  hll_vjp<DIR>(Lp, Rm, g.gam, gF, gL, gR);
  double* Gp = G + ((DIR * 2 + 1) * 6) * n;
  double* Gm = G + ((DIR * 2 + 0) * 6) * n;
  for (int q = 0; q < 6; ++q) {
    Gp[q * n + L] = fq(gL, q);
    Gm[q * n + R] = fq(gR, q);
  }
}

// R3: MUSCL adjoint per cell.  LQ planes: 7 direct primitive adjoints (q0..5, c);
// LS planes: [dir*6 + q] slope adjoints; SEL: [dir*6 + q] slope selections.
__global__ void k_r3_muscl(Geom g, const double* P, const double* G, double dt, double* LQ,
                           double* LS, uint8_t* SEL) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= g.ng) return;
  int x, y, z;
  decode(g, i, x, y, z);
  const long long n = g.ng;
  const bool in = ainterior(g, x, y, z);
  double lq[7] = {0, 0, 0, 0, 0, 0, 0};
  const int ndir = g.threed ? 3 : 2;
  const Prim c = pget(P, n, i);
  for (int dir = 0; dir < ndir; ++dir) {
    double gm[6], gp[6];
    for (int q = 0; q < 6; ++q) {
      gm[q] = G[((dir * 2 + 0) * 6 + q) * n + i];
      gp[q] = G[((dir * 2 + 1) * 6 + q) * n + i];
    }
    if (!in) {
      for (int q = 0; q < 6; ++q) lq[q] += gm[q] + gp[q];
      continue;
    }
    const long long st = dir == 0 ? 1 : dir == 1 ? g.sy : g.sz;
    const Prim m = pget(P, n, i - st), p = pget(P, n, i + st);
    double s[6];
    for (int q = 0; q < 6; ++q) {
      const double c0 = pq(m, q), c1 = pq(c, q), c2 = pq(p, q);
      s[q] = slope3(c0, c1, c2);
      SEL[(dir * 6 + q) * n + i] = (uint8_t)slope_sel(c0, c1, c2);
    }
    const double ud = ud_of(c, dir);
    const double ds = dir == 0 ? g.dx : dir == 1 ? g.dy : g.dz;
    const double rr = dt / ds;
    const double lp = fmax(ud + c.c, 0.0) * rr, lm = fmin(ud - c.c, 0.0) * rr;
    const double hm = kHalf * (-1.0 - lm), hp = kHalf * (1.0 - lp);
    double ghm = 0, ghp = 0;
    for (int q = 0; q < 6; ++q) {
      lq[q] += gm[q] + gp[q];
      LS[(dir * 6 + q) * n + i] = hm * gm[q] + hp * gp[q];
      ghm += s[q] * gm[q];
      ghp += s[q] * gp[q];
    }
    const double glm = -kHalf * ghm, glp = -kHalf * ghp;
    if (ud + c.c > 0.0) { lq[1 + dir] += glp * rr; lq[6] += glp * rr; }
    if (ud - c.c < 0.0) { lq[1 + dir] += glm * rr; lq[6] -= glm * rr; }
  }
  if (!in)
    for (int k = 0; k < 18; ++k) { LS[k * n + i] = 0.0; SEL[k * n + i] = 0; }
  else if (!g.threed)
    for (int k = 12; k < 18; ++k) { LS[k * n + i] = 0.0; SEL[k * n + i] = 0; }
  for (int q = 0; q < 7; ++q) LQ[q * n + i] = lq[q];
}

// R4: total primitive adjoint of cell k, then primitives -> conserved.
// GK planes: 0-4 adjoint of A's conserved values at k, 5-9 of B's (stage 1).
__global__ void k_r4_cells(Geom g, int stage, const double* A, const double* B, const double* P,
                           const double* LQ, const double* LS, const uint8_t* SEL, double* GK) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= g.ng) return;
  int x, y, z;
  decode(g, i, x, y, z);
  const long long n = g.ng;
  double gq[7];
  for (int q = 0; q < 7; ++q) gq[q] = LQ[q * n + i];
  const int ndir = g.threed ? 3 : 2;
  const int c[3] = {x, y, z};
  const int lim[3] = {g.nx, g.ny, g.nz};
  for (int dir = 0; dir < ndir; ++dir) {
    const long long st = dir == 0 ? 1 : dir == 1 ? g.sy : g.sz;
    // slopes of cells j = i - st (i is its plus neighbour), i, i + st (i is its minus neighbour)
    for (int o = -1; o <= 1; ++o) {
      const int cj = c[dir] + o;
      if (cj < 0 || cj >= lim[dir]) continue;
      const long long j = i + o * st;
      int jx = x, jy = y, jz = z;
      if (dir == 0) jx = cj; else if (dir == 1) jy = cj; else jz = cj;
      if (!ainterior(g, jx, jy, jz)) continue;
      for (int q = 0; q < 6; ++q) {
        const int sel = SEL[(dir * 6 + q) * n + j];
        if (!sel) continue;
        double k0, k1, k2;
        slope_coef(sel, k0, k1, k2);
        const double kk = o == 1 ? k0 : (o == 0 ? k1 : k2);
        gq[q] += kk * LS[(dir * 6 + q) * n + j];
      }
    }
  }
  // primitives -> conserved values (load through the donor rule, like R1)
  const C5 a = aload(A, n, g, x, y, z);
  const double rho = a.d;
  const double u[3] = {a.m1 / rho, a.m2 / rho, a.m3 / rho};
  const double K = u[0] * u[0] + u[1] * u[1] + u[2] * u[2];
  const double e = recon_eps(rho, a.E, u[0], u[1], u[2], g.small_eps);
  double p;
  double gA[5] = {0, 0, 0, 0, 0}, gB[5] = {0, 0, 0, 0, 0};
  double grho = gq[0], gu[3] = {gq[1], gq[2], gq[3]}, gp = gq[4], ge = gq[5];
  C5 b{};
  double us[3] = {0, 0, 0};
  if (stage == 0) {
    p = e * g.gm1;
  } else {
    b = aload(B, n, g, x, y, z);
    us[0] = b.m1 / b.d; us[1] = b.m2 / b.d; us[2] = b.m3 / b.d;
    p = eos_pressure(rho, a.E, us[0], us[1], us[2], g.gm1, g.small_eps);
  }
  const double cs = sqrt(p * g.gam / rho);
  if (cs > 0.0) {
    gp += gq[6] * cs / (2.0 * p);
    grho -= gq[6] * cs / (2.0 * rho);
  }
  if (stage == 0) {
    ge += gp * g.gm1;
  } else {
    const double Ks = us[0] * us[0] + us[1] * us[1] + us[2] * us[2];
    if (a.E - rho * kHalf * Ks > g.small_eps) {
      gA[4] += gp * g.gm1;
      grho += gp * g.gm1 * (-kHalf * Ks);
      double gus[3];
      for (int j = 0; j < 3; ++j) gus[j] = gp * g.gm1 * (-rho * us[j]);
      for (int j = 0; j < 3; ++j) {
        gB[1 + j] += gus[j] / b.d;
        gB[0] -= gus[j] * us[j] / b.d;
      }
    }
  }
  if (a.E - kHalf * rho * K > g.small_eps) {
    gA[4] += ge;
    grho += ge * (-kHalf * K);
    for (int j = 0; j < 3; ++j) gu[j] += ge * (-rho * u[j]);
  }
  for (int j = 0; j < 3; ++j) {
    gA[1 + j] += gu[j] / rho;
    grho -= gu[j] * u[j] / rho;
  }
  gA[0] += grho;
  for (int q = 0; q < 5; ++q) {
    GK[q * n + i] = gA[q];
    GK[(5 + q) * n + i] = gB[q];
  }
}

// R5: interior cell i collects its own adjoint and those of the face ghosts that
// read it (with the momentum signs of the donor rule); accumulates into outA/outB.
__global__ void k_r5_fold(Geom g, int stage, const double* GK, double* outA, double* outB) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= g.ng) return;
  int x, y, z;
  decode(g, i, x, y, z);
  if (!ainterior(g, x, y, z)) return;
  const long long n = g.ng;
  double a[10];
  for (int q = 0; q < 10; ++q) a[q] = GK[q * n + i];
  const int ndir = g.threed ? 3 : 2;
  const int lo[3] = {g.ax0, g.ay0, g.az0}, hi[3] = {g.ax1, g.ay1, g.az1};
  const int c[3] = {x, y, z};
  for (int dir = 0; dir < ndir; ++dir) {
    const int wl = g.wall[2 * dir], wr = g.wall[2 * dir + 1];
    const long long st = dir == 0 ? 1 : dir == 1 ? g.sy : g.sz;
    const int ghosts[4] = {lo[dir] - 2, lo[dir] - 1, hi[dir], hi[dir] + 1};
    for (int k = 0; k < 4; ++k) {
      bool flip = false;
      const int dnr = amap(ghosts[k], lo[dir], hi[dir], wl, wr, flip);
      if (dnr != c[dir]) continue;
      const long long gi = i + (long long)(ghosts[k] - c[dir]) * st;
      for (int q = 0; q < 10; ++q) {
        const double v = GK[q * n + gi];
        const bool neg = flip && ((q % 5) == 1 + dir);
        a[q] += neg ? -v : v;
      }
    }
  }
  for (int q = 0; q < 5; ++q) outA[q * n + i] += a[q];
  if (stage == 1)
    for (int q = 0; q < 5; ++q) outB[q * n + i] += a[5 + q];
  else
    for (int q = 0; q < 5; ++q) outA[q * n + i] += a[5 + q];
}

// C0' = src^nsrc(X) on interior cells (source.f90:176-182)
__global__ void k_adj_src(Geom g, const double* X, int nsrc, double* out) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= g.ng) return;
  const long long n = g.ng;
  double d = X[i], m1 = X[n + i], m2 = X[2 * n + i], m3 = X[3 * n + i], E = X[4 * n + i];
  for (int k = 0; k < nsrc; ++k) E = source_energy(d, m1, m2, m3, E, g.small_eps);
  out[i] = d;
  out[n + i] = m1;
  out[2 * n + i] = m2;
  out[3 * n + i] = m3;
  out[4 * n + i] = E;
}

// lam <- (d src^nsrc / dX)^T lam on interior cells (ghost entries set to zero)
__global__ void k_adj_src_vjp(Geom g, const double* X, int nsrc, double* lam) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= g.ng) return;
  int x, y, z;
  decode(g, i, x, y, z);
  const long long n = g.ng;
  if (!ainterior(g, x, y, z)) {
    for (int q = 0; q < 5; ++q) lam[q * n + i] = 0.0;
    return;
  }
  const double d = X[i], m[3] = {X[n + i], X[2 * n + i], X[3 * n + i]};
  double Es[3];
  Es[0] = X[4 * n + i];
  for (int k = 0; k < nsrc; ++k) Es[k + 1] = source_energy(d, m[0], m[1], m[2], Es[k], g.small_eps);
  double l[5];
  for (int q = 0; q < 5; ++q) l[q] = lam[q * n + i];
  const double K = kin_mom(d, m[0], m[1], m[2]);
  for (int k = nsrc - 1; k >= 0; --k) {
    // E' = max(E - K, eps) + K
    if (!(Es[k] - K > g.small_eps)) {
      const double gE = l[4];
      l[4] = 0.0;
      for (int j = 0; j < 3; ++j) l[1 + j] += gE * m[j] / d;
      l[0] += gE * (-K / d);
    }
  }
  for (int q = 0; q < 5; ++q) lam[q * n + i] = l[q];
}

__global__ void k_axpy(long long n, double a, const double* x, double* y) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i < n) y[i] += a * x[i];
}
__global__ void k_scale_copy(long long n, double a, const double* x, double* y) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i < n) y[i] = a * x[i];
}
__global__ void k_set_clock(Ctrl* c, double dt, int active) {
  c->dt = dt;
  c->active = active;
}
__global__ void k_record_dt(const Ctrl* c, double* dts, long long k) { dts[k] = c->dt; }

}  // namespace

// ------------------------------------------------------------------ host engine
struct bx_adj {
  bx_handle* h = nullptr;  // geometry, tiles, control block, stream
  long long ng = 0;
  long long nsteps = 0;
  int snaps = 0;
  std::vector<double*> pool;  // plane sets for snapshots
  std::vector<int> pool_free;
  std::vector<double> dts;    // frozen dt sequence
  double* d_dts = nullptr;
  std::vector<int> step_nsrc;
  // work planes
  double *W0 = nullptr, *W1 = nullptr, *W2 = nullptr;  // C0', C1, scratch state
  double* XT = nullptr;  // state after the last step of the forward run (C2_T)
  double *lamA = nullptr, *lamB = nullptr, *lamT = nullptr, *lamC1 = nullptr;
  double *P = nullptr, *G = nullptr, *LQ = nullptr, *LS = nullptr, *GK = nullptr;
  uint8_t* SEL = nullptr;
  double ms_fwd = 0.0, ms_bwd = 0.0;
  long long fwd_steps_in_bwd = 0;
  size_t bytes = 0;
  bool have_forward = false;
  int nsrc0 = 1;
  std::string err;
};

static std::string g_adj_err;

#define ACK(expr)                                                     \
  do {                                                                \
    cudaError_t e_ = (expr);                                          \
    if (e_ != cudaSuccess) {                                          \
      A->err = std::string(#expr) + ": " + cudaGetErrorString(e_);    \
      return e_ == cudaErrorMemoryAllocation ? BX_ERR_NOMEM : BX_ERR_CUDA; \
    }                                                                 \
  } while (0)

static int aerr(bx_adj* A, int code, const std::string& m) {
  if (A) A->err = m;
  else g_adj_err = m;
  return code;
}

static int amalloc(bx_adj* A, double** p, long long ndoubles) {
  ACK(cudaMalloc(p, std::max<long long>(ndoubles, 2) * sizeof(double)));
  A->bytes += ndoubles * sizeof(double);
  return BX_OK;
}

// one forward step from X into Y (fused stage kernels, dt frozen at dts[k]),
// using W1 for the stage-0 result.  Returns the guard flags in *flags if given.
static int fwd_step(bx_adj* A, const double* X, int nsrc, double dt, double* Y,
                    bool stage0_only = false) {
  bx_handle* h = A->h;
  StageArgs a{};
  a.ctrl = h->d_ctrl;
  a.geom = h->d_geom;
  a.tiles = h->d_tiles;
  a.ncells_total = h->g.ng;
  a.nsrc = nsrc;
  k_set_clock<<<1, 1, 0, h->stream>>>(h->d_ctrl, dt, 1);
  a.X = X;
  a.Y = nullptr;
  a.out = A->W1;
  ACK(launch_stage(0, h->g.pow2 ? 1 : 0, h->g.threed != 0, a, h->ntiles, h->stream));
  if (stage0_only) return BX_OK;
  a.Y = A->W1;
  a.out = Y;
  ACK(launch_stage(1, h->g.pow2 ? 1 : 0, h->g.threed != 0, a, h->ntiles, h->stream));
  return BX_OK;
}

// reverse of one stage: lamL = adjoint of the flux-operator output (interior cells);
// accumulates into outA (and outB for stage 1)
static int rev_stage(bx_adj* A, int stage, const double* SA, const double* SB, const double* lamL,
                     double dt, double* outA, double* outB) {
  bx_handle* h = A->h;
  const Geom& g = h->g;
  cudaStream_t s = h->stream;
  const long long n = g.ng;
  k_r1_prims<<<ablk(n), AB, 0, s>>>(g, stage, SA, SB, A->P);
  ACK(cudaMemsetAsync(A->G, 0, 36 * n * sizeof(double), s));
  k_r2_faces<0><<<ablk(n), AB, 0, s>>>(g, A->P, lamL, dt, A->G);
  k_r2_faces<1><<<ablk(n), AB, 0, s>>>(g, A->P, lamL, dt, A->G);
  if (g.threed) k_r2_faces<2><<<ablk(n), AB, 0, s>>>(g, A->P, lamL, dt, A->G);
  k_r3_muscl<<<ablk(n), AB, 0, s>>>(g, A->P, A->G, dt, A->LQ, A->LS, A->SEL);
  k_r4_cells<<<ablk(n), AB, 0, s>>>(g, stage, SA, SB, A->P, A->LQ, A->LS, A->SEL, A->GK);
  k_r5_fold<<<ablk(n), AB, 0, s>>>(g, stage, A->GK, outA, outB);
  ACK(cudaGetLastError());
  return BX_OK;
}

// lam (adjoint of the step output, C2) -> lam (adjoint of the step input X)
static int rev_step(bx_adj* A, const double* X, int nsrc, double dt, double* lam) {
  bx_handle* h = A->h;
  const Geom& g = h->g;
  cudaStream_t s = h->stream;
  const long long n5 = 5 * g.ng;
  // recompute C0' and C1
  k_adj_src<<<ablk(g.ng), AB, 0, s>>>(g, X, nsrc, A->W0);
  if (int r = fwd_step(A, X, nsrc, dt, nullptr, true)) return r;  // W1 <- C1
  // C2 = (C0' + C1 + L1)/2: half of lam to C0', C1 and the flux operator
  k_scale_copy<<<ablk(n5), AB, 0, s>>>(n5, kHalf, lam, A->lamT);   // lamT: lam/2 (L1 input)
  k_scale_copy<<<ablk(n5), AB, 0, s>>>(n5, kHalf, lam, A->lamC1);  // adjoint of C1
  k_scale_copy<<<ablk(n5), AB, 0, s>>>(n5, kHalf, lam, A->lamA);   // adjoint of C0'
  if (int r = rev_stage(A, 1, A->W1, A->W0, A->lamT, dt, A->lamC1, A->lamA)) return r;
  // C1 = C0' + L0(C0')
  k_axpy<<<ablk(n5), AB, 0, s>>>(n5, 1.0, A->lamC1, A->lamA);
  if (int r = rev_stage(A, 0, A->W0, A->W0, A->lamC1, dt, A->lamA, A->lamA)) return r;
  // through the sources: adjoint of X
  ACK(cudaMemcpyAsync(lam, A->lamA, n5 * sizeof(double), cudaMemcpyDeviceToDevice, s));
  k_adj_src_vjp<<<ablk(g.ng), AB, 0, s>>>(g, X, nsrc, lam);
  ACK(cudaGetLastError());
  return BX_OK;
}

static double* take_slot(bx_adj* A) {
  if (A->pool_free.empty()) return nullptr;
  const int k = A->pool_free.back();
  A->pool_free.pop_back();
  return A->pool[k];
}
static void give_slot(bx_adj* A, double* p) {
  for (size_t k = 0; k < A->pool.size(); ++k)
    if (A->pool[k] == p) A->pool_free.push_back((int)k);
}

static long long binom(long long n, long long k) {
  if (k < 0 || k > n) return 0;
  long long r = 1;
  for (long long i = 1; i <= k; ++i) {
    r = r * (n - k + i) / i;
    if (r > (1ll << 50)) return 1ll << 50;
  }
  return r;
}

// state of step `to` from the state of step `from` (held in src) into dst,
// ping-ponging between dst and W2 so the last step lands in dst
static int advance(bx_adj* A, const double* src, long long from, long long to, double* dst) {
  const long long n5 = 5 * A->h->g.ng;
  cudaStream_t s = A->h->stream;
  if (to == from) {
    ACK(cudaMemcpyAsync(dst, src, n5 * sizeof(double), cudaMemcpyDeviceToDevice, s));
    return BX_OK;
  }
  const double* cur = src;
  for (long long k = from; k < to; ++k) {
    double* out = ((to - k) % 2 == 1) ? dst : A->W2;
    if (int r = fwd_step(A, cur, A->step_nsrc[k], A->dts[k], out)) return r;
    cur = out;
    A->fwd_steps_in_bwd += 1;
  }
  return BX_OK;
}

// reverse steps [a, b) with the state of step a in Xa (owned by the caller)
static int reverse_range(bx_adj* A, const double* Xa, long long a, long long b, double* lam) {
  const long long l = b - a;
  if (l <= 0) return BX_OK;
  if (l == 1) return rev_step(A, Xa, A->step_nsrc[a], A->dts[a], lam);
  const int s = (int)A->pool_free.size();
  if (s == 0) {
    // no snapshot left: rebuild each state from Xa (into lamB, free during reversal)
    for (long long k = b - 1; k >= a; --k) {
      if (int r = advance(A, Xa, a, k, A->lamB)) return r;
      if (int r = rev_step(A, A->lamB, A->step_nsrc[k], A->dts[k], lam)) return r;
    }
    return BX_OK;
  }
  long long r = 1;
  while (binom(s + r, s) < l) ++r;
  long long l2 = std::min(binom(s - 1 + r, s - 1), l - 1);
  if (l2 < 1) l2 = 1;
  const long long m = b - l2;
  double* slot = take_slot(A);
  if (int rc = advance(A, Xa, a, m, slot)) return rc;
  if (int rc = reverse_range(A, slot, m, b, lam)) return rc;
  give_slot(A, slot);
  return reverse_range(A, Xa, a, m, lam);
}

extern "C" {

const char* bx_adj_last_error(bx_adj* A) { return A ? A->err.c_str() : g_adj_err.c_str(); }

int bx_adj_destroy(bx_adj* A) {
  if (!A) return BX_OK;
  if (A->h && A->h->stream) cudaStreamSynchronize(A->h->stream);
  for (double* p : A->pool) cudaFree(p);
  double* ps[] = {A->W0, A->W1, A->W2, A->XT, A->lamA, A->lamB, A->lamT, A->lamC1,
                  A->P,  A->G,  A->LQ, A->LS,   A->GK,   A->d_dts};
  for (double* p : ps) cudaFree(p);
  cudaFree(A->SEL);
  if (A->h) bx_destroy(A->h);
  delete A;
  return BX_OK;
}

int bx_adj_create(const bx_params* params, int64_t nsteps, int32_t snapshots, bx_adj** out) {
  if (!params || !out || nsteps <= 0 || snapshots < 1)
    return aerr(nullptr, BX_ERR_ARG, "bad arguments");
  bx_adj* A = new bx_adj();
  if (int r = bx_create(params, &A->h)) {
    g_adj_err = bx_last_error(nullptr);
    delete A;
    return r;
  }
  if (!A->h->eligible) {
    bx_adj_destroy(A);
    return aerr(nullptr, BX_ERR_UNSUPPORTED,
                "the adjoint follows the fused stage kernels; this grid's ghost fill does not "
                "resolve within two sweeps");
  }
  const long long n = A->h->g.ng;
  A->ng = n;
  A->nsteps = nsteps;
  A->snaps = (int)std::min<long long>(snapshots, nsteps);
  A->dts.assign(nsteps, 0.0);
  A->step_nsrc.assign(nsteps, 2);
  int rc = 0;
  auto fail = [&](int code) {
    g_adj_err = A->err;
    bx_adj_destroy(A);
    return code;
  };
  // the pool holds the initial state plus the free snapshots
  A->pool.assign(A->snaps + 1, nullptr);
  for (int k = 0; k <= A->snaps; ++k)
    if ((rc = amalloc(A, &A->pool[k], 5 * n))) return fail(rc);
  double** planes5[] = {&A->W0, &A->W1, &A->W2, &A->XT, &A->lamA, &A->lamB, &A->lamT, &A->lamC1};
  for (double** p : planes5)
    if ((rc = amalloc(A, p, 5 * n))) return fail(rc);
  if ((rc = amalloc(A, &A->P, 7 * n))) return fail(rc);
  if ((rc = amalloc(A, &A->G, 36 * n))) return fail(rc);
  if ((rc = amalloc(A, &A->LQ, 7 * n))) return fail(rc);
  if ((rc = amalloc(A, &A->LS, 18 * n))) return fail(rc);
  if ((rc = amalloc(A, &A->GK, 10 * n))) return fail(rc);
  if ((rc = amalloc(A, &A->d_dts, nsteps))) return fail(rc);
  if (cudaMalloc(&A->SEL, 18 * n) != cudaSuccess) {
    A->err = "SEL allocation";
    return fail(BX_ERR_NOMEM);
  }
  A->bytes += 18 * n;
  *out = A;
  return BX_OK;
}

int bx_adj_set_stream(bx_adj* A, void* s) {
  if (!A) return BX_ERR_ARG;
  return bx_set_stream(A->h, s);
}

// Forward run of nsteps from cons0 (device SoA planes of the reference cons,
// 5 x ngrid; ghosts are ignored) into consT (the reference cons after the
// run, ghosts filled).  frozen=0: dt by the CFL rule of main.f90, recorded;
// frozen=1: the recorded dt sequence of the last unfrozen forward.
int bx_adj_forward(bx_adj* A, const double* cons0, double* consT, int32_t frozen) {
  if (!A || !cons0 || !consT) return aerr(A, BX_ERR_ARG, "bad arguments");
  if (frozen && !A->have_forward) return aerr(A, BX_ERR_STATE, "no recorded dt sequence");
  bx_handle* h = A->h;
  const Geom& g = h->g;
  cudaStream_t s = h->stream;
  const long long n5 = 5 * g.ng;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  ACK(cudaEventRecord(e0, s));
  double* X0 = A->pool[0];
  ACK(cudaMemcpyAsync(X0, cons0, n5 * sizeof(double), cudaMemcpyDeviceToDevice, s));
  // initial Courant rate and clock
  Ctrl c{};
  c.cfl = h->P.cfl;
  c.endtime = 1e300;
  c.max_step = 1ll << 62;
  ACK(cudaMemcpyAsync(h->d_ctrl, &c, sizeof(Ctrl), cudaMemcpyHostToDevice, s));
  ACK(box_rate(g, X0, g.ng, h->d_ctrl, s));
  double* cur = X0;
  double* bufs[2] = {A->W0, A->W2};
  int nsrc = 1;
  for (long long k = 0; k < A->nsteps; ++k) {
    double* out = bufs[k & 1];
    StageArgs a{};
    a.ctrl = h->d_ctrl;
    a.geom = h->d_geom;
    a.tiles = h->d_tiles;
    a.ncells_total = g.ng;
    a.nsrc = nsrc;
    if (frozen) {
      k_set_clock<<<1, 1, 0, s>>>(h->d_ctrl, A->dts[k], 1);
    } else {
      ACK(launch_dt(h->d_ctrl, 1, s));
      k_record_dt<<<1, 1, 0, s>>>(h->d_ctrl, A->d_dts, k);
    }
    a.X = cur;
    a.out = A->W1;
    ACK(launch_stage(0, g.pow2 ? 1 : 0, g.threed != 0, a, h->ntiles, s));
    a.Y = A->W1;
    a.out = out;
    ACK(launch_stage(1, g.pow2 ? 1 : 0, g.threed != 0, a, h->ntiles, s));
    if (!frozen) ACK(launch_end(h->d_ctrl, 1, s));
    A->step_nsrc[k] = nsrc;
    nsrc = 2;
    cur = out;
  }
  ACK(cudaEventRecord(e1, s));
  ACK(cudaEventSynchronize(e1));
  float ms = 0.f;
  cudaEventElapsedTime(&ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (!frozen) {
    A->ms_fwd = ms;
    ACK(cudaMemcpy(A->dts.data(), A->d_dts, A->nsteps * sizeof(double), cudaMemcpyDeviceToHost));
  }
  Ctrl hc;
  ACK(cudaMemcpy(&hc, h->d_ctrl, sizeof(Ctrl), cudaMemcpyDeviceToHost));
  if (hc.flags & (kFlagVlimit | kFlagLowRho | kFlagNonFinite))
    return aerr(A, BX_ERR_STATE,
                "a guard fired in the forward run (velocity limiter, low density or non-finite "
                "values); the adjoint of this run is not defined by the fused stages");
  ACK(cudaMemcpyAsync(A->XT, cur, n5 * sizeof(double), cudaMemcpyDeviceToDevice, s));
  // reference cons after the run: one source more, ghosts filled
  PhaseArrays pa = h->pa;
  ACK(fused_to_phase(g, cur, 2, pa, h->nghost, h->d_dst, h->d_src2, h->d_sgn2, s));
  ACK(cudaMemcpyAsync(consT, h->pa.cons, n5 * sizeof(double), cudaMemcpyDeviceToDevice, s));
  ACK(cudaStreamSynchronize(s));
  if (!frozen) A->have_forward = true;
  return BX_OK;
}

// Vector-Jacobian product of the last unfrozen forward run: lamT (adjoint of the
// reference cons after the run, interior cells; 5 x ngrid SoA) -> lam0 (adjoint of
// cons0's interior cells; ghost entries zero).
int bx_adj_backward(bx_adj* A, const double* lamT, double* lam0) {
  if (!A || !lamT || !lam0) return aerr(A, BX_ERR_ARG, "bad arguments");
  if (!A->have_forward) return aerr(A, BX_ERR_STATE, "run bx_adj_forward first");
  bx_handle* h = A->h;
  const Geom& g = h->g;
  cudaStream_t s = h->stream;
  const long long n5 = 5 * g.ng;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  ACK(cudaEventRecord(e0, s));
  A->fwd_steps_in_bwd = 0;
  A->pool_free.clear();
  for (int k = 1; k <= A->snaps; ++k) A->pool_free.push_back(k);
  double* lam = lam0;
  ACK(cudaMemcpyAsync(lam, lamT, n5 * sizeof(double), cudaMemcpyDeviceToDevice, s));
  // the reference cons after the run is src(C2_T): its adjoint first
  k_adj_src_vjp<<<ablk(g.ng), AB, 0, s>>>(g, A->XT, 1, lam);
  if (int r = reverse_range(A, A->pool[0], 0, A->nsteps, lam)) return r;
  ACK(cudaEventRecord(e1, s));
  ACK(cudaEventSynchronize(e1));
  float ms = 0.f;
  cudaEventElapsedTime(&ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  A->ms_bwd = ms;
  return BX_OK;
}

int bx_adj_stats(bx_adj* A, double* ms_forward, double* ms_backward, int64_t* recomputed_steps,
                 int64_t* device_bytes) {
  if (!A) return BX_ERR_ARG;
  if (ms_forward) *ms_forward = A->ms_fwd;
  if (ms_backward) *ms_backward = A->ms_bwd;
  if (recomputed_steps) *recomputed_steps = A->fwd_steps_in_bwd;
  if (device_bytes) *device_bytes = (int64_t)A->bytes;
  return BX_OK;
}

int bx_adj_dts(bx_adj* A, double* dts) {
  if (!A || !dts) return BX_ERR_ARG;
  std::memcpy(dts, A->dts.data(), A->nsteps * sizeof(double));
  return BX_OK;
}

}  // extern "C"

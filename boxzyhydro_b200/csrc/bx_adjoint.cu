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
// The reverse of one stage runs, with two scratch plane sets of 7 (primitives
// P and their adjoints PA) beside the state planes:
//  k_r1_prims  primitives of every cell;
//  k_rdir<d>   for each direction, line segments in shared memory: face states
//              and the HLL derivative of every face once, the MUSCL and slope
//              derivatives, summed into PA (no atomics: each cell of a line
//              belongs to one segment, the directions run one after another);
//  k_rcell     per interior cell: primitives -> conserved variables for the cell
//              and the face ghosts it donates to, then the step combination
//              (and, for stage 0, the sources of the step input).
//
// Snapshots follow a checkpoint schedule over a fixed pool of plane sets (see
// build_schedule), so a run of any length is reversed in bounded memory.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
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
// grid: x threads by (y, z) blocks
__global__ void k_r1_prims(Geom g, int stage, const double* A, const double* B, double* P) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y, z = blockIdx.z;
  if (x >= g.nx) return;
  const long long i = x + (long long)y * g.sy + (long long)z * g.sz;
  const long long n = g.ng;
  const C5 a = aload(A, n, g, x, y, z);
  // the forward's quotients, bit for bit: one exact reciprocal per density
  const SharedDiv qa(a.d);
  const double u1 = qa(a.m1), u2 = qa(a.m2), u3 = qa(a.m3);
  const double e = recon_eps(a.d, a.E, u1, u2, u3, g.small_eps);
  double p;
  if (stage == 0) {
    p = e * g.gm1;
  } else {
    const C5 b = aload(B, n, g, x, y, z);
    const SharedDiv qb(b.d);
    const double s1 = qb(b.m1), s2 = qb(b.m2), s3 = qb(b.m3);
    p = eos_pressure(a.d, a.E, s1, s2, s3, g.gm1, g.small_eps);
  }
  P[i] = a.d;
  P[n + i] = u1;
  P[2 * n + i] = u2;
  P[3 * n + i] = u3;
  P[4 * n + i] = p;
  P[5 * n + i] = e;
  P[6 * n + i] = sqrt(qa(p * g.gam));
}

// ---- conserved-variable VJP at cell (x,y,z) of a stage: gq holds the adjoints
// of the primitives rho, u1, u2, u3, p, eps, c (whose values are in the P planes
// at index pi; a ghost's primitives are its donor's through the donor rule);
// returns the adjoints of A's (gA) and, for stage 1, B's (gB) conserved values
// at that location.  Branches (the eps floors) are taken as the forward took
// them: eps > small_eps exactly when the floor did not fire.
// the values the VJP reads: the cell's primitives, and for stage 1 A's energy
// and B's density and momenta at the location (through the donor rule)
struct CvIn {
  double rho, u[3], p, e, cs, aE, bd, bm[3];
};

__device__ __forceinline__ void cons_vjp_v(const Geom& g, int stage, const CvIn& v,
                                           const double gq[7], double gA[5], double gB[5]) {
  const double rho = v.rho, u[3] = {v.u[0], v.u[1], v.u[2]};
  const double p = v.p, e = v.e, cs = v.cs;
  // reciprocals of the derivative terms (not of values a branch depends on)
  const double ir = rcp_deriv(rho);
  for (int q = 0; q < 5; ++q) gA[q] = gB[q] = 0.0;
  double grho = gq[0], gu[3] = {gq[1], gq[2], gq[3]}, gp = gq[4], ge = gq[5];
  if (cs > 0.0) {
    // c = sqrt(gam p / rho)
    const double h = kHalf * gq[6] * cs;
    gp += h * rcp_deriv(p);
    grho -= h * ir;
  }
  if (stage == 0) {
    ge += gp * g.gm1;
  } else {
    // p = max(E - rho K(u*)/2, eps)(gam-1) with u* = m/rho of B (main.f90:351-355)
    const double us[3] = {v.bm[0] / v.bd, v.bm[1] / v.bd, v.bm[2] / v.bd};
    const double Ks = us[0] * us[0] + us[1] * us[1] + us[2] * us[2];
    if (v.aE - rho * kHalf * Ks > g.small_eps) {
      const double gpg = gp * g.gm1, ib = rcp_deriv(v.bd);
      gA[4] += gpg;
      grho = fma(gpg, -kHalf * Ks, grho);
      for (int j = 0; j < 3; ++j) {
        const double gus = gpg * (-rho * us[j]) * ib;
        gB[1 + j] += gus;
        gB[0] = fma(-gus, us[j], gB[0]);
      }
    }
  }
  if (e > g.small_eps) {
    const double K = u[0] * u[0] + u[1] * u[1] + u[2] * u[2];
    gA[4] += ge;
    grho = fma(ge, -kHalf * K, grho);
    for (int j = 0; j < 3; ++j) gu[j] = fma(ge, -rho * u[j], gu[j]);
  }
  for (int j = 0; j < 3; ++j) {
    const double t = gu[j] * ir;
    gA[1 + j] += t;
    grho = fma(-t, u[j], grho);
  }
  gA[0] += grho;
}

// the same at (x,y,z) with the values read from memory (P at index pi)
__device__ __forceinline__ void cons_vjp(const Geom& g, int stage, const double* P, long long pi,
                                         const double* A, const double* B, int x, int y, int z,
                                         const double gq[7], double gA[5], double gB[5]) {
  const long long n = g.ng;
  CvIn v;
  v.rho = P[pi];
  v.u[0] = P[n + pi]; v.u[1] = P[2 * n + pi]; v.u[2] = P[3 * n + pi];
  v.p = P[4 * n + pi]; v.e = P[5 * n + pi]; v.cs = P[6 * n + pi];
  v.aE = 0.0; v.bd = 1.0; v.bm[0] = v.bm[1] = v.bm[2] = 0.0;
  if (stage == 1) {
    const C5 a = aload(A, n, g, x, y, z);
    const C5 b = aload(B, n, g, x, y, z);
    v.aE = a.E;
    v.bd = b.d; v.bm[0] = b.m1; v.bm[1] = b.m2; v.bm[2] = b.m3;
  }
  cons_vjp_v(g, stage, v, gq, gA, gB);
}

// ---- reverse of the faces of one direction, line by line.
// A line is a row of cells along DIR at interior coordinates in the other
// directions, from the ghost below the interior (lo-1) to the ghost above (hi);
// those are exactly the cells the DIR faces of the stage touch.  A block takes NL
// lines and a segment of W cells [s0, s0+W) of each, with a halo of 3, and in
// shared memory:
//  P1 loads the primitives of [s0-3, s0+W+3);
//  P2 forms the face states (MUSCL, the forward's own arithmetic), slopes and
//     slope selections of [s0-2, s0+W+2);
//  P3 differentiates the HLL flux of each face with high cell in [s0-1, s0+W+1]
//     (flux adjoint coef*(lam_low - lam_high) from the interior cells' adjoints);
//  P4 takes each cell of [s0-1, s0+W] back through its MUSCL states: direct
//     primitive adjoints and the adjoints of its six slopes;
//  P5 gathers, for the cells of the segment, their direct adjoints and the
//     slope adjoints of the (up to three) slopes that read them, and adds the
//     sum to PA (7 planes: rho, u1, u2, u3, p, eps, c).
// Each face's states and HLL derivative are computed once.
// Segment shape: a line of Lc cells is cut into nseg equal segments of W <= wmax
// cells, and a block takes NL = floor(target/(W+4)) lines, so the state, face
// and MUSCL phases (W+4, W+3, W+2 cells per line) each take one pass of the
// block.  x lines: blocks of about 128 threads, four per SM (registers), so the
// barrier-separated phases of different blocks overlap.  y and z lines: 8 lines
// of adjacent x per block (256 threads, two per SM), so every global access of
// a segment cell moves 64 contiguous bytes (measured at 128^3: 6.5 % less
// backward time than 4 lines in 128-thread blocks; 11 or 16 lines with shorter
// segments were slower).
// first x of the y and z lines of the direction kernels (see k_rdir)
__host__ __device__ inline int rdir_x0(const Geom& g) { return g.ax0 & ~3; }

struct RShape {
  int NL, W, NQ, NS, NF, ND, nseg, threads;
  size_t r1, r2, r3, r4, smem;  // region sizes in doubles; smem in bytes
};

static RShape rshape(int Lc, int wmax, int target) {
  RShape r{};
  r.nseg = (Lc + wmax - 1) / wmax;
  r.W = (Lc + r.nseg - 1) / r.nseg;
  r.NQ = r.W + 6; r.NS = r.W + 4; r.NF = r.W + 3; r.ND = r.W + 2;
  r.NL = std::max(1, target / r.NS);
  r.threads = std::min(1024, ((r.NL * r.NS + 31) / 32) * 32);
  r.r1 = (size_t)std::max(7 * r.NQ + 5 * r.NS, 13 * r.ND) * r.NL;
  r.r2 = (size_t)21 * r.NS * r.NL;
  r.r3 = (size_t)12 * r.NF * r.NL;
  r.r4 = (size_t)7 * r.W * r.NL;  // PA of the segment, fetched while the block computes
  r.smem = (r.r1 + r.r2 + r.r3 + r.r4) * sizeof(double) + (size_t)r.NS * r.NL * sizeof(int);
  return r;
}

// asynchronous global -> shared copies (cp.async): the segment's PA values are
// in flight while the block forms states and face derivatives
__device__ __forceinline__ void cp_async8(double* smem, const double* gmem) {
  const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(sa), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

template <int DIR>
__device__ __forceinline__ int rsx(int l, int j, int M, int NL) {
  return DIR == 0 ? l * M + j : j * NL + l;
}

template <int DIR, bool POW2>
__global__ void __launch_bounds__(DIR == 0 ? 128 : 256, DIR == 0 ? 4 : 2)
k_rdir(Geom g, const double* P, const double* lamL, double lscale, double dt, double* PA,
       RShape sh) {
  const int NL = sh.NL, W = sh.W, NQ = sh.NQ, NS = sh.NS, NF = sh.NF, ND = sh.ND;
  extern __shared__ double sm[];
  // d slope(c+o) / d q(c) by the selected argument sq of genminmod (1:
  // theta*(c1-c0), 2: half*(c2-c0), 3: theta*(c2-c1), 0: none): row o+1, column
  // sq; c is the slope's c0 (o = +1), c1 (o = 0) or c2 (o = -1)
  __shared__ double kk_tab[12];
  if (threadIdx.x < 12) {
    const int o = (int)threadIdx.x / 4 - 1, sq = (int)threadIdx.x % 4;
    kk_tab[threadIdx.x] = o == 1 ? (sq == 1 ? -kTheta : (sq == 2 ? -kHalf : 0.0))
                        : o == 0 ? (sq == 1 ? kTheta : (sq == 3 ? -kTheta : 0.0))
                                 : (sq == 2 ? kHalf : (sq == 3 ? kTheta : 0.0));
  }
  double* r1 = sm;
  double* r2 = sm + sh.r1;
  double* r3 = r2 + sh.r2;
  double* pa_s = r3 + sh.r3;  // [7][NL*W]
  int* sel_s = reinterpret_cast<int*>(pa_s + sh.r4);
  double* lm_s = r1 + 7 * NL * NQ;  // lives in r1 beside the primitives until P4
  const long long n = g.ng;
  const int zlo = g.threed ? g.az0 : 0, zhi = g.threed ? g.az1 : g.nz;
  const int nyi = g.ay1 - g.ay0, nzi = zhi - zlo;
  // y and z lines: x from the interior start rounded down to 4 cells (32
  // bytes), so each 8-line group reads whole 32-byte sectors of a row; the
  // lines left of the interior are idle
  const int xs = rdir_x0(g), nxi = g.ax1 - xs;
  const int lo = DIR == 0 ? g.ax0 : DIR == 1 ? g.ay0 : g.az0;
  const int hi = DIR == 0 ? g.ax1 : DIR == 1 ? g.ay1 : g.az1;
  const long long st = DIR == 0 ? 1 : DIR == 1 ? g.sy : g.sz;
  const long long nlines = DIR == 0 ? (long long)nyi * nzi : DIR == 1 ? (long long)nxi * nzi
                                                                       : (long long)nxi * nyi;
  // the segments of a line group are consecutive blocks, so the cells that
  // neighbouring segments both load (their halos) are read while the other
  // segment's block still has them in L2
  const int seg = (int)(blockIdx.x % (unsigned)sh.nseg);
  const long long grp = (long long)(blockIdx.x / (unsigned)sh.nseg);
  const int s0 = lo - 1 + seg * W;
  const double ds = DIR == 0 ? g.dx : DIR == 1 ? g.dy : g.dz;
  const double ids = DIR == 0 ? g.idx : DIR == 1 ? g.idy : g.idz;
  const double area = DIR == 0 ? g.ayz : DIR == 1 ? g.axz : g.axy;
  const double coef = -(dt / g.vol) * area;
  const double rr = dt / ds;
  auto line_base = [&](int l, bool& ok) -> long long {
    const long long L = grp * NL + l;
    ok = L < nlines;
    if (!ok) return 0;
    if (DIR == 0) return (g.ay0 + L % nyi) * g.sy + (zlo + L / nyi) * g.sz;
    const int x = xs + (int)(L % nxi);
    ok = x >= g.ax0;
    if (DIR == 1) return x + (zlo + L / nxi) * g.sz;
    return x + (g.ay0 + L / nxi) * g.sy;
  };
  auto valid = [&](int c) { return c >= lo - 1 && c <= hi; };
  auto inner = [&](int c) { return c >= lo && c < hi; };
  // Each thread keeps one line l of the block and the positions j0, j0 + TPL,
  // ... along it in every phase (x lines: consecutive threads take consecutive
  // cells of a line; y/z lines: consecutive threads take adjacent lines), so the
  // item decomposition and the line's offset are computed once, not per item.
  const int TPL = blockDim.x / NL;
  const int l = DIR == 0 ? (int)threadIdx.x / TPL : (int)threadIdx.x % NL;
  const int j0 = DIR == 0 ? (int)threadIdx.x % TPL : (int)threadIdx.x / NL;
  const bool lane = l < NL;
  bool lok;
  const long long lb = lane ? line_base(l, lok) : 0;
  lok = lok && lane;

  // PA is written, not accumulated, where no earlier direction reached: by the
  // x lines everywhere (they run first and hold every interior cell and the
  // x-face ghosts), by y and z lines at their own face ghosts (lo-1 and hi),
  // which lie on no line of another direction.  So PA needs no clearing.
  auto first = [&](int c) { return DIR == 0 || c == lo - 1 || c == hi; };
  // P0: start fetching PA of the segment's other cells (used in P5)
  if (DIR != 0) {
    for (int j = j0; j < W && lok; j += TPL) {
      const int c = s0 + j;
      if (!valid(c) || first(c)) continue;
      const long long i = lb + c * st;
      const int kp = rsx<DIR>(l, j, W, NL);
      for (int q = 0; q < 7; ++q) cp_async8(pa_s + q * NL * W + kp, PA + q * n + i);
    }
    cp_async_commit();
  }

  // P1: primitives
  for (int j = j0; j < NQ && lane; j += TPL) {
    const int c = s0 - 3 + j;
    const bool ok = lok;
    const int k = rsx<DIR>(l, j, NQ, NL);
    const long long i = lb + c * st;
    if (ok && valid(c)) {
      for (int q = 0; q < 7; ++q) r1[q * NL * NQ + k] = P[q * n + i];
    } else {
      for (int q = 0; q < 7; ++q) r1[q * NL * NQ + k] = 1.0;
    }
    // scaled adjoints of the interior cells of [s0-2, s0+W+2) (zero elsewhere)
    if (j >= 1 && j <= NS) {
      const int kl = rsx<DIR>(l, j - 1, NS, NL);
      const bool in = ok && inner(c);
      for (int q = 0; q < 5; ++q) lm_s[q * NL * NS + kl] = in ? lscale * lamL[q * n + i] : 0.0;
    }
  }
  __syncthreads();
  // P2: face states, slopes, selections
  for (int j = j0; j < NS && lane; j += TPL) {
    const int c = s0 - 2 + j;
    const int k = rsx<DIR>(l, j, NS, NL);
    auto qv = [&](int jj) {
      const int kk = rsx<DIR>(l, jj, NQ, NL);
      return Prim{r1[kk], r1[NL * NQ + kk], r1[2 * NL * NQ + kk], r1[3 * NL * NQ + kk],
                  r1[4 * NL * NQ + kk], r1[5 * NL * NQ + kk], r1[6 * NL * NQ + kk]};
    };
    const Prim qc = qv(j + 1);
    FaceState mi, pl;
    double sl[6] = {0, 0, 0, 0, 0, 0};
    int sel = 0;
    double hm = 0.0, hp = 0.0, flg = 0.0;
    if (inner(c)) {
      const Prim qm = qv(j), qp = qv(j + 2);
      const double a0[6] = {qm.d, qm.u1, qm.u2, qm.u3, qm.p, qm.e};
      const double a1[6] = {qc.d, qc.u1, qc.u2, qc.u3, qc.p, qc.e};
      const double a2[6] = {qp.d, qp.u1, qp.u2, qp.u3, qp.p, qp.e};
#pragma unroll
      for (int q = 0; q < 6; ++q) {
        int sq;
        sl[q] = slope_and_sel(a0[q], a1[q], a2[q], sq);
        sel |= sq << (2 * q);
      }
      const double ud = DIR == 0 ? qc.u1 : DIR == 1 ? qc.u2 : qc.u3;
      muscl_states<POW2>(qc, ud, sl[0], sl[1], sl[2], sl[3], sl[4], sl[5], dt, ds, ids, mi, pl);
      double lp = fmax(ud + qc.c, 0.0) * dt, lm = fmin(ud - qc.c, 0.0) * dt;
      if (POW2) { lp *= ids; lm *= ids; }
      else { lp = cdiv(lp, ds, ids); lm = cdiv(lm, ds, ids); }
      hm = kHalf * (-1.0 - lm);
      hp = kHalf * (1.0 - lp);
      flg = (ud + qc.c > 0.0 ? 1.0 : 0.0) + (ud - qc.c < 0.0 ? 2.0 : 0.0);
    } else {
      ghost_states(qc, mi, pl);
    }
    const int M = NL * NS;
    const double mv[6] = {mi.d, mi.u1, mi.u2, mi.u3, mi.p, mi.e};
    const double pv[6] = {pl.d, pl.u1, pl.u2, pl.u3, pl.p, pl.e};
#pragma unroll
    for (int q = 0; q < 6; ++q) {
      r2[q * M + k] = mv[q];
      r2[(6 + q) * M + k] = pv[q];
      r2[(12 + q) * M + k] = sl[q];
    }
    r2[18 * M + k] = hm;
    r2[19 * M + k] = hp;
    r2[20 * M + k] = flg;
    sel_s[k] = sel;
  }
  __syncthreads();
  // P3: HLL derivative per face (high cell c = s0-1+j)
  for (int j = j0; j < NF && lane; j += TPL) {
    const int c = s0 - 1 + j;
    const bool ok = lok;
    const int k = rsx<DIR>(l, j, NF, NL);
    const int M3 = NL * NF;
    if (!(ok && c >= lo && c <= hi)) {
      for (int q = 0; q < 12; ++q) r3[q * M3 + k] = 0.0;
      continue;
    }
    const int M = NL * NS;
    const int kl = rsx<DIR>(l, j, NS, NL), kr = rsx<DIR>(l, j + 1, NS, NL);
    const FaceState L{r2[6 * M + kl], r2[7 * M + kl], r2[8 * M + kl], r2[9 * M + kl],
                      r2[10 * M + kl], r2[11 * M + kl]};
    const FaceState R{r2[kr], r2[M + kr], r2[2 * M + kr], r2[3 * M + kr], r2[4 * M + kr],
                      r2[5 * M + kr]};
    double gF[5];
#pragma unroll
    for (int q = 0; q < 5; ++q) gF[q] = coef * (lm_s[q * NL * NS + kl] - lm_s[q * NL * NS + kr]);
    FS6 gL, gR;
    hll_vjp<DIR>(L, R, g.gam, gF, gL, gR);
    const double a[12] = {gL.d, gL.u1, gL.u2, gL.u3, gL.p, gL.e,
                          gR.d, gR.u1, gR.u2, gR.u3, gR.p, gR.e};
#pragma unroll
    for (int q = 0; q < 12; ++q) r3[q * M3 + k] = a[q];
  }
  __syncthreads();
  // P4: MUSCL adjoint per cell c = s0-1+j (into r1: DQ planes 0-6, LS planes 7-12)
  for (int j = j0; j < ND && lane; j += TPL) {
    const int c = s0 - 1 + j;
    const int k = rsx<DIR>(l, j, ND, NL);
    const int M1 = NL * ND, M = NL * NS, M3 = NL * NF;
    double lq[7] = {0, 0, 0, 0, 0, 0, 0}, ls[6] = {0, 0, 0, 0, 0, 0};
    if (valid(c)) {
      const int kf0 = rsx<DIR>(l, j, NF, NL), kf1 = rsx<DIR>(l, j + 1, NF, NL);
      double gm[6], gp[6];
#pragma unroll
      for (int q = 0; q < 6; ++q) {
        gm[q] = r3[(6 + q) * M3 + kf0];  // minus state of c: high side of face (c-1, c)
        gp[q] = r3[q * M3 + kf1];        // plus state of c: low side of face (c, c+1)
        lq[q] = gm[q] + gp[q];
      }
      if (inner(c)) {
        const int ks = rsx<DIR>(l, j + 1, NS, NL);
        const double hm = r2[18 * M + ks], hp = r2[19 * M + ks];
        const int flg = (int)r2[20 * M + ks];
        double ghm = 0.0, ghp = 0.0;
#pragma unroll
        for (int q = 0; q < 6; ++q) {
          const double sq = r2[(12 + q) * M + ks];
          ls[q] = hm * gm[q] + hp * gp[q];
          ghm += sq * gm[q];
          ghp += sq * gp[q];
        }
        const double glm = -kHalf * ghm, glp = -kHalf * ghp;
        if (flg & 1) { lq[1 + DIR] += glp * rr; lq[6] += glp * rr; }
        if (flg & 2) { lq[1 + DIR] += glm * rr; lq[6] -= glm * rr; }
      }
    }
#pragma unroll
    for (int q = 0; q < 7; ++q) r1[q * M1 + k] = lq[q];
#pragma unroll
    for (int q = 0; q < 6; ++q) r1[(7 + q) * M1 + k] = ls[q];
  }
  __syncthreads();
  // P5: gather and accumulate
  if (DIR != 0) {
    cp_async_wait_all();
    __syncthreads();
  }
  for (int j = j0; j < W && lok; j += TPL) {
    const int c = s0 + j;
    if (!valid(c)) continue;
    const long long b = lb;
    const int kp = rsx<DIR>(l, j, W, NL);
    const int M1 = NL * ND;
    const int kc = rsx<DIR>(l, j + 1, ND, NL);
    double acc[7];
#pragma unroll
    for (int q = 0; q < 7; ++q) acc[q] = r1[q * M1 + kc];
#pragma unroll
    for (int o = -1; o <= 1; ++o) {
      if (!inner(c + o)) continue;
      const int sel = sel_s[rsx<DIR>(l, j + 2 + o, NS, NL)];
      const int kn = rsx<DIR>(l, j + 1 + o, ND, NL);
#pragma unroll
      for (int q = 0; q < 6; ++q)
        acc[q] += kk_tab[(o + 1) * 4 + ((sel >> (2 * q)) & 3)] * r1[(7 + q) * M1 + kn];
    }
    const long long i = b + c * st;
    if (first(c)) {
#pragma unroll
      for (int q = 0; q < 7; ++q) PA[q * n + i] = acc[q];
    } else {
#pragma unroll
      for (int q = 0; q < 7; ++q) PA[q * n + i] = pa_s[q * NL * W + kp] + acc[q];
    }
  }
}

// ---- per interior cell: conserved adjoints of its own primitives and of the
// face ghosts it donates to (momentum signs of the donor rule), then the step
// combination C2 = (C0' + C1 + L1(C1, C0'))/2, C1 = C0' + L0(C0'):
//  stage 1 (lin = adjoint of C2): o1 <- adjoint of C1 = lin/2 + a_A,
//           o2 <- adjoint of C0' so far = (lin/2 + a_B) + o1;
//  stage 0 (lin = adjoint of C0' so far): o1 <- (lin + a_A) + a_B, then through
//           the nsrc sources of X (source.f90:176-182); ghost entries of o1 zero.
// conserved adjoints of the face ghosts next to interior cell (x,y,z) whose donor
// it is, added to a (kept out of line: only boundary cells take it)
template <int STAGE>
__device__ __noinline__ void ghost_fold(const Geom& g, const double* SA, const double* SB,
                                        const double* P, const double* PA, int x, int y, int z,
                                        long long i, double a[10]) {
  const long long n = g.ng;
  const int ndir = g.threed ? 3 : 2;
  const int lo[3] = {g.ax0, g.ay0, g.az0}, hi[3] = {g.ax1, g.ay1, g.az1};
  const int c[3] = {x, y, z};
  double gq[7], gA[5], gB[5];
  for (int dir = 0; dir < ndir; ++dir) {
    const long long st = dir == 0 ? 1 : dir == 1 ? g.sy : g.sz;
    for (int side = 0; side < 2; ++side) {
      // the face ghost next to this cell (lo-1 or hi), whose donor is this cell
      if (c[dir] != (side == 0 ? lo[dir] : hi[dir] - 1)) continue;
      const int gc = side == 0 ? lo[dir] - 1 : hi[dir];
      const long long gi = i + (long long)(gc - c[dir]) * st;
      const bool flip = g.wall[2 * dir + side] != 0;
      for (int q = 0; q < 7; ++q) gq[q] = PA[q * n + gi];
      int gx = x, gy = y, gz = z;
      if (dir == 0) gx = gc; else if (dir == 1) gy = gc; else gz = gc;
      cons_vjp(g, STAGE, P, gi, SA, SB, gx, gy, gz, gq, gA, gB);
      for (int q = 0; q < 5; ++q) {
        const bool neg = flip && q == 1 + dir;
        a[q] += neg ? -gA[q] : gA[q];
        a[5 + q] += neg ? -gB[q] : gB[q];
      }
    }
  }
}

// grid over interior cells: x threads by (y, z) blocks.  Writes interior entries
// only (the ghost entries of the adjoint planes stay zero).
template <int STAGE>
__global__ void k_rcell(Geom g, const double* SA, const double* SB, const double* P,
                        const double* PA, const double* lin, double* o1, double* o2,
                        const double* X, int nsrc, int xedge) {
  // xedge = 0: the columns between the two x-edge columns (every warp takes the
  // ghost path together or not at all); xedge = 1: the two x-edge columns
  int x, y, z;
  if (xedge) {
    // one thread per x-edge cell: t = side + 2 (y + nyi z)
    const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    const int nyi = g.ay1 - g.ay0, nzi = g.threed ? g.az1 - g.az0 : g.nz;
    if (t >= 2ll * nyi * nzi) return;
    const int side = (int)(t & 1);
    if (side == 1 && g.ax1 - 1 == g.ax0) return;
    x = side ? g.ax1 - 1 : g.ax0;
    y = g.ay0 + (int)((t >> 1) % nyi);
    z = (g.threed ? g.az0 : 0) + (int)((t >> 1) / nyi);
  } else {
    x = g.ax0 + 1 + blockIdx.x * blockDim.x + threadIdx.x;
    if (x >= g.ax1 - 1) return;
    y = g.ay0 + blockIdx.y;
    z = (g.threed ? g.az0 : 0) + blockIdx.z;
  }
  const long long i = x + (long long)y * g.sy + (long long)z * g.sz;
  const long long n = g.ng;
  // every load of the cell first (an interior cell is its own donor)
  double gq[7], a[10], gA[5], gB[5], li[5], xs[5];
  CvIn v;
  for (int q = 0; q < 7; ++q) gq[q] = __ldg(PA + q * n + i);
  v.rho = __ldg(P + i);
  v.u[0] = __ldg(P + n + i); v.u[1] = __ldg(P + 2 * n + i); v.u[2] = __ldg(P + 3 * n + i);
  v.p = __ldg(P + 4 * n + i); v.e = __ldg(P + 5 * n + i); v.cs = __ldg(P + 6 * n + i);
  v.aE = 0.0; v.bd = 1.0; v.bm[0] = v.bm[1] = v.bm[2] = 0.0;
  if (STAGE == 1) {
    v.aE = __ldg(SA + 4 * n + i);
    v.bd = __ldg(SB + i);
    v.bm[0] = __ldg(SB + n + i); v.bm[1] = __ldg(SB + 2 * n + i); v.bm[2] = __ldg(SB + 3 * n + i);
  }
  for (int q = 0; q < 5; ++q) li[q] = __ldg(lin + q * n + i);
  if (STAGE == 0 && nsrc > 0)
    for (int q = 0; q < 5; ++q) xs[q] = __ldg(X + q * n + i);
  cons_vjp_v(g, STAGE, v, gq, gA, gB);
  for (int q = 0; q < 5; ++q) { a[q] = gA[q]; a[5 + q] = gB[q]; }
  const bool edge = x == g.ax0 || x == g.ax1 - 1 || y == g.ay0 || y == g.ay1 - 1 ||
                    (g.threed && (z == g.az0 || z == g.az1 - 1));
  if (edge) {
    // the fold takes its array through memory; only the edge cells pay for that
    double e[10];
    for (int q = 0; q < 10; ++q) e[q] = a[q];
    ghost_fold<STAGE>(g, SA, SB, P, PA, x, y, z, i, e);
    for (int q = 0; q < 10; ++q) a[q] = e[q];
  }
  if constexpr (STAGE == 1) {
    for (int q = 0; q < 5; ++q) {
      const double h = kHalf * li[q];
      const double c1 = h + a[q];
      o1[q * n + i] = c1;
      o2[q * n + i] = (h + a[5 + q]) + c1;
    }
  } else {
    double l[5];
    for (int q = 0; q < 5; ++q) l[q] = (li[q] + a[q]) + a[5 + q];
    if (nsrc > 0) {
      const double d = xs[0], m[3] = {xs[1], xs[2], xs[3]};
      // the energies before each of the (at most two) sources, unrolled so they
      // stay in registers
      const double E0 = xs[4];
      const double E1 = source_energy(d, m[0], m[1], m[2], E0, g.small_eps);
      const double K = kin_mom(d, m[0], m[1], m[2]);
#pragma unroll
      for (int k = 1; k >= 0; --k) {
        // E' = max(E - K, eps) + K
        if (k < nsrc && !((k == 0 ? E0 : E1) - K > g.small_eps)) {
          const double gE = l[4], id = rcp_deriv(d);
          l[4] = 0.0;
          for (int j = 0; j < 3; ++j) l[1 + j] += gE * m[j] * id;
          l[0] += gE * (-K * id);
        }
      }
    }
    for (int q = 0; q < 5; ++q) o1[q * n + i] = l[q];
  }
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
      const double gE = l[4], id = rcp_deriv(d);
      l[4] = 0.0;
      for (int j = 0; j < 3; ++j) l[1 + j] += gE * m[j] * id;
      l[0] += gE * (-K * id);
    }
  }
  for (int q = 0; q < 5; ++q) lam[q * n + i] = l[q];
}

__global__ void k_set_clock(Ctrl* c, double dt, int active) {
  c->dt = dt;
  c->active = active;
}
__global__ void k_record_dt(const Ctrl* c, double* dts, long long k) { dts[k] = c->dt; }

// ---- frozen-branch forward.  A base state and a perturbed state advance
// together through the fused step (dt frozen at the recorded sequence); the
// base values are the stage kernels' own, bit for bit (the same functions in
// the same order; their fast divisions are exact), and every max, min, floor,
// limiter selection and wave-speed choice of the perturbed state is the one the
// base values make, by the reverse kernels' tie rules.  The perturbed run is
// then a smooth function of its input near the base, whose derivative at the
// base is what the adjoint transposes: central differences of it check the
// adjoint where the step itself is not differentiable (ties of the limiter or
// of the wave speeds in flat or symmetric regions).
struct FB {  // one quantity of the base and the perturbed state
  double b, p;
};

// the sources of one cell (source.f90:176-182 with zero force), nsrc times;
// the floor max(E-K, eps) is taken where the base's E-K > eps says
__device__ __forceinline__ void fb_sources(double db, double m1b, double m2b, double m3b,
                                           double& Eb, double dp, double m1p, double m2p,
                                           double m3p, double& Ep, int nsrc, double eps) {
  const double Kb = kin_mom(db, m1b, m2b, m3b), Kp = kin_mom(dp, m1p, m2p, m3p);
  for (int k = 0; k < nsrc; ++k) {
    const bool act = Eb - Kb > eps;
    Eb = fmax(Eb - Kb, eps) + Kb;
    Ep = (act ? Ep - Kp : eps) + Kp;
  }
}

// primitives of an interior cell for both states (load_prim of the stage kernels)
template <int STAGE>
__global__ void k_fb_prims(Geom g, const double* Xb, const double* Xp, const double* Ub,
                           const double* Up, int nsrc, double* Pb, double* Pp, double* Uob,
                           double* Uop) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= g.ng) return;
  int x, y, z;
  decode(g, i, x, y, z);
  if (!ainterior(g, x, y, z)) return;
  const long long n = g.ng;
  double db = Xb[i], m1b = Xb[n + i], m2b = Xb[2 * n + i], m3b = Xb[3 * n + i], Eb = Xb[4 * n + i];
  double dp = Xp[i], m1p = Xp[n + i], m2p = Xp[2 * n + i], m3p = Xp[3 * n + i], Ep = Xp[4 * n + i];
  if (STAGE == 0) fb_sources(db, m1b, m2b, m3b, Eb, dp, m1p, m2p, m3p, Ep, nsrc, g.small_eps);
  const double u1b = m1b / db, u2b = m2b / db, u3b = m3b / db;
  const double u1p = m1p / dp, u2p = m2p / dp, u3p = m3p / dp;
  // eps = max(E - rho K/2, small_eps), floor where the base's says
  const double teb = Eb - kHalf * db * (u1b * u1b + u2b * u2b + u3b * u3b);
  const double eb = fmax(teb, g.small_eps);
  const double ep = teb > g.small_eps ? Ep - kHalf * dp * (u1p * u1p + u2p * u2p + u3p * u3p)
                                      : g.small_eps;
  double pb, pp;
  if (STAGE == 0) {
    pb = eb * g.gm1;
    pp = ep * g.gm1;
  } else {
    // state() with the stage-0 velocity (stored by stage 0 of the pair)
    const double s1b = Ub[i], s2b = Ub[n + i], s3b = Ub[2 * n + i];
    const double s1p = Up[i], s2p = Up[n + i], s3p = Up[2 * n + i];
    const double tpb = Eb - kin_rho_u(db, s1b, s2b, s3b);
    pb = fmax(tpb, g.small_eps) * g.gm1;
    pp = (tpb > g.small_eps ? Ep - kin_rho_u(dp, s1p, s2p, s3p) : g.small_eps) * g.gm1;
  }
  const double qb[7] = {db, u1b, u2b, u3b, pb, eb, sqrt(pb * g.gam / db)};
  const double qp[7] = {dp, u1p, u2p, u3p, pp, ep, sqrt(pp * g.gam / dp)};
  for (int q = 0; q < 7; ++q) {
    Pb[q * n + i] = qb[q];
    Pp[q * n + i] = qp[q];
  }
  if (STAGE == 0) {
    Uob[i] = u1b; Uob[n + i] = u2b; Uob[2 * n + i] = u3b;
    Uop[i] = u1p; Uop[n + i] = u2p; Uop[2 * n + i] = u3p;
  }
}

// primitives of both states at (x,y,z) through the donor rule
__device__ __forceinline__ void fb_prim(const Geom& g, const double* Pb, const double* Pp, int x,
                                        int y, int z, Prim& qb, Prim& qp) {
  long long c;
  unsigned sg;
  bool fx = false, fy = false, fz = false;
  const int xx = amap(x, g.ax0, g.ax1, g.wall[0], g.wall[1], fx);
  const int yy = amap(y, g.ay0, g.ay1, g.wall[2], g.wall[3], fy);
  const int zz = g.threed ? amap(z, g.az0, g.az1, g.wall[4], g.wall[5], fz) : z;
  c = xx + (long long)yy * g.sy + (long long)zz * g.sz;
  sg = (fx ? 1u : 0u) | (fy ? 2u : 0u) | (fz ? 4u : 0u);
  const long long n = g.ng;
  qb = Prim{Pb[c], Pb[n + c], Pb[2 * n + c], Pb[3 * n + c], Pb[4 * n + c], Pb[5 * n + c],
            Pb[6 * n + c]};
  qp = Prim{Pp[c], Pp[n + c], Pp[2 * n + c], Pp[3 * n + c], Pp[4 * n + c], Pp[5 * n + c],
            Pp[6 * n + c]};
  if (sg & 1) { qb.u1 = -qb.u1; qp.u1 = -qp.u1; }
  if (sg & 2) { qb.u2 = -qb.u2; qp.u2 = -qp.u2; }
  if (sg & 4) { qb.u3 = -qb.u3; qp.u3 = -qp.u3; }
}

// the perturbed slope with the base's selection (slope_and_sel's rule)
__device__ __forceinline__ double fb_slope(double c0b, double c1b, double c2b, double c0p,
                                           double c1p, double c2p) {
  int sel;
  slope_and_sel(c0b, c1b, c2b, sel);
  if (sel == 1) return kTheta * (c1p - c0p);
  if (sel == 2) return kHalf * (c2p - c0p);
  if (sel == 3) return kTheta * (c2p - c1p);
  return 0.0;
}

// minus and plus states of the middle cell along DIR for both states
template <int DIR>
__device__ __forceinline__ void fb_dir_states(const Geom& g, const Prim* mb, const Prim* mp,
                                              double dt, FaceState& mib, FaceState& plb,
                                              FaceState& mip, FaceState& plp) {
  const double ds = DIR == 0 ? g.dx : DIR == 1 ? g.dy : g.dz;
  const double ids = DIR == 0 ? g.idx : DIR == 1 ? g.idy : g.idz;
  const Prim &a = mb[0], &c = mb[1], &e = mb[2];
  const double udb = DIR == 0 ? c.u1 : DIR == 1 ? c.u2 : c.u3;
  // the base as the stage kernels' face states (dir_states; cdiv is exact,
  // and equals the multiplication by the reciprocal for power-of-two spacings)
  muscl_states<false>(c, udb, slope3(a.d, c.d, e.d), slope3(a.u1, c.u1, e.u1),
                      slope3(a.u2, c.u2, e.u2), slope3(a.u3, c.u3, e.u3), slope3(a.p, c.p, e.p),
                      slope3(a.e, c.e, e.e), dt, ds, ids, mib, plb);
  const Prim &ap = mp[0], &cp = mp[1], &ep = mp[2];
  const double udp = DIR == 0 ? cp.u1 : DIR == 1 ? cp.u2 : cp.u3;
  const double sd = fb_slope(a.d, c.d, e.d, ap.d, cp.d, ep.d);
  const double s1 = fb_slope(a.u1, c.u1, e.u1, ap.u1, cp.u1, ep.u1);
  const double s2 = fb_slope(a.u2, c.u2, e.u2, ap.u2, cp.u2, ep.u2);
  const double s3 = fb_slope(a.u3, c.u3, e.u3, ap.u3, cp.u3, ep.u3);
  const double sp = fb_slope(a.p, c.p, e.p, ap.p, cp.p, ep.p);
  const double se = fb_slope(a.e, c.e, e.e, ap.e, cp.e, ep.e);
  // lambdas: max(u+c, 0) and min(u-c, 0) where the base's u+c > 0 and u-c < 0 say
  const double lp = (udb + c.c > 0.0 ? udp + cp.c : 0.0) * dt / ds;
  const double lm = (udb - c.c < 0.0 ? udp - cp.c : 0.0) * dt / ds;
  const double hm = kHalf * (-1.0 - lm), hp = kHalf * (1.0 - lp);
  mip = FaceState{cp.d + hm * sd, cp.u1 + hm * s1, cp.u2 + hm * s2, cp.u3 + hm * s3,
                  cp.p + hm * sp, cp.e + hm * se};
  plp = FaceState{cp.d + hp * sd, cp.u1 + hp * s1, cp.u2 + hp * s2, cp.u3 + hp * s3,
                  cp.p + hp * sp, cp.e + hp * se};
}

// HLL flux of both states; the perturbed wave speeds take the base's choice
// (hll_vjp's rule)
template <int DIR>
__device__ __forceinline__ void fb_hll(const FaceState& Lb, const FaceState& Rb,
                                       const FaceState& Lp, const FaceState& Rp, double gam,
                                       double Fb[5], double Fp[5]) {
  hll_flux<DIR>(Lb, Rb, gam, Fb);
  const double vlb = DIR == 0 ? Lb.u1 : DIR == 1 ? Lb.u2 : Lb.u3;
  const double vrb = DIR == 0 ? Rb.u1 : DIR == 1 ? Rb.u2 : Rb.u3;
  const double crb = sqrt(gam * Rb.p / Rb.d), clb = sqrt(gam * Lb.p / Lb.d);
  const double a1 = vrb + crb, a2 = vlb + clb, b1 = -(vrb - crb), b2 = -(vlb - clb);
  const int sap = (a2 > fmax(0.0, a1)) ? 2 : (a1 > 0.0 ? 1 : 0);
  const int sam = (b2 > fmax(0.0, b1)) ? 2 : (b1 > 0.0 ? 1 : 0);
  const double vl = DIR == 0 ? Lp.u1 : DIR == 1 ? Lp.u2 : Lp.u3;
  const double vr = DIR == 0 ? Rp.u1 : DIR == 1 ? Rp.u2 : Rp.u3;
  const double cr = sqrt(gam * Rp.p / Rp.d), cl = sqrt(gam * Lp.p / Lp.d);
  const double ap = sap == 1 ? vr + cr : (sap == 2 ? vl + cl : 0.0);
  const double am = sam == 1 ? -(vr - cr) : (sam == 2 ? -(vl - cl) : 0.0);
  const double sl[5] = {Lp.d, Lp.d * Lp.u1, Lp.d * Lp.u2, Lp.d * Lp.u3,
                        Lp.e + kHalf * Lp.d * (Lp.u1 * Lp.u1 + Lp.u2 * Lp.u2 + Lp.u3 * Lp.u3)};
  const double sr[5] = {Rp.d, Rp.d * Rp.u1, Rp.d * Rp.u2, Rp.d * Rp.u3,
                        Rp.e + kHalf * Rp.d * (Rp.u1 * Rp.u1 + Rp.u2 * Rp.u2 + Rp.u3 * Rp.u3)};
  double fl[5], fr[5];
  for (int k = 0; k < 5; ++k) {
    fl[k] = sl[k] * vl;
    fr[k] = sr[k] * vr;
  }
  fl[1 + DIR] += Lp.p;
  fr[1 + DIR] += Rp.p;
  fl[4] = (sl[4] + Lp.p) * vl;
  fr[4] = (sr[4] + Rp.p) * vr;
  for (int k = 0; k < 5; ++k) Fp[k] = (ap * fl[k] + am * fr[k] - ap * am * (sr[k] - sl[k])) / (ap + am);
}

// the flux of both states through the face between cells lo and lo+1 along DIR
// (lo given by its coordinates); a cell outside the interior along DIR takes
// ghost states (no slopes, flux.f90:53-54)
template <int DIR>
__device__ __forceinline__ void fb_face(const Geom& g, const double* Pb, const double* Pp,
                                        int x, int y, int z, double dt, double Fb[5],
                                        double Fp[5]) {
  const int ex = DIR == 0, ey = DIR == 1, ez = DIR == 2;
  FaceState Lb, Lp, Rb, Rp, t0, t1;
  Prim mb[3], mp[3];
  auto outside = [&](int cx, int cy, int cz) {
    const int c = DIR == 0 ? cx : DIR == 1 ? cy : cz;
    const int a0 = DIR == 0 ? g.ax0 : DIR == 1 ? g.ay0 : g.az0;
    const int a1 = DIR == 0 ? g.ax1 : DIR == 1 ? g.ay1 : g.az1;
    return c < a0 || c >= a1;
  };
  // plus state of the low cell
  for (int k = 0; k < 3; ++k)
    fb_prim(g, Pb, Pp, x + (k - 1) * ex, y + (k - 1) * ey, z + (k - 1) * ez, mb[k], mp[k]);
  if (outside(x, y, z)) {
    ghost_states(mb[1], t0, Lb);
    ghost_states(mp[1], t1, Lp);
  } else {
    fb_dir_states<DIR>(g, mb, mp, dt, t0, Lb, t1, Lp);
  }
  // minus state of the high cell
  const int hx = x + ex, hy = y + ey, hz = z + ez;
  for (int k = 0; k < 3; ++k)
    fb_prim(g, Pb, Pp, hx + (k - 1) * ex, hy + (k - 1) * ey, hz + (k - 1) * ez, mb[k], mp[k]);
  if (outside(hx, hy, hz)) {
    ghost_states(mb[1], Rb, t0);
    ghost_states(mp[1], Rp, t1);
  } else {
    fb_dir_states<DIR>(g, mb, mp, dt, Rb, t0, Rp, t1);
  }
  fb_hll<DIR>(Lb, Rb, Lp, Rp, g.gam, Fb, Fp);
}

// the conservative update of an interior cell for both states (the epilogue of
// the stage kernels: C1 = C0' + L(C0') or C2 = (C0' + C1 + L(C1))/2, floors)
template <int STAGE>
__global__ void k_fb_update(Geom g, const double* Pb, const double* Pp, const double* Xb,
                            const double* Xp, const double* Yb, const double* Yp, int nsrc,
                            double dt, double* Ob, double* Op) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= g.ng) return;
  int x, y, z;
  decode(g, i, x, y, z);
  if (!ainterior(g, x, y, z)) return;
  const long long n = g.ng;
  double hb[5], hp[5], lb[5], lp[5], sb[5], sp[5];
  fb_face<0>(g, Pb, Pp, x - 1, y, z, dt, lb, lp);
  fb_face<0>(g, Pb, Pp, x, y, z, dt, hb, hp);
  for (int q = 0; q < 5; ++q) { sb[q] = g.ayz * (hb[q] - lb[q]); sp[q] = g.ayz * (hp[q] - lp[q]); }
  fb_face<1>(g, Pb, Pp, x, y - 1, z, dt, lb, lp);
  fb_face<1>(g, Pb, Pp, x, y, z, dt, hb, hp);
  for (int q = 0; q < 5; ++q) {
    sb[q] = sb[q] + g.axz * (hb[q] - lb[q]);
    sp[q] = sp[q] + g.axz * (hp[q] - lp[q]);
  }
  if (g.threed) {
    fb_face<2>(g, Pb, Pp, x, y, z - 1, dt, lb, lp);
    fb_face<2>(g, Pb, Pp, x, y, z, dt, hb, hp);
    for (int q = 0; q < 5; ++q) {
      sb[q] = sb[q] + g.axy * (hb[q] - lb[q]);
      sp[q] = sp[q] + g.axy * (hp[q] - lp[q]);
    }
  }
  double cb[5], cp[5], nb[5], np[5];
  for (int q = 0; q < 5; ++q) { cb[q] = Xb[q * n + i]; cp[q] = Xp[q * n + i]; }
  fb_sources(cb[0], cb[1], cb[2], cb[3], cb[4], cp[0], cp[1], cp[2], cp[3], cp[4], nsrc,
             g.small_eps);
  for (int q = 0; q < 5; ++q) {
    const double fb = (-sb[q] * dt) / g.vol, fp = (-sp[q] * dt) / g.vol;
    if (STAGE == 0) {
      nb[q] = cb[q] + fb;
      np[q] = cp[q] + fp;
    } else {
      nb[q] = kHalf * (cb[q] + Yb[q * n + i] + fb);
      np[q] = kHalf * (cp[q] + Yp[q * n + i] + fp);
    }
  }
  // floors (flux.f90:223-230) where the base's values put them
  const bool dfl = !(nb[0] >= g.small_rho), efl = nb[4] < 0.0;
  floors(nb[0], nb[1], nb[2], nb[3], nb[4], g.small_rho, g.small_eps);
  if (dfl) np[0] = g.small_rho;
  if (efl) np[4] = kin_mom(np[0], np[1], np[2], np[3]) + g.small_eps;
  for (int q = 0; q < 5; ++q) {
    Ob[q * n + i] = nb[q];
    Op[q * n + i] = np[q];
  }
}

// reference cons of interior cells at the end of the run: the planes plus the
// source still pending (k_f2p_interior with nsrc 2), for both states
__global__ void k_fb_finish(Geom g, const double* Xb, const double* Xp, double* Ob, double* Op) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= g.ng) return;
  int x, y, z;
  decode(g, i, x, y, z);
  const long long n = g.ng;
  if (!ainterior(g, x, y, z)) {
    for (int q = 0; q < 5; ++q) Ob[q * n + i] = Op[q * n + i] = 0.0;
    return;
  }
  double cb[5], cp[5];
  for (int q = 0; q < 5; ++q) { cb[q] = Xb[q * n + i]; cp[q] = Xp[q * n + i]; }
  fb_sources(cb[0], cb[1], cb[2], cb[3], cb[4], cp[0], cp[1], cp[2], cp[3], cp[4], 1,
             g.small_eps);
  for (int q = 0; q < 5; ++q) {
    Ob[q * n + i] = cb[q];
    Op[q * n + i] = cp[q];
  }
}

}  // namespace

// ------------------------------------------------------------------ host engine
// Checkpoint schedule.  Reversing l steps from a held state with s free
// snapshot slots costs C(l, s) recomputed steps; splitting at m (advance m steps,
// store, reverse the last l-m with s-1 slots, then the first m with s):
//   C(l, s) = min_m  m + C(l-m, s-1) + C(m, s),   C(l, 0) = l(l-1)/2,  C(1, s) = 0.
// The snapshots of the first chain of splits are stored by the forward run
// itself, so their advances cost nothing:
//   F(l, s) = min_m  F(l-m, s-1) + C(m, s),   F(l, 0) = C(l, 0).
// Solved by dynamic programming when l^2 s is small enough; otherwise by the
// closed-form split rules of split_of, which reach the same optimum.
struct Schedule {
  long long L = 0;
  int S = 0;
  bool dp = false;
  std::vector<long long> C, F;
  std::vector<int> mc, mf;
  size_t at(long long l, int s) const { return (size_t)l * (S + 1) + s; }
};

static void build_schedule(Schedule& sc, long long L, int S) {
  sc.L = L;
  sc.S = S;
  sc.dp = (double)L * (double)L * (double)S <= 4e8;
  if (!sc.dp) return;
  const size_t N = (size_t)(L + 1) * (S + 1);
  sc.C.assign(N, 0);
  sc.F.assign(N, 0);
  sc.mc.assign(N, 1);
  sc.mf.assign(N, 1);
  for (int s = 0; s <= S; ++s) {
    for (long long l = 2; l <= L; ++l) {
      const size_t k = sc.at(l, s);
      if (s == 0) {
        sc.C[k] = sc.F[k] = l * (l - 1) / 2;
        continue;
      }
      if (s >= l - 1) {
        sc.C[k] = l - 1;
        sc.F[k] = 0;
        sc.mc[k] = sc.mf[k] = 1;
        continue;
      }
      long long bc = -1, bf = -1;
      int mc = 1, mf = 1;
      for (long long m = 1; m < l; ++m) {
        const long long right_c = sc.C[sc.at(l - m, s - 1)], left = sc.C[sc.at(m, s)];
        const long long vc = m + right_c + left;
        const long long vf = sc.F[sc.at(l - m, s - 1)] + left;
        if (bc < 0 || vc < bc) { bc = vc; mc = (int)m; }
        if (bf < 0 || vf <= bf) { bf = vf; mf = (int)m; }
      }
      sc.C[k] = bc;
      sc.F[k] = bf;
      sc.mc[k] = mc;
      sc.mf[k] = mf;
    }
  }
}

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
  // checkpoint schedule: splits of the recursion, and the chain of snapshots
  // the unfrozen forward stores on its way (pool slot 1 + j holds chain[j])
  Schedule sched;
  std::vector<long long> chain;
  std::vector<int> chain_slot_of;  // per step index: pool slot holding it, or -1
  bool chain_valid = false;
  int chain_left = 0;
  // optional: the stage-0 result C1 of every step, kept by the unfrozen forward
  // so the backward skips its recomputation (nsteps state sets)
  double* c1pool = nullptr;
  bool c1_valid = false;
  // stage-0 results left by the last step of recent advances, tagged with
  // their step (-1: empty): the reverse of that step then skips its stage-0
  // recompute.  At least two entries, so an advance to state k can leave C1 of
  // step k-1 while the entry of step k, needed first, stays
  // (bx_adj_stage0_cache sets the count).
  std::vector<double*> c1c;
  std::vector<long long> c1tag;
  long long c1_hits = 0;
  long long rev_done = 0;  // last reversed step (steps are reversed downwards)
  // work planes
  double *W0 = nullptr, *W1 = nullptr, *W2 = nullptr;  // C0', C1, scratch state
  double* XT = nullptr;  // state after the last step of the forward run (C2_T)
  double *lamA = nullptr, *lamB = nullptr, *lamC1 = nullptr;
  // primitives and their adjoints (7 planes each); forward steps use the first
  // 3 planes of P for the stage-0 velocity
  double *P = nullptr, *PA = nullptr;
  // optional host level of the schedule (bx_adj_host_level): the unfrozen
  // forward copies the state of every hstride-th step into pinned host memory,
  // and the backward reverses the segments between those steps one after
  // another, last first, each with the device pool.  Pool slots snaps and
  // snaps-1 hold segment starts: segment j's start in hold[j & 1] while the
  // start of segment j-1 is copied into the other from the host.
  long long hstride = 0;
  std::vector<double*> hsnap;  // hsnap[j-1]: state of step j*hstride
  size_t host_bytes = 0;
  double* hold[2] = {nullptr, nullptr};
  long long hold_step[2] = {-1, -1};  // step whose state hold[b] holds
  cudaStream_t cstream = nullptr;     // host <-> device copies of the host level
  cudaEvent_t cev[2] = {nullptr, nullptr};  // last copy into or out of hold[b] done
  cudaEvent_t uev[2] = {nullptr, nullptr};  // the compute stream's use of hold[b] done
  bool host_valid = false;
  double ms_fwd = 0.0, ms_bwd = 0.0;
  long long fwd_steps_in_bwd = 0;
  size_t bytes = 0;
  bool have_forward = false;
  // the grid's two-sweep ghost plan leaves corner ghosts lagging (reflective
  // 3-D boxes): they enter only the Courant maximum, so the fused stage
  // arithmetic holds with the dt sequence of the per-phase kernels, which an
  // unfrozen forward takes from a run of those first
  bool dt_phase = false;
  int nsrc0 = 1;
  std::string err;
};

// the message of the calling thread's last failed call made without a handle
static thread_local std::string g_adj_err;

// two timing events, destroyed when the scope ends (on the error returns too)
struct EventPair {
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  EventPair() {
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
  }
  ~EventPair() {
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
  }
  EventPair(const EventPair&) = delete;
  EventPair& operator=(const EventPair&) = delete;
};

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
// with the stage-0 result in c1out, or in W1 when c1out is null.
static int fwd_step(bx_adj* A, const double* X, int nsrc, double dt, double* Y,
                    bool stage0_only = false, double* c1out = nullptr) {
  bx_handle* h = A->h;
  StageArgs a{};
  a.ctrl = h->d_ctrl;
  a.geom = h->d_geom;
  a.tiles = h->d_tiles;
  a.ncells_total = h->g.ng;
  a.nsrc = nsrc;
  a.U = A->P;  // the primitives are rebuilt by every reverse stage
  k_set_clock<<<1, 1, 0, h->stream>>>(h->d_ctrl, dt, 1);
  a.X = X;
  a.Y = nullptr;
  a.out = c1out ? c1out : A->W1;
  ACK(launch_stage(0, h->g.pow2 ? 1 : 0, h->g.threed != 0, a, h->ntiles, h->stream));
  if (stage0_only) return BX_OK;
  a.Y = a.out;
  a.out = Y;
  ACK(launch_stage(1, h->g.pow2 ? 1 : 0, h->g.threed != 0, a, h->ntiles, h->stream));
  return BX_OK;
}

template <int DIR, bool POW2>
static cudaError_t launch_rdir(const Geom& g, const double* P, const double* lamL, double lscale,
                               double dt, double* PA, cudaStream_t s) {
  const long long nzi = g.threed ? g.az1 - g.az0 : g.nz;
  const long long nxi = g.ax1 - rdir_x0(g), nyi = g.ay1 - g.ay0;
  const long long nlines = DIR == 0 ? nyi * nzi : DIR == 1 ? nxi * nzi : nxi * nyi;
  const int lo = DIR == 0 ? g.ax0 : DIR == 1 ? g.ay0 : g.az0;
  const int hi = DIR == 0 ? g.ax1 : DIR == 1 ? g.ay1 : g.az1;
  // x lines run along contiguous memory: long segments; y/z lines: 8 lines of
  // adjacent x per block (coalesced), short segments
  const RShape sh = DIR == 0 ? rshape(hi - lo + 2, 60, 128) : rshape(hi - lo + 2, 28, 256);
  cudaError_t e = ensure_dyn_smem((const void*)k_rdir<DIR, POW2>, sh.smem);
  if (e != cudaSuccess) return e;
  const long long ngrp = (nlines + sh.NL - 1) / sh.NL;
  const dim3 grid((unsigned)(ngrp * sh.nseg));
  k_rdir<DIR, POW2><<<grid, sh.threads, sh.smem, s>>>(g, P, lamL, lscale, dt, PA, sh);
  return cudaGetLastError();
}

template <int DIR>
static cudaError_t launch_rdir(const Geom& g, const double* P, const double* lamL, double lscale,
                               double dt, double* PA, cudaStream_t s) {
  return g.pow2 ? launch_rdir<DIR, true>(g, P, lamL, lscale, dt, PA, s)
                : launch_rdir<DIR, false>(g, P, lamL, lscale, dt, PA, s);
}

// reverse of one stage: lamL*lscale = adjoint of the flux-operator output on
// interior cells; k_rcell combines the result with the step's other terms
static int rev_stage(bx_adj* A, int stage, const double* SA, const double* SB, const double* lamL,
                     double lscale, double dt, const double* lin, double* o1, double* o2,
                     const double* X, int nsrc) {
  bx_handle* h = A->h;
  const Geom& g = h->g;
  cudaStream_t s = h->stream;
  // primitives of every cell: one block row per (y, z)
  const int tp = std::min(512, ((g.nx + 31) / 32) * 32);
  const dim3 pgrid((unsigned)((g.nx + tp - 1) / tp), (unsigned)g.ny, (unsigned)g.nz);
  k_r1_prims<<<pgrid, tp, 0, s>>>(g, stage, SA, SB, A->P);
  // interior cells
  const int nxm = std::max(1, g.ax1 - g.ax0 - 2), tc = std::min(256, ((nxm + 31) / 32) * 32);
  const dim3 cgrid((unsigned)((nxm + tc - 1) / tc), (unsigned)(g.ay1 - g.ay0),
                   (unsigned)(g.threed ? g.az1 - g.az0 : g.nz));
  const long long nedge = 2ll * cgrid.y * cgrid.z;
  const dim3 egrid((unsigned)((nedge + 127) / 128));
  ACK(launch_rdir<0>(g, A->P, lamL, lscale, dt, A->PA, s));
  ACK(launch_rdir<1>(g, A->P, lamL, lscale, dt, A->PA, s));
  if (g.threed) ACK(launch_rdir<2>(g, A->P, lamL, lscale, dt, A->PA, s));
  if (stage == 1) {
    k_rcell<1><<<cgrid, tc, 0, s>>>(g, SA, SB, A->P, A->PA, lin, o1, o2, X, nsrc, 0);
    k_rcell<1><<<egrid, 128, 0, s>>>(g, SA, SB, A->P, A->PA, lin, o1, o2, X, nsrc, 1);
  } else {
    k_rcell<0><<<cgrid, tc, 0, s>>>(g, SA, SB, A->P, A->PA, lin, o1, o2, X, nsrc, 0);
    k_rcell<0><<<egrid, 128, 0, s>>>(g, SA, SB, A->P, A->PA, lin, o1, o2, X, nsrc, 1);
  }
  ACK(cudaGetLastError());
  return BX_OK;
}

// lam (adjoint of the step output, C2) -> lam (adjoint of the step input X)
static int rev_step(bx_adj* A, const double* X, long long k, double* lam) {
  bx_handle* h = A->h;
  const Geom& g = h->g;
  cudaStream_t s = h->stream;
  const int nsrc = A->step_nsrc[k];
  const double dt = A->dts[k];
  // C0' and C1 of step k (C1 kept by the forward run, or recomputed)
  k_adj_src<<<ablk(g.ng), AB, 0, s>>>(g, X, nsrc, A->W0);
  const double* C1 = A->W1;
  if (A->c1pool && A->c1_valid) {
    C1 = A->c1pool + k * 5 * g.ng;
  } else if (std::find(A->c1tag.begin(), A->c1tag.end(), k) != A->c1tag.end()) {
    C1 = A->c1c[std::find(A->c1tag.begin(), A->c1tag.end(), k) - A->c1tag.begin()];
    A->c1_hits += 1;
  } else {
    if (int r = fwd_step(A, X, nsrc, dt, nullptr, true)) return r;  // W1 <- C1
  }
  A->rev_done = k;
  // stage 1 reads lam/2; writes lamC1 (adjoint of C1) and lamA (of C0')
  if (int r = rev_stage(A, 1, C1, A->W0, lam, kHalf, dt, lam, A->lamC1, A->lamA, X, nsrc))
    return r;
  // stage 0 reads lamC1; lam <- adjoint of X through the sources
  if (int r = rev_stage(A, 0, A->W0, A->W0, A->lamC1, 1.0, dt, A->lamA, lam, nullptr, X, nsrc))
    return r;
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

// binomial coefficient (n over k), saturating at 2^50 (far above any step count)
static long long binom(long long n, long long k) {
  if (k < 0 || k > n) return 0;
  k = std::min(k, n - k);
  const long long cap = 1ll << 50;
  long long r = 1;
  for (long long i = 1; i <= k; ++i) {
    // r = (n-k+i over i) after this line: the division is exact
    const __int128 v = (__int128)r * (n - k + i) / i;
    if (v > cap) return cap;
    r = (long long)v;
  }
  return r;
}

// beta(c, r) = (c + r over c): the most steps c checkpoints reverse with r
// repetitions (Griewank 1992, "Achieving logarithmic growth of temporal and
// spatial complexity in reverse automatic differentiation"); 0 for r < 0
static long long beta(long long c, long long r) { return r < 0 ? 0 : binom(c + r, c); }

// First split m (1 <= m < l) of reversing l steps with s >= 1 free slots.
// Beyond the dynamic programme's table the split follows closed-form rules with
// the same optimum.  C (repeated reversal): with c = s + 1 checkpoints (the held
// state and the free slots) and r the smallest repetition number with
// beta(c, r) >= l, C(l, s) = r l - beta(c + 1, r - 1), and a split is optimal when
//   max(beta(c, r-2), l - beta(c-1, r)) <= m <= min(beta(c, r-1), l - beta(c-1, r-1)).
// F (the chain the forward run stores): the chain spreads l steps over segments
// reversed with s, s-1, ..., 0 free slots, each costing C, which is convex in the
// segment length with slope r.  A segment with k slots holds up to beta(k+1, lam)
// steps at marginal cost <= lam, all of them together beta(s+1, lam+1) - 1; with
// the smallest lam that holds l, the first segment takes
//   m = max(beta(s+1, lam-1), l - beta(s, lam+1) + 1).
static long long split_of(const Schedule& sc, bool chain, long long l, int s) {
  if (sc.dp && l <= sc.L && s <= sc.S) return chain ? sc.mf[sc.at(l, s)] : sc.mc[sc.at(l, s)];
  if (s >= l - 1) return 1;
  long long m;
  if (chain) {
    long long lam = 0;
    while (beta(s + 1, lam + 1) - 1 < l) ++lam;
    m = std::max(beta(s + 1, lam - 1), l - beta(s, lam + 1) + 1);
  } else {
    const long long c = s + 1;
    long long r = 0;
    while (beta(c, r) < l) ++r;
    m = std::max(beta(c, r - 2), l - beta(c - 1, r));
  }
  return std::min(std::max(m, 1ll), l - 1);
}

// the chain of snapshots the unfrozen forward run stores: the step index of each
// split of the first chain of the recursion
static std::vector<long long> chain_of(const Schedule& sc, long long nsteps, int snaps) {
  std::vector<long long> chain;
  long long a = 0, l = nsteps;
  for (int sl = snaps; l > 1 && sl > 0; --sl) {
    const long long m = split_of(sc, true, l, sl);
    a += m;
    l -= m;
    chain.push_back(a);
  }
  return chain;
}

// Recomputed steps of reverse_range over l steps, counted on the host: the same
// walk with the free-slot and chain counters in place of the plane sets.
static long long plan_range(const Schedule& sc, long long l, bool chain, int& free_slots,
                            int& chain_left) {
  if (l <= 1) return 0;
  const int s = free_slots + (chain ? chain_left : 0);
  if (s == 0) return l * (l - 1) / 2;
  const long long m = split_of(sc, chain, l, s);
  long long n = 0;
  if (chain) {
    chain_left -= 1;
  } else {
    free_slots -= 1;
    n += m;
  }
  n += plan_range(sc, l - m, chain, free_slots, chain_left);
  free_slots += 1;
  return n + plan_range(sc, m, false, free_slots, chain_left);
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
    double* c1out = nullptr;
    if (k == to - 1 && !A->c1pool && !A->c1c.empty()) {
      // keep C1 of step to-1 (reversed soon after step `to` when no further
      // split comes between them) in an entry that is free or already used;
      // else in the one of the step reversed last, never in step `to`'s
      auto dead = [&](long long t) { return t < 0 || t >= A->rev_done; };
      int j = -1;
      for (int e = 0; e < (int)A->c1tag.size() && j < 0; ++e)
        if (A->c1tag[e] != to && dead(A->c1tag[e])) j = e;
      for (int e = 0; e < (int)A->c1tag.size() && j < 0; ++e)
        if (A->c1tag[e] != to) j = e;
      if (j < 0) j = 0;
      for (int e = 0; e < (int)A->c1tag.size(); ++e)
        if (A->c1tag[e] != to && !dead(A->c1tag[e]) && A->c1tag[e] < A->c1tag[j] &&
            !dead(A->c1tag[j]))
          j = e;
      A->c1tag[j] = k;
      c1out = A->c1c[j];
    }
    if (int r = fwd_step(A, cur, A->step_nsrc[k], A->dts[k], out, false, c1out)) return r;
    cur = out;
    A->fwd_steps_in_bwd += 1;
  }
  return BX_OK;
}

// reverse steps [a, b) with the state of step a in Xa (owned by the caller);
// chain: the split snapshots come from the forward run (no advance)
static int reverse_range(bx_adj* A, const double* Xa, long long a, long long b, double* lam,
                         bool chain) {
  const long long l = b - a;
  if (l <= 0) return BX_OK;
  if (l == 1) return rev_step(A, Xa, a, lam);
  const int s = (int)A->pool_free.size() + (chain ? A->chain_left : 0);
  if (s == 0) {
    // no snapshot left: rebuild each state from Xa (into lamB, free during reversal)
    for (long long k = b - 1; k >= a; --k) {
      if (int r = advance(A, Xa, a, k, A->lamB)) return r;
      if (int r = rev_step(A, A->lamB, k, lam)) return r;
    }
    return BX_OK;
  }
  const long long m = a + split_of(A->sched, chain, l, s);
  double* slot;
  if (chain) {
    const int k = A->chain_slot_of[m];
    if (k < 0) return aerr(A, BX_ERR_STATE, "checkpoint chain does not match the schedule");
    slot = A->pool[k];
    A->chain_left -= 1;
  } else {
    slot = take_slot(A);
    if (int rc = advance(A, Xa, a, m, slot)) return rc;
  }
  if (int rc = reverse_range(A, slot, m, b, lam, chain)) return rc;
  give_slot(A, slot);
  return reverse_range(A, Xa, a, m, lam, false);
}

// The grids the adjoint takes: face ghosts on the stage kernels' donor rule
// (the stencils read no others), fixed gamma, no flux_ang.  Their two-sweep
// plan may leave corner ghosts lagging; those enter only the Courant maximum.
static bool adjoint_grid(const bx_params& P, const GhostTable& T) {
  return T.face_rule_ok && !(P.flags & BX_FLAG_PHASE_ONLY) && !P.fluxangmom && P.h2stat == -1;
}

// dt sequence of nsteps steps of the per-phase kernels (the reference data
// flow, lagging corner ghosts included) from the planes X0, on a handle of its
// own; into A->dts and A->d_dts
static int phase_dts(bx_adj* A, const double* X0) {
  bx_handle* h2 = nullptr;
  if (int r = bx_create(&A->h->P, &h2)) return aerr(A, r, bx_last_error(nullptr));
  struct Closer {
    bx_handle* h;
    ~Closer() { bx_destroy(h); }
  } closer{h2};
  if (int r = bx_set_stream(h2, A->h->stream)) return aerr(A, r, bx_last_error(h2));
  if (int r = bx_handle_start_from_planes(h2, X0)) return aerr(A, r, bx_last_error(h2));
  if (int r = bx_set_clock(h2, 0.0, 0.0, 0)) return aerr(A, r, bx_last_error(h2));
  for (long long k = 0; k < A->nsteps; ++k) {
    int32_t ran = 0;
    if (int r = bx_step(h2, 1e300, &ran)) return aerr(A, r, bx_last_error(h2));
    double t, dt, dtold;
    int64_t step;
    if (int r = bx_get_clock(h2, &t, &dt, &dtold, &step)) return aerr(A, r, bx_last_error(h2));
    if (!ran) return aerr(A, BX_ERR_STATE, "the per-phase run stopped early");
    A->dts[k] = dt;
  }
  uint32_t bits = 0;
  int32_t path = 0;
  bx_status(h2, &bits, &path);
  if (bits & (kFlagVlimit | kFlagLowRho | kFlagNonFinite))
    return aerr(A, BX_ERR_STATE,
                "a guard fired in the forward run (velocity limiter, low density or non-finite "
                "values); the adjoint of this run is not defined by the fused stages");
  ACK(cudaMemcpyAsync(A->d_dts, A->dts.data(), A->nsteps * sizeof(double),
                      cudaMemcpyHostToDevice, A->h->stream));
  return BX_OK;
}

// ---- host level of the schedule

static void free_host_level(bx_adj* A) {
  if (A->cstream) cudaStreamSynchronize(A->cstream);
  for (double* p : A->hsnap) cudaFreeHost(p);
  A->hsnap.clear();
  for (int b = 0; b < 2; ++b) {
    if (A->cev[b]) cudaEventDestroy(A->cev[b]);
    if (A->uev[b]) cudaEventDestroy(A->uev[b]);
    A->cev[b] = A->uev[b] = nullptr;
    A->hold[b] = nullptr;
    A->hold_step[b] = -1;
  }
  if (A->cstream) cudaStreamDestroy(A->cstream);
  A->cstream = nullptr;
  A->hstride = 0;
  A->host_bytes = 0;
  A->host_valid = false;
}

// MemAvailable of /proc/meminfo in bytes, or 0 when it cannot be read
static unsigned long long host_mem_available() {
  FILE* f = std::fopen("/proc/meminfo", "r");
  if (!f) return 0;
  char line[256];
  unsigned long long kb = 0;
  while (std::fgets(line, sizeof line, f))
    if (std::sscanf(line, "MemAvailable: %llu kB", &kb) == 1) break;
  std::fclose(f);
  return kb * 1024ull;
}

// copy the state of step `step` (host snapshot j-1, j = step / hstride) into
// hold[b] on the copy stream, after the compute stream's work so far is done
// with that buffer
static int fetch_hold(bx_adj* A, int b, long long step) {
  const size_t bytes = 5 * A->ng * sizeof(double);
  ACK(cudaEventRecord(A->uev[b], A->h->stream));
  ACK(cudaStreamWaitEvent(A->cstream, A->uev[b], 0));
  ACK(cudaMemcpyAsync(A->hold[b], A->hsnap[step / A->hstride - 1], bytes, cudaMemcpyHostToDevice,
                      A->cstream));
  ACK(cudaEventRecord(A->cev[b], A->cstream));
  A->hold_step[b] = step;
  return BX_OK;
}

// reverse every step with the host level: segments [j L, (j+1) L) from the
// last to the first, each by reverse_range over the device pool
static int reverse_host_level(bx_adj* A, double* lam) {
  const long long L = A->hstride;
  const long long nseg = (A->nsteps + L - 1) / L;
  for (long long j = nseg - 1; j >= 0; --j) {
    const long long a = j * L, b = std::min(A->nsteps, a + L);
    const double* Xa = A->pool[0];
    if (j > 0) {
      const int hb = (int)(j & 1);
      if (A->hold_step[hb] != a)
        if (int r = fetch_hold(A, hb, a)) return r;
      ACK(cudaStreamWaitEvent(A->h->stream, A->cev[hb], 0));
      Xa = A->hold[hb];
    }
    // the start of segment j-1 goes into the buffer segment j+1 used
    if (j - 1 >= 1 && A->hold_step[(j - 1) & 1] != a - L)
      if (int r = fetch_hold(A, (int)((j - 1) & 1), a - L)) return r;
    if (int r = reverse_range(A, Xa, a, b, lam, false)) return r;
  }
  return BX_OK;
}

extern "C" {

const char* bx_adj_last_error(bx_adj* A) { return A ? A->err.c_str() : g_adj_err.c_str(); }

int bx_adj_destroy(bx_adj* A) {
  if (!A) return BX_OK;
  if (A->h && A->h->stream) cudaStreamSynchronize(A->h->stream);
  free_host_level(A);
  for (double* p : A->pool) cudaFree(p);
  double* ps[] = {A->W0, A->W1, A->W2, A->XT, A->lamA, A->lamB, A->lamC1,
                  A->P,  A->PA, A->d_dts};
  for (double* p : ps) cudaFree(p);
  for (double* p : A->c1c) cudaFree(p);
  cudaFree(A->c1pool);
  if (A->h) bx_destroy(A->h);
  delete A;
  return BX_OK;
}

int bx_adj_create(const bx_params* params, int64_t nsteps, int32_t snapshots, bx_adj** out) {
  if (!params || !out || nsteps <= 0 || snapshots < 1)
    return aerr(nullptr, BX_ERR_ARG, "bad arguments");
  bx_adj* A = new bx_adj();
  if (int r = bx_create_lean(params, &A->h)) {
    g_adj_err = bx_last_error(nullptr);
    delete A;
    return r;
  }
  if (!adjoint_grid(*params, A->h->T)) {
    bx_adj_destroy(A);
    return aerr(nullptr, BX_ERR_UNSUPPORTED,
                "the adjoint follows the fused stage arithmetic, which this grid does not have "
                "(face ghosts off the donor rule, fluxangmom or a tabulated EOS)");
  }
  A->dt_phase = !A->h->T.resolved2;
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
  double** planes5[] = {&A->W0, &A->W1, &A->W2, &A->XT, &A->lamA, &A->lamB, &A->lamC1};
  for (double** p : planes5)
    if ((rc = amalloc(A, p, 5 * n))) return fail(rc);
  A->c1c.assign(2, nullptr);
  A->c1tag.assign(2, -1);
  for (double*& p : A->c1c)
    if ((rc = amalloc(A, &p, 5 * n))) return fail(rc);
  if ((rc = amalloc(A, &A->P, 7 * n))) return fail(rc);
  if ((rc = amalloc(A, &A->PA, 7 * n))) return fail(rc);
  if ((rc = amalloc(A, &A->d_dts, nsteps))) return fail(rc);
  build_schedule(A->sched, nsteps, A->snaps);
  A->chain_slot_of.assign(nsteps + 1, -1);
  A->chain = chain_of(A->sched, nsteps, A->snaps);
  for (size_t j = 0; j < A->chain.size(); ++j) A->chain_slot_of[A->chain[j]] = 1 + (int)j;
  *out = A;
  return BX_OK;
}

int bx_adj_keep_stage0(bx_adj* A, int32_t enable) {
  if (!A) return aerr(A, BX_ERR_ARG, "bad arguments");
  if (enable && !A->c1pool) {
    const size_t bytes = (size_t)A->nsteps * 5 * A->ng * sizeof(double);
    if (cudaMalloc(&A->c1pool, bytes) != cudaSuccess) {
      cudaGetLastError();
      A->c1pool = nullptr;
      return aerr(A, BX_ERR_NOMEM, "no room for the stage-0 results of every step");
    }
    A->bytes += bytes;
  } else if (!enable && A->c1pool) {
    cudaFree(A->c1pool);
    A->c1pool = nullptr;
    A->bytes -= (size_t)A->nsteps * 5 * A->ng * sizeof(double);
  }
  A->c1_valid = false;  // filled by the next unfrozen forward run
  return BX_OK;
}

int bx_adj_stage0_cache(bx_adj* A, int32_t entries) {
  if (!A || entries < 2) return aerr(A, BX_ERR_ARG, "the stage-0 cache needs at least 2 entries");
  const long long n5 = 5 * A->ng;
  if (A->h && A->h->stream) cudaStreamSynchronize(A->h->stream);
  while ((int)A->c1c.size() > entries) {
    cudaFree(A->c1c.back());
    A->c1c.pop_back();
    A->bytes -= n5 * sizeof(double);
  }
  while ((int)A->c1c.size() < entries) {
    double* p = nullptr;
    if (cudaMalloc(&p, n5 * sizeof(double)) != cudaSuccess) {
      cudaGetLastError();
      A->c1tag.assign(A->c1c.size(), -1);
      return aerr(A, BX_ERR_NOMEM, "no room for the stage-0 cache entries");
    }
    A->c1c.push_back(p);
    A->bytes += n5 * sizeof(double);
  }
  A->c1tag.assign(A->c1c.size(), -1);
  return BX_OK;
}

int bx_adj_host_level(bx_adj* A, int64_t stride, int64_t* host_bytes) {
  if (!A || stride < 0 || stride == 1) return aerr(A, BX_ERR_ARG, "bad arguments");
  if (A->h && A->h->stream) cudaStreamSynchronize(A->h->stream);
  free_host_level(A);
  if (host_bytes) *host_bytes = 0;
  if (stride == 0 || stride >= A->nsteps) return BX_OK;
  if (A->snaps < 3)
    return aerr(A, BX_ERR_ARG, "the host level needs at least 3 snapshots (2 hold segment starts)");
  const long long nhost = (A->nsteps - 1) / stride;  // steps stride, 2 stride, ... < nsteps
  const size_t per = 5 * A->ng * sizeof(double);
  const unsigned long long need = (unsigned long long)nhost * per;
  const unsigned long long avail = host_mem_available();
  // pinned pages cannot be swapped out: leave the system half of what it has
  if (avail == 0 || need > avail / 2)
    return aerr(A, BX_ERR_NOMEM,
                "host level: " + std::to_string(need >> 20) + " MiB of pinned memory requested, " +
                    std::to_string(avail >> 20) + " MiB available (at most half is taken)");
  int rc = BX_OK;
  auto fail = [&](int code) {
    free_host_level(A);
    return code;
  };
  ACK(cudaStreamCreateWithFlags(&A->cstream, cudaStreamNonBlocking));
  for (int b = 0; b < 2; ++b) {
    if ((rc = (cudaEventCreateWithFlags(&A->cev[b], cudaEventDisableTiming) == cudaSuccess &&
               cudaEventCreateWithFlags(&A->uev[b], cudaEventDisableTiming) == cudaSuccess)
                  ? BX_OK
                  : BX_ERR_CUDA))
      return fail(aerr(A, rc, "host level: event creation failed"));
  }
  A->hsnap.assign(nhost, nullptr);
  for (long long j = 0; j < nhost; ++j)
    if (cudaHostAlloc(&A->hsnap[j], per, cudaHostAllocDefault) != cudaSuccess) {
      cudaGetLastError();
      A->hsnap[j] = nullptr;
      return fail(aerr(A, BX_ERR_NOMEM, "host level: pinned allocation failed"));
    }
  A->hold[0] = A->pool[A->snaps];
  A->hold[1] = A->pool[A->snaps - 1];
  A->hstride = stride;
  A->host_bytes = need;
  A->host_valid = false;  // filled by the next unfrozen forward run
  if (host_bytes) *host_bytes = (int64_t)need;
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
  EventPair ev;
  ACK(cudaEventRecord(ev.e0, s));
  // the unfrozen run keeps its initial state and the chain snapshots for the
  // backward pass; frozen runs start from lamB and store nothing
  double* X0 = frozen ? A->lamB : A->pool[0];
  ACK(cudaMemcpyAsync(X0, cons0, n5 * sizeof(double), cudaMemcpyDeviceToDevice, s));
  // initial Courant rate and clock
  Ctrl c{};
  c.cfl = h->P.cfl;
  c.endtime = 1e300;
  c.max_step = 1ll << 62;
  ACK(cudaMemcpyAsync(h->d_ctrl, &c, sizeof(Ctrl), cudaMemcpyHostToDevice, s));
  ACK(box_rate(g, X0, g.ng, h->d_ctrl, s));
  // dt from the recorded sequence: frozen runs, and unfrozen ones on grids
  // whose dt comes from the per-phase kernels (computed first)
  const bool given_dt = frozen || A->dt_phase;
  if (!frozen && A->dt_phase)
    if (int r = phase_dts(A, X0)) return r;
  double* cur = X0;
  double* bufs[2] = {A->W0, A->W2};
  int nsrc = 1;
  for (long long k = 0; k < A->nsteps; ++k) {
    double* out = bufs[k & 1];
    int hb = -1;  // host level: the hold buffer this step's output goes to
    if (!frozen && A->hstride) {
      if ((k + 1) % A->hstride == 0 && k + 1 < A->nsteps) {
        hb = (int)(((k + 1) / A->hstride) & 1);
        // the copy out of this buffer two host snapshots ago must be done
        ACK(cudaStreamWaitEvent(s, A->cev[hb], 0));
        out = A->hold[hb];
      }
    } else if (!frozen && A->chain_slot_of[k + 1] >= 0) {
      out = A->pool[A->chain_slot_of[k + 1]];
    }
    StageArgs a{};
    a.ctrl = h->d_ctrl;
    a.geom = h->d_geom;
    a.tiles = h->d_tiles;
    a.ncells_total = g.ng;
    a.nsrc = nsrc;
    a.U = A->P;
    if (given_dt) {
      k_set_clock<<<1, 1, 0, s>>>(h->d_ctrl, A->dts[k], 1);
    } else {
      ACK(launch_dt(h->d_ctrl, 1, s));
      k_record_dt<<<1, 1, 0, s>>>(h->d_ctrl, A->d_dts, k);
    }
    a.X = cur;
    a.out = (!frozen && A->c1pool) ? A->c1pool + k * n5 : A->W1;
    ACK(launch_stage(0, g.pow2 ? 1 : 0, g.threed != 0, a, h->ntiles, s));
    a.Y = a.out;
    a.out = out;
    ACK(launch_stage(1, g.pow2 ? 1 : 0, g.threed != 0, a, h->ntiles, s));
    if (!given_dt) ACK(launch_end(h->d_ctrl, 1, s));
    if (hb >= 0) {
      ACK(cudaEventRecord(A->uev[hb], s));
      ACK(cudaStreamWaitEvent(A->cstream, A->uev[hb], 0));
      ACK(cudaMemcpyAsync(A->hsnap[(k + 1) / A->hstride - 1], out, n5 * sizeof(double),
                          cudaMemcpyDeviceToHost, A->cstream));
      ACK(cudaEventRecord(A->cev[hb], A->cstream));
      A->hold_step[hb] = k + 1;
    }
    A->step_nsrc[k] = nsrc;
    nsrc = 2;
    cur = out;
  }
  if (!frozen && A->hstride) {
    // the forward's time includes its copies to the host
    ACK(cudaStreamWaitEvent(s, A->cev[0], 0));
    ACK(cudaStreamWaitEvent(s, A->cev[1], 0));
  }
  ACK(cudaEventRecord(ev.e1, s));
  ACK(cudaEventSynchronize(ev.e1));
  float ms = 0.f;
  cudaEventElapsedTime(&ms, ev.e0, ev.e1);
  if (!frozen) {
    A->ms_fwd = ms;
    if (!A->dt_phase)
      ACK(cudaMemcpy(A->dts.data(), A->d_dts, A->nsteps * sizeof(double),
                     cudaMemcpyDeviceToHost));
  }
  Ctrl hc;
  ACK(cudaMemcpy(&hc, h->d_ctrl, sizeof(Ctrl), cudaMemcpyDeviceToHost));
  if (hc.flags & (kFlagVlimit | kFlagLowRho | kFlagNonFinite))
    return aerr(A, BX_ERR_STATE,
                "a guard fired in the forward run (velocity limiter, low density or non-finite "
                "values); the adjoint of this run is not defined by the fused stages");
  ACK(cudaMemcpyAsync(A->XT, cur, n5 * sizeof(double), cudaMemcpyDeviceToDevice, s));
  // reference cons after the run: one source more, ghosts filled
  ACK(fused_to_cons(g, cur, 2, consT, h->nghost, h->d_dst, h->d_src2, h->d_sgn2, s));
  ACK(cudaStreamSynchronize(s));
  if (!frozen) {
    A->have_forward = true;
    A->chain_valid = A->hstride == 0;
    A->host_valid = A->hstride != 0;
    A->c1_valid = A->c1pool != nullptr;
  }
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
  EventPair ev;
  ACK(cudaEventRecord(ev.e0, s));
  A->fwd_steps_in_bwd = 0;
  std::fill(A->c1tag.begin(), A->c1tag.end(), -1);
  A->c1_hits = 0;
  A->rev_done = A->nsteps;
  A->pool_free.clear();
  if (A->hstride && !A->host_valid)
    return aerr(A, BX_ERR_STATE, "the host level was set after the forward run: run it again");
  const bool chain = A->chain_valid && !A->hstride;
  // with the host level the two top slots hold segment starts
  for (int k = A->hstride ? A->snaps - 2 : A->snaps; k >= 1; --k)
    if (!chain || k > (int)A->chain.size()) A->pool_free.push_back(k);
  A->chain_left = chain ? (int)A->chain.size() : 0;
  double* lam = lam0;
  ACK(cudaMemcpyAsync(lam, lamT, n5 * sizeof(double), cudaMemcpyDeviceToDevice, s));
  // the reference cons after the run is src(C2_T): its adjoint first
  k_adj_src_vjp<<<ablk(g.ng), AB, 0, s>>>(g, A->XT, 1, lam);
  // the chain snapshots are overwritten while reversing: a later backward
  // without a new forward rebuilds them
  A->chain_valid = false;
  if (A->hstride) {
    if (int r = reverse_host_level(A, lam)) return r;
  } else if (int r = reverse_range(A, A->pool[0], 0, A->nsteps, lam, chain)) {
    return r;
  }
  ACK(cudaEventRecord(ev.e1, s));
  ACK(cudaEventSynchronize(ev.e1));
  float ms = 0.f;
  cudaEventElapsedTime(&ms, ev.e0, ev.e1);
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

int bx_adj_plan(int64_t nsteps, int32_t snapshots, int64_t* recomputed_first,
                int64_t* recomputed_again, int32_t* chain_snapshots) {
  if (nsteps <= 0 || snapshots < 1) return aerr(nullptr, BX_ERR_ARG, "bad arguments");
  const int snaps = (int)std::min<long long>(snapshots, nsteps);
  Schedule sc;
  build_schedule(sc, nsteps, snaps);
  const std::vector<long long> chain = chain_of(sc, nsteps, snaps);
  int free_slots = snaps - (int)chain.size(), chain_left = (int)chain.size();
  if (recomputed_first)
    *recomputed_first = plan_range(sc, nsteps, true, free_slots, chain_left);
  free_slots = snaps;
  chain_left = 0;
  if (recomputed_again)
    *recomputed_again = plan_range(sc, nsteps, false, free_slots, chain_left);
  if (chain_snapshots) *chain_snapshots = (int32_t)chain.size();
  return BX_OK;
}

int bx_adj_device_bytes(const bx_params* params, int64_t nsteps, int32_t snapshots,
                        int32_t stage0_cache_entries, int32_t keep_stage0, int64_t* bytes) {
  if (!params || !bytes || nsteps <= 0 || snapshots < 1 || stage0_cache_entries < 2 ||
      params->nx < 5 || params->ny < 5 || params->nz < 1)
    return aerr(nullptr, BX_ERR_ARG, "bad arguments");
  if ((long long)params->nx * params->ny * params->nz >= (1ll << 31))
    return aerr(nullptr, BX_ERR_ARG, "grid exceeds 2^31 cells");
  // the grids bx_adj_create takes
  {
    GhostTable T;
    build_ghost_tables(*params, T);
    if (!adjoint_grid(*params, T))
      return aerr(nullptr, BX_ERR_UNSUPPORTED,
                  "the adjoint follows the fused stage arithmetic, which this grid does not have "
                  "(face ghosts off the donor rule, fluxangmom or a tabulated EOS)");
  }
  const __int128 n = (__int128)params->nx * params->ny * params->nz;
  const __int128 snaps = std::min<long long>(snapshots, nsteps);
  // what bx_adj_create, bx_adj_stage0_cache and bx_adj_keep_stage0 allocate:
  // plane sets of 5 x n doubles (the initial state and the snapshots, seven
  // work sets, the stage-0 cache entries), the 14 primitive and adjoint planes,
  // the dt record and, kept, the stage-0 result of every step
  __int128 d = 5 * n * (snaps + 1 + 7 + stage0_cache_entries) + 14 * n + nsteps;
  if (keep_stage0) d += (__int128)nsteps * 5 * n;
  d *= (__int128)sizeof(double);
  *bytes = d > (__int128)INT64_MAX ? INT64_MAX : (int64_t)d;
  return BX_OK;
}

int bx_adj_forward_branches(bx_adj* A, const double* cons_base0, const double* cons_pert0,
                            double* consT_base, double* consT_pert) {
  if (!A || !cons_base0 || !cons_pert0 || !consT_base || !consT_pert)
    return aerr(A, BX_ERR_ARG, "bad arguments");
  if (!A->have_forward) return aerr(A, BX_ERR_STATE, "no recorded dt sequence");
  bx_handle* h = A->h;
  const Geom& g = h->g;
  cudaStream_t s = h->stream;
  const long long n = g.ng, n5 = 5 * n;
  // scratch: the engine's work planes (a frozen forward uses them too); the
  // snapshot pool, the stage-0 cache and the final state stay untouched
  double *Xb = A->lamA, *Xp = A->lamB, *Yb = A->lamC1, *Yp = A->W0;
  double *Ub = A->W1, *Up = A->W2, *Pb = A->P, *Pp = A->PA;
  ACK(cudaMemcpyAsync(Xb, cons_base0, n5 * sizeof(double), cudaMemcpyDeviceToDevice, s));
  ACK(cudaMemcpyAsync(Xp, cons_pert0, n5 * sizeof(double), cudaMemcpyDeviceToDevice, s));
  for (long long k = 0; k < A->nsteps; ++k) {
    const int nsrc = A->step_nsrc[k];
    const double dt = A->dts[k];
    k_fb_prims<0><<<ablk(n), AB, 0, s>>>(g, Xb, Xp, nullptr, nullptr, nsrc, Pb, Pp, Ub, Up);
    k_fb_update<0><<<ablk(n), AB, 0, s>>>(g, Pb, Pp, Xb, Xp, nullptr, nullptr, nsrc, dt, Yb, Yp);
    k_fb_prims<1><<<ablk(n), AB, 0, s>>>(g, Yb, Yp, Ub, Up, nsrc, Pb, Pp, nullptr, nullptr);
    // in place: each cell reads only its own step input and stage-0 result
    k_fb_update<1><<<ablk(n), AB, 0, s>>>(g, Pb, Pp, Xb, Xp, Yb, Yp, nsrc, dt, Xb, Xp);
    ACK(cudaGetLastError());
  }
  k_fb_finish<<<ablk(n), AB, 0, s>>>(g, Xb, Xp, consT_base, consT_pert);
  ACK(cudaGetLastError());
  ACK(cudaStreamSynchronize(s));
  return BX_OK;
}

int bx_adj_dts(bx_adj* A, double* dts) {
  if (!A || !dts) return BX_ERR_ARG;
  std::memcpy(dts, A->dts.data(), A->nsteps * sizeof(double));
  return BX_OK;
}

}  // extern "C"

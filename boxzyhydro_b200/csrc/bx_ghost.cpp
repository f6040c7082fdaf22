// bx_ghost.cpp -- ghost-cell tables and box geometry, built once per grid on the host.
//
// The reference fills ghost cells in index order (utils.f90:305-480): each
// ghost copies a donor chosen by ineigh (init_grid.f90:180-247) and
// check_corner (utils.f90:200-281), then reflective walls overwrite it with a
// mirrored cell three or one cells inward with the normal momentum negated.
// Donors can themselves be ghosts, updated earlier in the same sweep or not.
// Here that sweep is executed symbolically: every ghost's new value is
// expressed as (sign mask) x (value of a source cell read before the sweep),
// which the device then applies as a gather into scratch followed by a scatter
// -- the exact single-threaded result, in parallel.  Composing two sweeps
// gives the state after the pairs of consecutive fills the main loop performs
// (flux()+main, source()+main); when that resolves every ghost to an interior
// cell, the fused stage kernels can read ghosts on the fly instead of storing
// them.
#include <algorithm>
#include <cmath>
#include <cstring>

#include "bx_internal.h"

namespace bx {

bool is_pow2(double x) {
  if (!(x > 0.0) || !std::isfinite(x)) return false;
  int e;
  double m = std::frexp(x, &e);
  return m == 0.5 && e > -1000 && e < 1000;
}

void fill_geom(const bx_params& P, Geom& g) {
  std::memset(&g, 0, sizeof(g));
  g.nx = P.nx;
  g.ny = P.ny;
  g.nz = P.nz;
  g.threed = P.nz >= 6 ? 1 : 0;
  g.ax0 = 2;
  g.ax1 = P.nx - 2;
  g.ay0 = 2;
  g.ay1 = P.ny - 2;
  g.az0 = g.threed ? 2 : 0;
  g.az1 = g.threed ? P.nz - 2 : P.nz;
  g.sy = P.nx;
  g.sz = (long long)P.nx * P.ny;
  g.ng = (long long)P.nx * P.ny * P.nz;
  for (int k = 0; k < 6; ++k) g.wall[k] = P.no_outflow[k] ? 1 : 0;
  if (!g.threed) g.wall[4] = g.wall[5] = 0;  // init_grid.f90:76-79
  g.dx = P.dx;
  g.dy = P.dy;
  g.dz = P.dz;
  g.pow2 = (is_pow2(P.dx) && is_pow2(P.dy) && is_pow2(P.dz)) ? 1 : 0;
  g.idx = 1.0 / P.dx;
  g.idy = 1.0 / P.dy;
  g.idz = 1.0 / P.dz;
  g.axy = P.dy * P.dx;  // flux.f90:28-31
  g.ayz = P.dy * P.dz;
  g.axz = P.dx * P.dz;
  g.vol = P.dx * P.dy * P.dz;
  g.ivol = 1.0 / g.vol;
  g.gam = P.gammafix;
  g.gm1 = P.gammafix - 1.0;
  g.small_rho = P.small_rho;
  g.small_eps = P.small_eps;
  g.vlimit = P.vlimit;
  g.cfl = P.cfl;
  g.muc = P.muc;
  g.rgas = P.rgas;
  g.ang = P.fluxangmom ? 1 : 0;
  g.tab = P.h2stat >= 0 ? 1 : 0;
  g.yoff = P.yoffset;
}

namespace {

struct Ref {
  int64_t root;   // source cell
  uint8_t sgn;    // momentum sign mask
  uint8_t prefill;// 1: value of a ghost read before the sweep
};

struct Sim {
  int nx, ny, nz;
  int w[6];
  std::vector<int32_t> bnd;  // per cell
  std::vector<int64_t> ghosts;
  std::vector<int32_t> slot;  // ghost slot per cell, -1 interior
  int64_t id(int ix, int iy, int iz) const {  // 1-based -> 0-based cell
    return (int64_t)(ix - 1) + (int64_t)(iy - 1) * nx + (int64_t)(iz - 1) * nx * ny;
  }
};

// check_corner, utils.f90:200-281 (including its iz>=6 test at line 215)
int64_t check_corner(const Sim& s, int ix, int iy, int iz, int64_t ineigh) {
  const int nx = s.nx, ny = s.ny, nz = s.nz;
  if (ix < 3) {
    if (iy < 3) {
      if (nz >= 6) {
        if (iz < 3) return s.id(3, 3, 3);
        if (iz > nz - 2) return s.id(3, 3, nz - 2);
        return s.id(3, 3, iz);
      }
      return s.id(3, 3, iz);
    } else if (iy > ny - 2) {
      if (iz >= 6) {
        if (iz < 3) return s.id(3, ny - 2, 3);
        if (iz > nz - 2) return s.id(3, ny - 2, nz - 2);
        return s.id(3, ny - 2, iz);
      }
      return s.id(3, ny - 2, iz);
    } else {
      if (nz >= 6) {
        if (iz < 3) return s.id(3, iy, 3);
        if (iz > nz - 2) return s.id(3, iy, nz - 2);
        return ineigh;
      }
      return s.id(3, iy, iz);
    }
  } else if (ix > nx - 2) {
    if (iy < 3) {
      if (nz >= 6) {
        if (iz < 3) return s.id(nx - 2, 3, 3);
        if (iz > nz - 2) return s.id(nx - 2, 3, nz - 2);
        return s.id(nx - 2, 3, iz);
      }
      return s.id(nx - 2, 3, iz);
    } else if (iy > ny - 2) {
      if (nz >= 6) {
        if (iz < 3) return s.id(nx - 2, ny - 2, 3);
        if (iz > nz - 2) return s.id(nx - 2, ny - 2, nz - 2);
        return s.id(nx - 2, ny - 2, iz);
      }
      return s.id(nx - 2, ny - 2, iz);
    } else {
      if (nz >= 6) {
        if (iz < 3) return s.id(nx - 2, iy, 3);
        if (iz > nz - 2) return s.id(nx - 2, iy, nz - 2);
        return ineigh;
      }
      return s.id(nx - 2, iy, iz);
    }
  } else {
    if (iy < 3) {
      if (nz >= 6) {
        if (iz < 3) return s.id(ix, 3, 3);
        if (iz > nz - 2) return s.id(ix, 3, nz - 2);
        return ineigh;
      }
      return s.id(ix, 3, iz);
    } else if (iy > ny - 2) {
      if (nz >= 6) {
        if (iz < 3) return s.id(ix, ny - 2, 3);
        if (iz > nz - 2) return s.id(ix, ny - 2, nz - 2);
        return ineigh;
      }
      return s.id(ix, ny - 2, iz);
    }
  }
  return ineigh;
}

// One sweep of set_ghost_cells over symbolic values. `before` holds each ghost's
// value at sweep start; returns the values after the sweep.
std::vector<Ref> sweep(const Sim& s, const std::vector<Ref>& before) {
  std::vector<Ref> cur = before;
  const int nx = s.nx, ny = s.ny, nz = s.nz;
  auto val = [&](int64_t c) -> Ref {
    int32_t sl = s.slot[c];
    if (sl < 0) return Ref{c, 0, 0};
    return cur[sl];
  };
  auto flip = [](Ref r, uint8_t m) { r.sgn ^= m; return r; };
  for (size_t k = 0; k < s.ghosts.size(); ++k) {
    const int64_t g = s.ghosts[k];
    const int ix = (int)(g % nx) + 1;
    const int iy = (int)((g / nx) % ny) + 1;
    const int iz = (int)(g / ((int64_t)nx * ny)) + 1;
    int64_t ineigh = -1;
    if (s.bnd[g] == 1) {  // init_grid.f90:180-203 (donor kept in ineigh(1))
      if (ix == 1) ineigh = g + 2;
      else if (ix == nx) ineigh = g - 2;
      else if (iy == 1) ineigh = g + 2 * (int64_t)nx;
      else if (iy == ny) ineigh = g - 2 * (int64_t)nx;
      else if (iz == 1) ineigh = nz < 6 ? g : g + 2 * (int64_t)nx * ny;
      else ineigh = nz < 6 ? g : g - 2 * (int64_t)nx * ny;
    } else {  // utils.f90:320-330
      if (ix == 2) ineigh = g + 1;
      else if (ix == nx - 1) ineigh = g - 1;
      else if (iy == 2) ineigh = g + nx;
      else if (iy == ny - 1) ineigh = g - nx;
      else if (iz == 2) ineigh = nz < 6 ? g : g + (int64_t)nx * ny;
      else if (iz == nz - 1) ineigh = nz < 6 ? g : g - (int64_t)nx * ny;
    }
    ineigh = check_corner(s, ix, iy, iz, ineigh);
    Ref v = val(ineigh);
    if (s.w[0]) {
      if (ix == 1) v = flip(val(s.id(ix + 3, iy, iz)), 1);
      else if (ix == 2) v = flip(val(s.id(ix + 1, iy, iz)), 1);
    }
    if (s.w[1]) {
      if (ix == nx) v = flip(val(s.id(ix - 3, iy, iz)), 1);
      else if (ix == nx - 1) v = flip(val(s.id(ix - 1, iy, iz)), 1);
    }
    if (s.w[2]) {
      if (iy == 1) v = flip(val(s.id(ix, iy + 3, iz)), 2);
      else if (iy == 2) v = flip(val(s.id(ix, iy + 1, iz)), 2);
    }
    if (s.w[3]) {
      if (iy == ny) v = flip(val(s.id(ix, iy - 3, iz)), 2);
      else if (iy == ny - 1) v = flip(val(s.id(ix, iy - 1, iz)), 2);
    }
    if (s.w[4]) {
      if (iz == 1) v = flip(val(s.id(ix, iy, iz + 3)), 4);
      else if (iz == 2) v = flip(val(s.id(ix, iy, iz + 1)), 4);
    }
    if (s.w[5]) {
      if (iz == nz) v = flip(val(s.id(ix, iy, iz - 3)), 4);
      else if (iz == nz - 1) v = flip(val(s.id(ix, iy, iz - 1)), 4);
    }
    cur[k] = v;
  }
  return cur;
}

}  // namespace

void build_ghost_tables(const bx_params& P, GhostTable& T) {
  Sim s;
  s.nx = P.nx;
  s.ny = P.ny;
  s.nz = P.nz;
  for (int k = 0; k < 6; ++k) s.w[k] = P.no_outflow[k] ? 1 : 0;
  if (P.nz < 6) s.w[4] = s.w[5] = 0;
  const int64_t ng = (int64_t)P.nx * P.ny * P.nz;
  s.bnd.assign(ng, 0);
  s.slot.assign(ng, -1);
  for (int iz = 1; iz <= P.nz; ++iz) {
    const bool f1z = P.nz >= 6 && (iz == 1 || iz == P.nz);
    const bool f2z = P.nz >= 6 && (iz == 2 || iz == P.nz - 1);
    for (int iy = 1; iy <= P.ny; ++iy)
      for (int ix = 1; ix <= P.nx; ++ix) {
        const bool f1 = f1z || ix == 1 || ix == P.nx || iy == 1 || iy == P.ny;
        const bool f2 = f2z || ix == 2 || ix == P.nx - 1 || iy == 2 || iy == P.ny - 1;
        const int64_t c = s.id(ix, iy, iz);
        s.bnd[c] = f1 ? 1 : (f2 ? 2 : 0);
        if (f1 || f2) {
          s.slot[c] = (int32_t)s.ghosts.size();
          s.ghosts.push_back(c);
        }
      }
  }
  const size_t n = s.ghosts.size();
  std::vector<Ref> leaf(n);
  for (size_t k = 0; k < n; ++k) leaf[k] = Ref{s.ghosts[k], 0, 1};
  std::vector<Ref> one = sweep(s, leaf);
  std::vector<Ref> two = sweep(s, one);
  T.dst.resize(n);
  T.src1.resize(n);
  T.sgn1.resize(n);
  T.src2.resize(n);
  T.sgn2.resize(n);
  bool resolved = true;
  for (size_t k = 0; k < n; ++k) {
    T.dst[k] = (int32_t)s.ghosts[k];
    T.src1[k] = (int32_t)one[k].root;
    T.sgn1[k] = one[k].sgn;
    T.src2[k] = (int32_t)two[k].root;
    T.sgn2[k] = two[k].sgn;
    if (two[k].prefill || s.bnd[two[k].root] != 0) resolved = false;
  }
  T.resolved2 = resolved;
  // face ghosts (one coordinate in the ghost band) must follow the donor rule
  // used by the stage kernels: outflow -> first interior cell, reflective ->
  // mirror image across the wall with that axis' momentum negated.  Checked on
  // unresolved plans too: there the stencils still read face ghosts only, and
  // the lagging edge and corner ghosts enter nothing but the Courant maximum.
  bool ok = true;
  const int nx = P.nx, ny = P.ny, nz = P.nz;
  const bool threed = nz >= 6;
  auto donor = [&](int c, int a0, int a1, int wl, int wr, uint8_t bit, uint8_t& sg) {
    if (c < a0) { if (wl) { sg |= bit; return 2 * a0 - 1 - c; } return a0; }
    if (c >= a1) { if (wr) { sg |= bit; return 2 * a1 - 1 - c; } return a1 - 1; }
    return c;
  };
  for (size_t k = 0; k < n && ok; ++k) {
    const int64_t g = s.ghosts[k];
    const int x = (int)(g % nx), y = (int)((g / nx) % ny), z = (int)(g / ((int64_t)nx * ny));
    const int gx = (x < 2 || x >= nx - 2), gy = (y < 2 || y >= ny - 2);
    const int gz = threed && (z < 2 || z >= nz - 2);
    if (gx + gy + gz != 1) continue;
    uint8_t sg = 0;
    const int dxn = donor(x, 2, nx - 2, s.w[0], s.w[1], 1, sg);
    const int dyn = donor(y, 2, ny - 2, s.w[2], s.w[3], 2, sg);
    const int dzn = threed ? donor(z, 2, nz - 2, s.w[4], s.w[5], 4, sg) : z;
    const int64_t want = (int64_t)dxn + (int64_t)dyn * nx + (int64_t)dzn * nx * ny;
    if (two[k].root != want || two[k].sgn != sg) ok = false;
  }
  T.face_rule_ok = ok;
}

}  // namespace bx

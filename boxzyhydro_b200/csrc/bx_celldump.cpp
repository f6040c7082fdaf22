// bx_celldump.cpp -- the reference's celldump file: writer (write_files.f90:55-63)
// and restart reader (read_hydro.f90:122-187), for hosts that drive the library
// without the reference's Fortran main.
//
// File: Fortran unformatted sequential, gfortran with -frecord-marker=4
// (Makefile:20), little endian: every record is [int32 n][n bytes][int32 n].
//   1: int32 readtest = 1234
//   2: float64 time, int32 step
//   3: the units record, 8 x float64 in the order of derived_types.f90:14-15
//      (length, time, mass, density, rgas, eps, kelvin, vel), units.f90:10-17
//   4..ngrid+3: float64 x, y, z, rho, p, u1, u2, u3, phi, E, muc; int32 boundary
#include <cuda_runtime.h>

#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "bx_handle.h"
#include "bx_internal.h"

namespace {

struct Units {
  double length, time, mass, density, rgas, eps, kelvin, vel;
};

// units.f90:10-17 with the constants of parameters.f90:7-11
Units get_units() {
  const double pi = 3.1415926535897931, gcgs = 6.67e-8, rgas_cgs = 8.254e7;
  Units s;
  s.length = 1.496e13;
  s.time = (3600.0 * 365.25 * 24.0) / (2.0 * pi);
  s.density = 1.0 / (gcgs * (s.time * s.time));
  s.mass = s.density * (s.length * s.length * s.length);
  s.vel = s.length / s.time;
  s.eps = s.vel * s.vel * s.mass / (s.length * s.length * s.length);
  s.kelvin = 1.0;
  s.rgas = rgas_cgs / (s.vel * s.vel / s.kelvin);
  return s;
}

// boundary flag of a cell (init_grid.f90:81-104): 1 on the outermost layer,
// 2 on the next, 0 inside; z layers only when nz >= 6
int boundary_flag(const bx_params& P, int ix, int iy, int iz) {  // 1-based
  const bool zon = P.nz >= 6;
  const bool f1 = ix == 1 || ix == P.nx || iy == 1 || iy == P.ny || (zon && (iz == 1 || iz == P.nz));
  const bool f2 = ix == 2 || ix == P.nx - 1 || iy == 2 || iy == P.ny - 1 ||
                  (zon && (iz == 2 || iz == P.nz - 1));
  return f1 ? 1 : (f2 ? 2 : 0);
}

// cell centre along one axis (init_grid.f90:84,88,92)
inline double centre(double d, int i, int n) { return d * ((double)i - ((double)n + 1.0) / 2.0); }

class Writer {
 public:
  explicit Writer(FILE* f) : f_(f) { buf_.reserve(1 << 20); }
  void record(const void* p, int32_t n) {
    put(&n, 4);
    put(p, n);
    put(&n, 4);
  }
  void put(const void* p, size_t n) {
    const char* c = static_cast<const char*>(p);
    buf_.insert(buf_.end(), c, c + n);
    if (buf_.size() >= (1u << 20)) flush();
  }
  bool flush() {
    if (!buf_.empty() && std::fwrite(buf_.data(), 1, buf_.size(), f_) != buf_.size()) ok_ = false;
    buf_.clear();
    return ok_;
  }
  bool ok() const { return ok_; }

 private:
  FILE* f_;
  std::vector<char> buf_;
  bool ok_ = true;
};

// reads one record of exactly n bytes into p; false on a short file or a
// record length that differs
bool read_record(FILE* f, void* p, int32_t n) {
  int32_t a = 0, b = 0;
  if (std::fread(&a, 4, 1, f) != 1 || a != n) return false;
  if (n > 0 && std::fread(p, 1, n, f) != (size_t)n) return false;
  if (std::fread(&b, 4, 1, f) != 1 || b != n) return false;
  return true;
}

}  // namespace

extern "C" {

int bx_write_celldump(bx_handle* h, const char* path, const double* phi) {
  if (!h || !path) return BX_ERR_ARG;
  // write_files.f90:32: state() first, with its effect on the arrays
  if (int r = bx_state(h)) return r;
  const bx_params& P = h->P;
  const long long ng = (long long)P.nx * P.ny * P.nz;
  std::vector<double> cons(5 * ng), u(3 * ng), p(ng);
  if (int r = bx_download(h, cons.data(), u.data(), p.data())) return r;
  double time = 0.0, dt = 0.0, dtold = 0.0;
  int64_t step = 0;
  if (int r = bx_get_clock(h, &time, &dt, &dtold, &step)) return r;
  // muc_array: the tables' mu per cell (H2STAT >= 0), else the constant muc
  std::vector<double> mucv;
  if (h->pa.muc) {
    mucv.resize(ng);
    if (cudaMemcpy(mucv.data(), h->pa.muc, ng * sizeof(double), cudaMemcpyDeviceToHost) !=
        cudaSuccess) {
      h->err = "muc download failed";
      return BX_ERR_CUDA;
    }
  }
  FILE* f = std::fopen(path, "wb");
  if (!f) {
    h->err = std::string("cannot open ") + path + " for writing";
    return BX_ERR_ARG;
  }
  Writer w(f);
  const int32_t readtest = 1234;
  w.record(&readtest, 4);
  char r2[12];
  const int32_t step32 = (int32_t)step;
  std::memcpy(r2, &time, 8);
  std::memcpy(r2 + 8, &step32, 4);
  w.record(r2, 12);
  const Units s = get_units();
  w.record(&s, 64);
  char rec[92];
  long long i = 0;
  for (int iz = 1; iz <= P.nz; ++iz) {
    const double z = centre(P.dz, iz, P.nz);
    for (int iy = 1; iy <= P.ny; ++iy) {
      const double y = centre(P.dy, iy, P.ny);
      for (int ix = 1; ix <= P.nx; ++ix, ++i) {
        const double v[11] = {centre(P.dx, ix, P.nx), y, z, cons[5 * i], p[i], u[3 * i],
                              u[3 * i + 1], u[3 * i + 2], phi ? phi[i] : 0.0, cons[5 * i + 4],
                              mucv.empty() ? P.muc : mucv[i]};
        const int32_t b = boundary_flag(P, ix, iy, iz);
        std::memcpy(rec, v, 88);
        std::memcpy(rec + 88, &b, 4);
        w.record(rec, 92);
      }
    }
  }
  const bool ok = w.flush();
  const bool closed = std::fclose(f) == 0;
  if (!ok || !closed) {
    h->err = std::string("write error on ") + path;
    return BX_ERR_ARG;
  }
  return BX_OK;
}

int bx_read_celldump(bx_handle* h, const char* path, double* phi, double* time_out,
                     int64_t* step_out) {
  if (!h || !path) return BX_ERR_ARG;
  const bx_params& P = h->P;
  const long long ng = (long long)P.nx * P.ny * P.nz;
  FILE* f = std::fopen(path, "rb");
  if (!f) {
    h->err = std::string("cannot open ") + path;
    return BX_ERR_ARG;
  }
  auto bad = [&](const char* what) {
    std::fclose(f);
    h->err = std::string(path) + ": " + what;
    return BX_ERR_ARG;
  };
  int32_t readtest = 0;
  char r2[12];
  Units s;
  if (!read_record(f, &readtest, 4)) return bad("first record is not one integer");
  if (!read_record(f, r2, 12)) return bad("second record is not (time, step)");
  if (!read_record(f, &s, 64)) return bad("third record is not the 8 units");
  double time;
  int32_t step32;
  std::memcpy(&time, r2, 8);
  std::memcpy(&step32, r2 + 8, 4);
  std::vector<double> cons(5 * ng), u(3 * ng), p(ng);
  char rec[92];
  double v[11];
  for (long long i = 0; i < ng; ++i) {
    if (!read_record(f, rec, 92)) return bad("fewer cell records than the grid has cells");
    std::memcpy(v, rec, 88);
    // read_hydro.f90:130-132 and :155-158: m = u*rho
    cons[5 * i] = v[3];
    p[i] = v[4];
    u[3 * i] = v[5];
    u[3 * i + 1] = v[6];
    u[3 * i + 2] = v[7];
    if (phi) phi[i] = v[8];
    cons[5 * i + 4] = v[9];
    cons[5 * i + 1] = u[3 * i] * cons[5 * i];
    cons[5 * i + 2] = u[3 * i + 1] * cons[5 * i];
    cons[5 * i + 3] = u[3 * i + 2] * cons[5 * i];
  }
  std::fclose(f);
  // read_hydro.f90:174-180: the outermost layer (indx_bound) reset
  long long i = 0;
  for (int iz = 1; iz <= P.nz; ++iz)
    for (int iy = 1; iy <= P.ny; ++iy)
      for (int ix = 1; ix <= P.nx; ++ix, ++i)
        if (boundary_flag(P, ix, iy, iz) == 1) {
          cons[5 * i] = P.small_rho;
          cons[5 * i + 1] = 0.0;
          cons[5 * i + 2] = 0.0;
          cons[5 * i + 3] = 0.0;
          cons[5 * i + 4] = P.small_eps;
        }
  if (int r = bx_upload(h, cons.data(), u.data(), p.data())) return r;
  // read_hydro.f90:183 state(); main.f90:196-199: dtold = 0, step = irestart
  if (int r = bx_state(h)) return r;
  if (int r = bx_set_clock(h, time, 0.0, (int64_t)step32)) return r;
  if (time_out) *time_out = time;
  if (step_out) *step_out = step32;
  return BX_OK;
}

}  // extern "C"

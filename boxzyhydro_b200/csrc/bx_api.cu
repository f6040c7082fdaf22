// bx_api.cu -- the C ABI of include/boxzy_gpu.h.
//
// A handle holds one reference grid in two interchangeable device forms:
//  * the reference's module arrays (cons, cons_old, u, p, adindx) for the
//    per-phase kernels, and
//  * the fused form: conserved planes only (velocity and pressure are
//    recomputed from them), advanced by two stage kernels per step.
// A step runs fused when the grid's ghost fill resolves to interior cells
// within the two consecutive fills the main loop performs and the previous
// step left u == m/rho and no low-density cell; the stage kernels raise a
// flag when the velocity limiter or the low-density EOS branch would fire, and
// the step is then redone from its (untouched) input with the per-phase
// kernels, which follow the reference's data flow exactly.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <string>

#include "bx_internal.h"

using namespace bx;


#include "bx_handle.h"

// the message of the calling thread's last failed call made without a handle
static thread_local std::string g_create_err;

#define CK(expr)                                                                  \
  do {                                                                            \
    cudaError_t e_ = (expr);                                                      \
    if (e_ != cudaSuccess) {                                                      \
      h->err = std::string(#expr) + ": " + cudaGetErrorString(e_);                \
      return BX_ERR_CUDA;                                                         \
    }                                                                             \
  } while (0)

#define CHECK_H()                    \
  do {                               \
    if (!h) return BX_ERR_ARG;       \
  } while (0)

static int set_err(bx_handle* h, int code, const std::string& m) {
  if (h) h->err = m;
  else g_create_err = m;
  return code;
}

static cudaError_t dalloc(void** p, size_t bytes) {
  if (bytes == 0) bytes = 16;
  return cudaMalloc(p, bytes);
}

// ---- tiles: TX x TY column tiles times z chunks sized so the launch fills the GPU
static std::vector<Tile> make_tiles(const Geom& g, int box, int slots, int zc_force = 0,
                                    int shape = 0) {
  const int TX = shape_tx(shape), TY = shape_ty(shape);
  const int NAx = g.ax1 - g.ax0, NAy = g.ay1 - g.ay0, NAz = g.az1 - g.az0;
  const int tx = (NAx + TX - 1) / TX, ty = (NAy + TY - 1) / TY;
  const long long cols = (long long)tx * ty;
  int best = NAz;
  double best_cost = 1e300;
  for (int zc = 1; zc <= NAz && !zc_force; ++zc) {
    const long long chunks = (NAz + zc - 1) / zc;
    const long long blocks = cols * chunks;
    const long long waves = (blocks + slots - 1) / slots;
    const double per = g.threed ? zc + 1.0 : (double)zc;
    const double cost = waves * per;
    if (cost < best_cost - 1e-9) {
      best_cost = cost;
      best = zc;
    }
  }
  if (zc_force) best = std::min(zc_force, NAz);
  std::vector<Tile> tiles;
  for (int z = 0; z < NAz; z += best)
    for (int y = 0; y < ty; ++y)
      for (int x = 0; x < tx; ++x) tiles.push_back(Tile{box, x * TX, y * TY, z, std::min(NAz, z + best)});
  return tiles;
}

static int create_handle(const bx_params* params, bx_handle** out, bool lean);

// whether the steps may run on the fused stage kernels: a grid they take, and
// the physics they have: fixed gamma or the tabulated EOS with its tables set
// and nz != 1 (the scale-height branch reads the previous gamma), flux_ang only
// with fixed gamma, and the tabulated EOS or flux_ang without a force (the
// force instances have the fixed-gamma tile shape)
static void update_eligible(bx_handle* h) {
  const bx_params& P = h->P;
  bool ok = h->fusable;
  if (P.h2stat >= 0) ok = ok && !P.fluxangmom && P.nz != 1 && h->d_eos != nullptr;
  if (h->shape != 0) ok = ok && !h->gforce_set;
  h->eligible = ok;
}

extern "C" {

const char* bx_version(void) { return "boxzy-b200 1.0 (sm_100a, FP64)"; }

const char* bx_last_error(bx_handle* h) {
  if (!h) return g_create_err.c_str();
  return h->err.c_str();
}

int bx_create(const bx_params* params, bx_handle** out) {
  return create_handle(params, out, false);
}

}  // extern "C"

int bx_create_lean(const bx_params* params, bx_handle** out) {
  return create_handle(params, out, true);
}

// lean: geometry, ghost tables, tiles, control block and stream only (no state
// planes); for engines that keep their own planes and call the stage kernels
static int create_handle(const bx_params* params, bx_handle** out, bool lean) {
  if (!params || !out) return set_err(nullptr, BX_ERR_ARG, "null argument");
  const bx_params& P = *params;
  if (P.h2stat < -1)
    return set_err(nullptr, BX_ERR_ARG, "H2STAT must be -1 (fixed gamma) or >= 0 (tables)");
  if (P.nx < 5 || P.ny < 5 || P.nz < 1)
    return set_err(nullptr, BX_ERR_ARG, "grid too small: need nx,ny>=5, nz>=1");
  if ((long long)P.nx * P.ny * P.nz >= (1ll << 31))
    return set_err(nullptr, BX_ERR_ARG, "grid exceeds 2^31 cells");
  if (!(P.dx > 0 && P.dy > 0 && P.dz > 0 && P.gammafix > 1.0 && P.cfl > 0))
    return set_err(nullptr, BX_ERR_ARG, "dx,dy,dz,cfl must be >0 and gammafix>1");
  // divisions by the cell sizes and volume use their correctly rounded
  // reciprocals, exact while these stay far from the overflow/subnormal range
  if (!(P.dx >= 1e-40 && P.dx <= 1e40 && P.dy >= 1e-40 && P.dy <= 1e40 && P.dz >= 1e-40 &&
        P.dz <= 1e40))
    return set_err(nullptr, BX_ERR_ARG, "dx,dy,dz must lie in [1e-40, 1e40]");
  bx_handle* h = new bx_handle();
  h->P = P;
  fill_geom(P, h->g);
  build_ghost_tables(P, h->T);
  h->fusable = h->T.resolved2 && h->T.face_rule_ok && !(P.flags & BX_FLAG_PHASE_ONLY);
  h->shape = P.h2stat >= 0 ? 2 : P.fluxangmom ? 3 : 0;
  update_eligible(h);
  const long long ng = h->g.ng;
  h->nghost = (int)h->T.dst.size();
  auto fail = [&](int code) {
    g_create_err = h->err;
    bx_destroy(h);
    return code;
  };
#define CKC(expr)                                                               \
  do {                                                                          \
    cudaError_t e_ = (expr);                                                    \
    if (e_ != cudaSuccess) {                                                    \
      h->err = std::string(#expr) + ": " + cudaGetErrorString(e_);              \
      return fail(e_ == cudaErrorMemoryAllocation ? BX_ERR_NOMEM : BX_ERR_CUDA); \
    }                                                                           \
  } while (0)
  CKC(cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking));
  h->own_stream = true;
  if (!lean) {
    for (int k = 0; k < 3; ++k) CKC(dalloc((void**)&h->buf[k], 5 * ng * sizeof(double)));
    CKC(dalloc((void**)&h->pa.cons, 5 * ng * sizeof(double)));
    CKC(dalloc((void**)&h->pa.cons_old, 5 * ng * sizeof(double)));
    CKC(dalloc((void**)&h->pa.u, 3 * ng * sizeof(double)));
    CKC(dalloc((void**)&h->pa.p, ng * sizeof(double)));
    CKC(dalloc((void**)&h->pa.adindx, ng * sizeof(double)));
    CKC(dalloc((void**)&h->pa.gtmp, 5 * (size_t)h->nghost * sizeof(double)));
    CKC(cudaMemset(h->pa.cons, 0, 5 * ng * sizeof(double)));
    CKC(cudaMemset(h->pa.u, 0, 3 * ng * sizeof(double)));
    CKC(cudaMemset(h->pa.p, 0, ng * sizeof(double)));
  }
  const int n = h->nghost;
  CKC(dalloc((void**)&h->d_dst, n * sizeof(int32_t)));
  CKC(dalloc((void**)&h->d_src1, n * sizeof(int32_t)));
  CKC(dalloc((void**)&h->d_src2, n * sizeof(int32_t)));
  CKC(dalloc((void**)&h->d_sgn1, n));
  CKC(dalloc((void**)&h->d_sgn2, n));
  if (n) {
    CKC(cudaMemcpy(h->d_dst, h->T.dst.data(), n * sizeof(int32_t), cudaMemcpyHostToDevice));
    CKC(cudaMemcpy(h->d_src1, h->T.src1.data(), n * sizeof(int32_t), cudaMemcpyHostToDevice));
    CKC(cudaMemcpy(h->d_src2, h->T.src2.data(), n * sizeof(int32_t), cudaMemcpyHostToDevice));
    CKC(cudaMemcpy(h->d_sgn1, h->T.sgn1.data(), n, cudaMemcpyHostToDevice));
    CKC(cudaMemcpy(h->d_sgn2, h->T.sgn2.data(), n, cudaMemcpyHostToDevice));
  }
  CKC(dalloc((void**)&h->d_geom, sizeof(Geom)));
  CKC(cudaMemcpy(h->d_geom, &h->g, sizeof(Geom), cudaMemcpyHostToDevice));
  int dev = 0, sms = 148;
  CKC(cudaGetDevice(&dev));
  CKC(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  const int per_sm = std::max(1, stage_blocks_per_sm(1, h->g.pow2, h->g.threed, h->shape));
  std::vector<Tile> tiles = make_tiles(h->g, 0, sms * per_sm, 0, h->shape);
  h->ntiles = (int)tiles.size();
  CKC(dalloc((void**)&h->d_tiles, tiles.size() * sizeof(Tile)));
  CKC(cudaMemcpy(h->d_tiles, tiles.data(), tiles.size() * sizeof(Tile), cudaMemcpyHostToDevice));
  CKC(dalloc((void**)&h->d_ctrl, sizeof(Ctrl)));
  CKC(cudaMallocHost((void**)&h->h_ctrl, sizeof(Ctrl)));
  std::memset(&h->clock, 0, sizeof(Ctrl));
  h->clock.cfl = P.cfl;
  h->clock.endtime = 0.0;
  h->clock.max_step = (1ll << 62);
  CKC(cudaMemcpy(h->d_ctrl, &h->clock, sizeof(Ctrl), cudaMemcpyHostToDevice));
#undef CKC
  *out = h;
  return BX_OK;
}

extern "C" {

int bx_destroy(bx_handle* h) {
  if (!h) return BX_OK;
  if (h->stream) cudaStreamSynchronize(h->stream);
  for (int k = 0; k < 3; ++k) cudaFree(h->buf[k]);
  cudaFree(h->pa.cons);
  cudaFree(h->pa.cons_old);
  cudaFree(h->pa.u);
  cudaFree(h->pa.p);
  cudaFree(h->pa.adindx);
  cudaFree(h->pa.gforce);
  cudaFree(h->pa.states);
  cudaFree(h->pa.gtmp);
  cudaFree(h->pa.muc);
  cudaFree(h->d_eos);
  for (cudaGraphExec_t x : h->run_graph)
    if (x) cudaGraphExecDestroy(x);
  for (cudaStream_t x : h->hs)
    if (x) cudaStreamDestroy(x);
  for (cudaEvent_t e : h->hev) cudaEventDestroy(e);
  for (cudaEvent_t e : h->io_tev) cudaEventDestroy(e);
  cudaFree(h->d_io_tiles);
  cudaFree(h->d_dst);
  cudaFree(h->d_src1);
  cudaFree(h->d_src2);
  cudaFree(h->d_sgn1);
  cudaFree(h->d_sgn2);
  cudaFree(h->d_geom);
  cudaFree(h->d_tiles);
  cudaFree(h->d_ctrl);
  if (h->h_ctrl) cudaFreeHost(h->h_ctrl);
  for (int k = 0; k < 3; ++k)
    if (h->ev[k]) cudaEventDestroy(h->ev[k]);
  if (h->own_stream && h->stream) cudaStreamDestroy(h->stream);
  delete h;
  return BX_OK;
}

int bx_set_stream(bx_handle* h, void* s) {
  CHECK_H();
  CK(cudaStreamSynchronize(h->stream));
  if (h->own_stream && h->stream) cudaStreamDestroy(h->stream);
  if (s) {
    h->stream = (cudaStream_t)s;
    h->own_stream = false;
  } else {
    CK(cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking));
    h->own_stream = true;
  }
  return BX_OK;
}

// device -> host clock mirror (synchronises the stream)
static int pull_clock(bx_handle* h) {
  CK(cudaMemcpyAsync(h->h_ctrl, h->d_ctrl, sizeof(Ctrl), cudaMemcpyDeviceToHost, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  h->clock = *h->h_ctrl;
  return BX_OK;
}
static int push_clock(bx_handle* h) {
  *h->h_ctrl = h->clock;
  CK(cudaMemcpyAsync(h->d_ctrl, h->h_ctrl, sizeof(Ctrl), cudaMemcpyHostToDevice, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  return BX_OK;
}

static int ensure_states(bx_handle* h) {
  if (!h->pa.states)
    CK(dalloc((void**)&h->pa.states, (h->g.ang ? 54 : 57) * h->g.ng * sizeof(double)));
  return BX_OK;
}

static int bx_adindx_fill(bx_handle* h) {
  // adindx(:) = gammafix, as state() sets it (state.f90:50)
  CK(fill_const(h->pa.adindx, h->g.ng, h->P.gammafix, h->stream));
  h->launches += 1;
  return BX_OK;
}

// the reference arrays of the fused state (p as state() leaves it after a step
// with a force, whose velocity array is the one of before source(1))
static int fused_arrays(bx_handle* h) {
  CK(fused_to_phase(h->g, h->buf[h->cur], h->nsrc, h->pa, h->nghost, h->d_dst, h->d_src2,
                    h->d_sgn2, h->stream));
  h->launches += 3;
  if (h->g.tab) {
    // state() with the tables: p, gamma and mu from the conserved variables and
    // u = m/rho (the velocity array at a step boundary of the fused path)
    CK(phase_state(h->g, h->pa, h->d_ctrl, h->stream));
    h->launches += 1;
  } else if (h->p_saved) {
    // no fused step since the planes took the reference arrays: their p stands
    CK(cudaMemcpyAsync(h->pa.p, h->pa.cons_old + 3 * h->g.ng, h->g.ng * sizeof(double),
                       cudaMemcpyDeviceToDevice, h->stream));
  } else if (h->grav_step) {
    CK(p_after_force(h->g, h->pa, h->pa.cons_old, h->nghost, h->d_dst, h->d_src2, h->stream));
    h->launches += 2;
  }
  return BX_OK;
}

// make the reference arrays current (from the fused planes if needed)
static int to_phase(bx_handle* h) {
  if (h->mode == 0) return BX_OK;
  if (int r = fused_arrays(h)) return r;
  h->mode = 0;
  return BX_OK;
}

// staging buffer for the AoS<->SoA transposes: a fused plane set that does not
// hold the current state
static double* staging(bx_handle* h) { return h->buf[(h->cur + 1) % 3]; }

static int enter_fused(bx_handle* h);

int bx_upload(bx_handle* h, const double* cons, const double* u, const double* p) {
  CHECK_H();
  if (!cons) return set_err(h, BX_ERR_ARG, "cons is required");
  const long long n = h->g.ng;
  double* tmp = staging(h);
  cudaStream_t s = h->stream;
  CK(cudaMemcpyAsync(tmp, cons, 5 * n * sizeof(double), cudaMemcpyHostToDevice, s));
  CK(aos_to_soa(tmp, h->pa.cons, n, 5, s));
  if (u) {
    CK(cudaMemcpyAsync(tmp, u, 3 * n * sizeof(double), cudaMemcpyHostToDevice, s));
    CK(aos_to_soa(tmp, h->pa.u, n, 3, s));
  } else {
    CK(cudaMemsetAsync(h->pa.u, 0, 3 * n * sizeof(double), s));
  }
  if (p) CK(cudaMemcpyAsync(h->pa.p, p, n * sizeof(double), cudaMemcpyHostToDevice, s));
  else CK(cudaMemsetAsync(h->pa.p, 0, n * sizeof(double), s));
  h->launches += 2;
  h->mode = 0;
  // a state the fused stages reproduce exactly (as left by a previous step)
  // continues on them; anything else starts on the per-phase kernels
  if (h->eligible) {
    if (int r = pull_clock(h)) return r;
    h->clock.flags = 0;
    if (int r = push_clock(h)) return r;
    CK(check_clean(h->g, h->pa, h->nghost, h->d_dst, h->d_src2, h->d_sgn2, h->d_ctrl, s));
    h->launches += 2;
    if (int r = pull_clock(h)) return r;
    const bool clean = !(h->clock.flags & kFlagNotClean);
    h->clock.flags = 0;
    if (int r = push_clock(h)) return r;
    if (clean) {
      // adindx = gammafix is what state() leaves; set it like the other path does
      return enter_fused(h);
    }
  }
  return bx_adindx_fill(h);
}

int bx_upload_conserved(bx_handle* h, const double* cons) {
  CHECK_H();
  if (!cons) return set_err(h, BX_ERR_ARG, "cons is required");
  if (h->g.tab) return set_err(h, BX_ERR_STATE, "H2STAT >= 0: upload u and p with bx_upload");
  const long long n = h->g.ng;
  cudaStream_t s = h->stream;
  double* tmp = staging(h);
  CK(cudaMemcpyAsync(tmp, cons, 5 * n * sizeof(double), cudaMemcpyHostToDevice, s));
  CK(aos_to_soa(tmp, h->pa.cons, n, 5, s));
  // u = m/rho (velocity() ran last) and p of state() with that u
  CK(prims_from_cons(h->g, h->pa, s));
  h->launches += 2;
  h->mode = 0;
  if (h->eligible) {
    if (int r = pull_clock(h)) return r;
    h->clock.flags = 0;
    if (int r = push_clock(h)) return r;
    CK(check_clean(h->g, h->pa, h->nghost, h->d_dst, h->d_src2, h->d_sgn2, h->d_ctrl, s));
    h->launches += 2;
    if (int r = pull_clock(h)) return r;
    const bool clean = !(h->clock.flags & kFlagNotClean);
    h->clock.flags = 0;
    if (int r = push_clock(h)) return r;
    if (clean) return enter_fused(h);
  }
  return bx_adindx_fill(h);
}

int bx_download(bx_handle* h, double* cons, double* u, double* p) {
  CHECK_H();
  const long long n = h->g.ng;
  cudaStream_t s = h->stream;
  if (h->mode == 1) {
    if (int r = fused_arrays(h)) return r;
  }
  double* tmp = staging(h);
  if (cons) {
    CK(soa_to_aos(h->pa.cons, tmp, n, 5, s));
    CK(cudaMemcpyAsync(cons, tmp, 5 * n * sizeof(double), cudaMemcpyDeviceToHost, s));
    h->launches += 1;
  }
  if (u) {
    // the transpose of u must not overwrite cons before its copy is done: the
    // stream orders them
    CK(soa_to_aos(h->pa.u, tmp + 5 * n - 3 * n, n, 3, s));
    CK(cudaMemcpyAsync(u, tmp + 5 * n - 3 * n, 3 * n * sizeof(double), cudaMemcpyDeviceToHost, s));
    h->launches += 1;
  }
  if (p) CK(cudaMemcpyAsync(p, h->pa.p, n * sizeof(double), cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  return BX_OK;
}

int bx_set_clock(bx_handle* h, double time, double dtold, int64_t step) {
  CHECK_H();
  if (int r = pull_clock(h)) return r;
  h->clock.time = time;
  h->clock.dtold = dtold;
  h->clock.step = step;
  return push_clock(h);
}

int bx_get_clock(bx_handle* h, double* time, double* dt, double* dtold, int64_t* step) {
  CHECK_H();
  if (int r = pull_clock(h)) return r;
  if (time) *time = h->clock.time;
  if (dt) *dt = h->clock.dt;
  if (dtold) *dtold = h->clock.dtold;
  if (step) *step = h->clock.step;
  return BX_OK;
}

int bx_set_dt(bx_handle* h, double dt) {
  CHECK_H();
  if (int r = pull_clock(h)) return r;
  h->clock.dt = dt;
  return push_clock(h);
}

// ---- per-phase entry points
int bx_state(bx_handle* h) {
  CHECK_H();
  if (h->g.tab && !h->pa.muc)
    return set_err(h, BX_ERR_STATE, "H2STAT >= 0: bx_set_eos_table must come first");
  if (int r = to_phase(h)) return r;
  CK(phase_state(h->g, h->pa, h->d_ctrl, h->stream));
  return pull_clock(h);
}
int bx_velocity(bx_handle* h) {
  CHECK_H();
  if (int r = to_phase(h)) return r;
  CK(phase_velocity(h->g, h->pa, h->d_ctrl, h->stream));
  return pull_clock(h);
}
int bx_courant(bx_handle* h, double* dt) {
  CHECK_H();
  if (int r = to_phase(h)) return r;
  CK(cudaMemsetAsync(&h->d_ctrl->rate_bits, 0, sizeof(unsigned long long), h->stream));
  CK(phase_courant(h->g, h->pa, h->d_ctrl, h->stream));
  CK(phase_courant_finish(h->d_ctrl, h->stream));
  if (int r = pull_clock(h)) return r;
  if (dt) *dt = h->clock.dt;
  return BX_OK;
}
int bx_ghost(bx_handle* h) {
  CHECK_H();
  if (int r = to_phase(h)) return r;
  CK(phase_ghost(h->nghost, h->d_dst, h->d_src1, h->d_sgn1, h->pa, h->g.ng, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  return BX_OK;
}
int bx_source(bx_handle* h, int32_t siter) {
  CHECK_H();
  (void)siter;
  if (int r = to_phase(h)) return r;
  CK(phase_source(h->g, h->pa, h->d_ctrl, 1.0, h->stream));
  CK(phase_ghost(h->nghost, h->d_dst, h->d_src1, h->d_sgn1, h->pa, h->g.ng, h->stream));
  return pull_clock(h);
}
int bx_flux(bx_handle* h, int32_t avg) {
  CHECK_H();
  if (avg != 0 && avg != 1) return set_err(h, BX_ERR_ARG, "avg must be 0 or 1");
  if (int r = to_phase(h)) return r;
  if (int r = ensure_states(h)) return r;
  CK(phase_flux(h->g, h->pa, h->d_ctrl, avg, h->stream));
  CK(phase_ghost(h->nghost, h->d_dst, h->d_src1, h->d_sgn1, h->pa, h->g.ng, h->stream));
  return pull_clock(h);
}
int bx_set_avmag(bx_handle* h, double avmagx, double avmagy, double avmagz) {
  CHECK_H();
  h->avmag[0] = avmagx;
  h->avmag[1] = avmagy;
  h->avmag[2] = avmagz;
  return BX_OK;
}
int bx_avisc(bx_handle* h) {
  CHECK_H();
  if (int r = to_phase(h)) return r;
  if (!h->d_qq) {
    if (cudaMalloc(&h->d_qq, 3 * h->g.ng * sizeof(double)) != cudaSuccess) {
      cudaGetLastError();
      h->d_qq = nullptr;
      return set_err(h, BX_ERR_NOMEM, "cudaMalloc of the qq array failed");
    }
  }
  CK(phase_avisc(h->g, h->pa.u, h->avmag, h->d_qq, h->stream));
  h->launches += 1;
  CK(cudaStreamSynchronize(h->stream));
  return BX_OK;
}
int bx_download_qq(bx_handle* h, double* qq) {
  CHECK_H();
  if (!qq) return set_err(h, BX_ERR_ARG, "qq is NULL");
  const long long n = h->g.ng;
  if (!h->d_qq) {
    // the reference's qq before any avisc call: zero (init_grid.f90:298)
    std::memset(qq, 0, 3 * n * sizeof(double));
    return BX_OK;
  }
  double* tmp = staging(h);
  CK(soa_to_aos(h->d_qq, tmp, n, 3, h->stream));
  h->launches += 1;
  CK(cudaMemcpyAsync(qq, tmp, 3 * n * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  return BX_OK;
}
int bx_save_cons_old(bx_handle* h) {
  CHECK_H();
  if (int r = to_phase(h)) return r;
  CK(phase_copy_old(h->g, h->pa, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  return BX_OK;
}

// a grid with the tabulated EOS or flux_ang takes the fused kernels only
// without a force (their force instances have the fixed-gamma tile shape): the
// state goes to the reference arrays when a force is set, and back with the
// next clean step once it is cleared
static int tab_force_switch(bx_handle* h, bool force) {
  if (h->shape == 0) return BX_OK;
  if (force && h->mode == 1)
    if (int r = to_phase(h)) return r;
  return BX_OK;
}

int bx_set_gforce(bx_handle* h, const double* gforce) {
  CHECK_H();
  const long long n = h->g.ng;
  if (int r = tab_force_switch(h, gforce != nullptr)) return r;
  if (!gforce) {
    h->gforce_set = false;
    update_eligible(h);
    CK(cudaStreamSynchronize(h->stream));
    cudaFree(h->pa.gforce);
    h->pa.gforce = nullptr;
    return BX_OK;
  }
  if (!h->pa.gforce) CK(dalloc((void**)&h->pa.gforce, 3 * n * sizeof(double)));
  // the staging planes hold no state in either form
  double* tmp = staging(h);
  CK(cudaMemcpyAsync(tmp, gforce, 3 * n * sizeof(double), cudaMemcpyHostToDevice, h->stream));
  CK(aos_to_soa(tmp, h->pa.gforce, n, 3, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  h->gforce_set = true;
  update_eligible(h);
  return BX_OK;
}

int bx_set_eos_table(bx_handle* h, const bx_eos_table* t) {
  CHECK_H();
  if (!t || t->neos < 2 || t->neos_rho < 1 || !t->eng_table2 || !t->gamma_table2 ||
      !t->muc_table2 || !t->tk_table2 || !t->rho_table || !t->deng_eos_array)
    return set_err(h, BX_ERR_ARG, "incomplete EOS table (need neos >= 2, neos_rho >= 1)");
  if (!h->g.tab) return set_err(h, BX_ERR_STATE, "the grid was created with H2STAT = -1");
  if (int r = to_phase(h)) return r;
  const long long n2 = (long long)t->neos * t->neos_rho, nr = t->neos_rho;
  cudaFree(h->d_eos);
  h->d_eos = nullptr;
  CK(dalloc((void**)&h->d_eos, (4 * n2 + 3 * nr) * sizeof(double)));
  const double* src[4] = {t->eng_table2, t->gamma_table2, t->muc_table2, t->tk_table2};
  for (int k = 0; k < 4; ++k)
    CK(cudaMemcpy(h->d_eos + k * n2, src[k], n2 * sizeof(double), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(h->d_eos + 4 * n2, t->rho_table, nr * sizeof(double), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(h->d_eos + 4 * n2 + nr, t->deng_eos_array, nr * sizeof(double),
                cudaMemcpyHostToDevice));
  if (!h->pa.muc) {
    CK(dalloc((void**)&h->pa.muc, h->g.ng * sizeof(double)));
    CK(cudaMemset(h->pa.muc, 0, h->g.ng * sizeof(double)));
  }
  EosDev& e = h->pa.eos;
  e.neos = t->neos;
  e.neos_rho = t->neos_rho;
  e.log_rho_low = t->log_rho_eos_low;
  e.drho = t->drho_eos;
  e.density_unit = t->density_unit;
  e.tk_bgrnd = t->tk_bgrnd;
  e.eng2 = h->d_eos;
  e.gam2 = h->d_eos + n2;
  e.muc2 = h->d_eos + 2 * n2;
  e.tk2 = h->d_eos + 3 * n2;
  e.rho = h->d_eos + 4 * n2;
  e.deng = h->d_eos + 4 * n2 + nr;
  e.log_eng1 = h->d_eos + 4 * n2 + 2 * nr;
  CK(eos_log_rows(e.eng2, e.neos, (int)nr, h->d_eos + 4 * n2 + 2 * nr, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  // the fused kernels read the tables from here on (not while a force is set)
  update_eligible(h);
  return BX_OK;
}

int bx_set_phi(bx_handle* h, const double* phi) {
  CHECK_H();
  if (!phi) return bx_set_gforce(h, nullptr);
  if (int r = tab_force_switch(h, true)) return r;
  const long long n = h->g.ng;
  if (!h->pa.gforce) CK(dalloc((void**)&h->pa.gforce, 3 * n * sizeof(double)));
  double* tmp = staging(h);
  CK(cudaMemcpyAsync(tmp, phi, n * sizeof(double), cudaMemcpyHostToDevice, h->stream));
  CK(phase_calc_gforce(h->g, tmp, h->pa.gforce, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  h->gforce_set = true;
  update_eligible(h);
  return BX_OK;
}

int bx_status(bx_handle* h, uint32_t* bits, int32_t* last_path) {
  CHECK_H();
  if (bits) *bits = h->status;
  if (last_path) *last_path = h->last_path;
  h->status = 0;
  return BX_OK;
}

int bx_device_cons(bx_handle* h, double** cons_soa, int64_t* ngrid) {
  CHECK_H();
  if (h->mode == 1)
    if (int r = fused_arrays(h)) return r;
  CK(cudaStreamSynchronize(h->stream));
  if (cons_soa) *cons_soa = h->pa.cons;
  if (ngrid) *ngrid = h->g.ng;
  return BX_OK;
}

// ---- whole steps
static int ghost1(bx_handle* h) {
  CK(phase_ghost(h->nghost, h->d_dst, h->d_src1, h->d_sgn1, h->pa, h->g.ng, h->stream));
  return BX_OK;
}

// main.f90:212-545 with the per-phase kernels (reference data flow)
static int phase_step(bx_handle* h) {
  if (int r = ensure_states(h)) return r;
  Geom& g = h->g;
  PhaseArrays& a = h->pa;
  cudaStream_t s = h->stream;
  Ctrl* c = h->d_ctrl;
  CK(phase_state(g, a, c, s));
  CK(cudaMemsetAsync(&c->rate_bits, 0, sizeof(unsigned long long), s));
  CK(phase_courant(g, a, c, s));
  CK(launch_dt(c, 1, s));
  CK(phase_source(g, a, c, 0.5, s));   // source(time,0) with dt/2
  if (int r = ghost1(h)) return r;
  if (int r = ghost1(h)) return r;     // main.f90:312
  CK(phase_state(g, a, c, s));
  CK(phase_velocity(g, a, c, s));
  CK(phase_copy_old(g, a, s));
  CK(phase_flux(g, a, c, 0, s));
  if (int r = ghost1(h)) return r;     // flux.f90:231
  if (int r = ghost1(h)) return r;     // main.f90:351
  CK(phase_state(g, a, c, s));
  CK(phase_velocity(g, a, c, s));
  CK(phase_flux(g, a, c, 1, s));
  if (int r = ghost1(h)) return r;
  if (int r = ghost1(h)) return r;     // main.f90:374
  CK(phase_state(g, a, c, s));
  CK(phase_velocity(g, a, c, s));
  CK(phase_source(g, a, c, 0.5, s));   // source(time+dt,1) with dt/2
  if (int r = ghost1(h)) return r;
  if (int r = ghost1(h)) return r;     // main.f90:511
  CK(phase_state(g, a, c, s));
  CK(phase_velocity(g, a, c, s));
  CK(launch_end(c, 1, s));
  h->launches += 46;
  return BX_OK;
}

static int fused_launch(bx_handle* h) {
  const int X = h->cur, Y = (h->cur + 1) % 3, Z = (h->cur + 2) % 3;
  StageArgs a{};
  a.ctrl = h->d_ctrl;
  a.geom = h->d_geom;
  a.tiles = h->d_tiles;
  a.ncells_total = h->g.ng;
  a.eos = h->pa.eos;
  a.nsrc = h->nsrc;
  // the velocity array is stale while the state lives in the planes (to_phase
  // rebuilds it), so it holds the stage-0 velocity here; cons_old likewise
  // takes the velocity after flux(1) of a step with a force
  a.U = h->pa.u;
  a.G = h->gforce_set ? h->pa.gforce : nullptr;
  a.UC = h->pa.cons_old;
  const bool p2 = h->g.pow2 != 0, t3 = h->g.threed != 0;
  CK(launch_dt(h->d_ctrl, 1, h->stream));
  a.X = h->buf[X];
  a.Y = nullptr;
  a.out = h->buf[Y];
  if (h->prof) CK(cudaEventRecord(h->ev[0], h->stream));
  CK(launch_stage(0, p2, t3, a, h->ntiles, h->stream, h->shape));
  if (h->prof) CK(cudaEventRecord(h->ev[1], h->stream));
  a.Y = h->buf[Y];
  a.out = h->buf[Z];
  CK(launch_stage(1, p2, t3, a, h->ntiles, h->stream, h->shape));
  if (h->prof) CK(cudaEventRecord(h->ev[2], h->stream));
  CK(launch_end(h->d_ctrl, 1, h->stream));
  h->launches += 4;
  return BX_OK;
}

// switch to the fused form after a clean per-phase step: the planes take the
// reference cons (sources of this step already applied: nsrc=1) and the Courant
// rate of the next step's state()/courant() is accumulated now.
static int enter_fused(bx_handle* h) {
  if (int r = bx_adindx_fill(h)) return r;
  // p of the reference arrays (after a step with a force, state() read a
  // velocity that m/rho of the planes no longer gives) kept until the next step
  CK(cudaMemcpyAsync(h->pa.cons_old + 3 * h->g.ng, h->pa.p, h->g.ng * sizeof(double),
                     cudaMemcpyDeviceToDevice, h->stream));
  h->p_saved = true;
  CK(cudaMemcpyAsync(h->buf[h->cur], h->pa.cons, 5 * h->g.ng * sizeof(double),
                     cudaMemcpyDeviceToDevice, h->stream));
  CK(phase_state(h->g, h->pa, h->d_ctrl, h->stream));
  CK(cudaMemsetAsync(&h->d_ctrl->rate_bits, 0, sizeof(unsigned long long), h->stream));
  CK(phase_courant(h->g, h->pa, h->d_ctrl, h->stream));
  h->launches += 2;
  h->nsrc = 1;
  h->mode = 1;
  h->grav_step = false;
  return pull_clock(h);
}

// the step on the per-phase kernels (reference data flow), then back to the
// fused form when the step left a state it reproduces
static int phase_path(bx_handle* h, int32_t* ran) {
  if (int r = phase_step(h)) return r;
  if (int r = pull_clock(h)) return r;
  const unsigned f = h->clock.flags;
  h->status |= f;
  h->last_path = 0;
  if (ran) *ran = 1;
  h->clock.flags = 0;
  if (int r = push_clock(h)) return r;
  if (f & kFlagNonFinite) return set_err(h, BX_ERR_STATE, "non-finite state produced by the step");
  if (h->eligible && !(f & (kFlagVlimit | kFlagLowRho))) return enter_fused(h);
  return BX_OK;
}

// after the fused launches of a step from the clock `before`: commit it, or
// redo it on the per-phase kernels when the limiter or the low-density branch
// fired (the input planes are untouched)
static int after_fused(bx_handle* h, const Ctrl& before, int32_t* ran, bool timed) {
  if (int r = pull_clock(h)) return r;
  const unsigned f = h->clock.flags;
  if (f & kFlagNonFinite) {
    h->status |= f;
    return set_err(h, BX_ERR_STATE, "non-finite state produced by the step");
  }
  if (timed && h->prof) {
    float t0 = 0.f, t1 = 0.f;
    CK(cudaEventElapsedTime(&t0, h->ev[0], h->ev[1]));
    CK(cudaEventElapsedTime(&t1, h->ev[1], h->ev[2]));
    h->ms_stage[0] += t0;
    h->ms_stage[1] += t1;
    h->n_stage += 1;
  }
  if (!(f & (kFlagVlimit | kFlagLowRho))) {
    h->cur = (h->cur + 2) % 3;
    // with a force the step's last source is applied in stage 1
    h->grav_step = h->gforce_set;
    h->p_saved = false;
    h->nsrc = h->gforce_set ? 1 : 2;
    h->clock.flags = 0;
    if (int r = push_clock(h)) return r;
    h->last_path = 1;
    if (ran) *ran = 1;
    return BX_OK;
  }
  // the limiter or the low-density branch fires in this step: redo it from
  // its untouched input with the reference data flow
  h->status |= f & (kFlagVlimit | kFlagLowRho);
  h->clock = before;
  h->clock.rate_bits = 0;
  if (int r = push_clock(h)) return r;
  if (int r = to_phase(h)) return r;
  return phase_path(h, ran);
}

int bx_step(bx_handle* h, double endtime, int32_t* ran) {
  CHECK_H();
  if (ran) *ran = 0;
  if (h->g.tab && !h->pa.muc)
    return set_err(h, BX_ERR_STATE, "H2STAT >= 0: bx_set_eos_table must come first");
  if (!(h->clock.time < endtime) || h->clock.step >= 1000000) return BX_OK;
  if (h->clock.endtime != endtime) {
    h->clock.endtime = endtime;
    if (int r = push_clock(h)) return r;
  }
  const Ctrl before = h->clock;
  if (h->mode == 1) {
    if (int r = fused_launch(h)) return r;
    return after_fused(h, before, ran, true);
  }
  return phase_path(h, ran);
}

// ---- one step with the state on the host, copies overlapped with the step.
// Slabs: groups of consecutive tile z-chunks (the tiles are z-chunk major),
// each with its cell range and the entries of the (igrid-ordered) ghost plan
// in it; a slab takes the next chunk too while a ghost of it has its donor
// beyond it, so every slab's ghosts can be filled once the slab is done.  For
// each slab: the last uploaded slab its stage 0 needs (the planes up to two
// beyond it), and the last its stage 1 needs (the stage-0 results up to two
// planes beyond it).
static int host_io_setup(bx_handle* h) {
  if (!h->slabs.empty()) return BX_OK;
  const Geom& g = h->g;
  const long long n = g.ng;
  // thin chunks (about 64 slabs, at least 2 planes each): a slab's copy back
  // can start once the planes up to four beyond it are in (256^3 measured
  // 15.8 ms per step with 64 slabs, 17.0 with 32, 21.1 with the 8 chunks of
  // the stage launches)
  const int naz = g.az1 - g.az0;
  const std::vector<Tile> tiles = make_tiles(g, 0, 1, std::max(2, (naz + 63) / 64));
  CK(cudaMalloc((void**)&h->d_io_tiles, tiles.size() * sizeof(Tile)));
  CK(cudaMemcpy(h->d_io_tiles, tiles.data(), tiles.size() * sizeof(Tile), cudaMemcpyHostToDevice));
  struct Chunk {
    int z0, z1, t0, nt;
  };
  std::vector<Chunk> ch;
  for (int t = 0; t < (int)tiles.size(); ++t) {
    const Tile& T = tiles[t];
    if (ch.empty() || ch.back().z0 != T.z0) ch.push_back(Chunk{T.z0, T.z1, t, 0});
    ch.back().nt += 1;
  }
  const std::vector<int32_t>& dst = h->T.dst;
  const std::vector<int32_t>& src = h->T.src2;
  auto first_ghost = [&](long long i) {
    return (int)(std::lower_bound(dst.begin(), dst.end(), (int32_t)std::min<long long>(i, INT32_MAX)) -
                 dst.begin());
  };
  size_t c = 0;
  while (c < ch.size()) {
    bx_handle::Slab sl{};
    sl.t0 = ch[c].t0;
    sl.z0 = ch[c].z0;
    sl.i0 = h->slabs.empty() ? 0 : h->slabs.back().i1;
    sl.g0 = first_ghost(sl.i0);
    size_t e = c;
    for (;;) {
      const bool last = e + 1 == ch.size();
      sl.i1 = last ? n : (long long)(g.az0 + ch[e].z1) * g.sz;
      sl.g1 = first_ghost(sl.i1);
      bool ok = true;
      for (int k = sl.g0; k < sl.g1 && ok; ++k) ok = src[k] < sl.i1;
      if (ok || last) break;
      ++e;
    }
    sl.z1 = ch[e].z1;
    sl.nt = ch[e].t0 + ch[e].nt - sl.t0;
    h->slabs.push_back(sl);
    c = e + 1;
  }
  const int ns = (int)h->slabs.size();
  auto last_slab_before = [&](long long cell_end) {  // last slab with i0 < cell_end
    int k = 0;
    while (k + 1 < ns && h->slabs[k + 1].i0 < cell_end) ++k;
    return k;
  };
  for (int j = 0; j < ns; ++j) {
    bx_handle::Slab& sl = h->slabs[j];
    if (!g.threed) {
      sl.s0_after = sl.s1_after = j;
      continue;
    }
    const int zhi = std::min(sl.z1 + 2, naz);
    sl.s0_after = std::max(j, last_slab_before((long long)(g.az0 + zhi) * g.sz));
  }
  for (int j = 0; j < ns; ++j) {
    bx_handle::Slab& sl = h->slabs[j];
    if (!g.threed) continue;
    int m = j;
    while (m + 1 < ns && h->slabs[m + 1].z0 < std::min(sl.z1 + 2, naz)) ++m;
    sl.s1_after = h->slabs[m].s0_after;
  }
  for (int k = 0; k < 4; ++k)
    CK(cudaStreamCreateWithFlags(&h->hs[k], cudaStreamNonBlocking));
  const size_t nev = 4 * (size_t)ns + 2;
  h->hev.assign(nev, nullptr);
  for (size_t k = 0; k < nev; ++k) CK(cudaEventCreateWithFlags(&h->hev[k], cudaEventDisableTiming));
  return BX_OK;
}

// Enqueue, slab by slab: the upload of cons_in (if given: copy on the upload
// stream, transpose into the planes X and the slab's Courant rate into
// rate_bits0 on the handle's stream) and, if `stages`, the stage launches whose
// inputs are in place once the slab is -- stage 0 on the handle's stream;
// stage 1 on it and the second compute stream in turn, each finished slab
// converted to the (5, ngrid) layout on the conversion stream and copied to
// cons_out on the download stream.  Nothing waits on the host.
static int host_io_enqueue(bx_handle* h, const double* cons_in, double* cons_out, bool stages) {
  const Geom& g = h->g;
  const long long n = g.ng;
  const int ns = (int)h->slabs.size();
  cudaStream_t s = h->stream, up = h->hs[0], down = h->hs[1], cs = h->hs[2], s2 = h->hs[3];
  cudaEvent_t* ev_in = h->hev.data() + 2;
  cudaEvent_t* ev_s0 = ev_in + ns;
  cudaEvent_t* ev_st1 = ev_s0 + ns;
  cudaEvent_t* ev_cv = ev_st1 + ns;
  double* aos = h->pa.cons;
  double* X = h->buf[h->cur];
  const int Yi = (h->cur + 1) % 3, Zi = (h->cur + 2) % 3;
  const bool p2 = g.pow2 != 0, t3 = g.threed != 0;
  const size_t cell = 5 * sizeof(double);
  StageArgs a{};
  a.ctrl = h->d_ctrl;
  a.geom = h->d_geom;
  a.ncells_total = n;
  a.nsrc = h->nsrc;
  a.U = h->pa.u;
  a.G = h->gforce_set ? h->pa.gforce : nullptr;
  a.UC = h->pa.cons_old;
  a.X = X;
  // the reference cons after the step: stage 1 applied source(1) itself when
  // the step has a force, else it is one force-free source short
  const int nsrc_out = h->gforce_set ? 1 : 2;
  int st1 = 0;  // stage-1 launches so far (alternating streams)
  const bool tp = h->io_prof && !h->io_tev.empty();
  auto tev = [&](int slab, int what) { return h->io_tev[1 + (size_t)kIoEv * slab + what]; };
  for (int k = 0; k < ns; ++k) {
    const bx_handle::Slab& sk = h->slabs[k];
    if (cons_in) {
      if (tp) CK(cudaEventRecord(tev(k, 0), up));
      CK(cudaMemcpyAsync(aos + 5 * sk.i0, cons_in + 5 * sk.i0, (sk.i1 - sk.i0) * cell,
                         cudaMemcpyHostToDevice, up));
      if (tp) CK(cudaEventRecord(tev(k, 1), up));
      CK(cudaEventRecord(ev_in[k], up));
      CK(cudaStreamWaitEvent(s, ev_in[k], 0));
      CK(slab_in(aos, X, n, sk.i0, sk.i1, s));
      CK(slab_rate(g, X, n, sk.i0, sk.i1, &h->d_ctrl->rate_bits0, s));
      h->launches += 2;
    }
    if (!stages) continue;
    for (int j = 0; j < ns; ++j) {
      const bx_handle::Slab& sl = h->slabs[j];
      if (sl.s0_after != k) continue;
      StageArgs aj = a;
      aj.tiles = h->d_io_tiles + sl.t0;
      aj.out = h->buf[Yi];
      CK(launch_stage(0, p2, t3, aj, sl.nt, s));
      h->launches += 1;
    }
    CK(cudaEventRecord(ev_s0[k], s));
    if (tp) CK(cudaEventRecord(tev(k, 2), s));
    for (int j = 0; j < ns; ++j) {
      const bx_handle::Slab& sl = h->slabs[j];
      if (sl.s1_after != k) continue;
      cudaStream_t sj = (st1++ & 1) ? s2 : s;
      if (sj == s2) CK(cudaStreamWaitEvent(s2, ev_s0[k], 0));
      StageArgs aj = a;
      aj.tiles = h->d_io_tiles + sl.t0;
      aj.Y = h->buf[Yi];
      aj.out = h->buf[Zi];
      CK(launch_stage(1, p2, t3, aj, sl.nt, sj));
      CK(cudaEventRecord(ev_st1[j], sj));
      if (tp) CK(cudaEventRecord(tev(j, 3), sj));
      CK(cudaStreamWaitEvent(cs, ev_st1[j], 0));
      CK(slab_out(g, h->buf[Zi], n, nsrc_out, aos, sl.i0, sl.i1, h->d_dst, h->d_src2, h->d_sgn2,
                  sl.g0, sl.g1, cs));
      CK(cudaEventRecord(ev_cv[j], cs));
      if (tp) CK(cudaEventRecord(tev(j, 4), cs));
      CK(cudaStreamWaitEvent(down, ev_cv[j], 0));
      if (tp) CK(cudaEventRecord(tev(j, 5), down));
      CK(cudaMemcpyAsync(cons_out + 5 * sl.i0, aos + 5 * sl.i0, (sl.i1 - sl.i0) * cell,
                         cudaMemcpyDeviceToHost, down));
      if (tp) CK(cudaEventRecord(tev(j, 6), down));
      h->launches += 3;
    }
  }
  return BX_OK;
}

// every stream of the host-overlapped step idle (the handle's stream included)
static int host_io_drain(bx_handle* h) {
  for (cudaStream_t x : h->hs) CK(cudaStreamSynchronize(x));
  CK(cudaStreamSynchronize(h->stream));
  return BX_OK;
}

// The step on the fused path is started before the upload has finished: its
// dt comes from the Courant rate the device holds (the one the previous fused
// step accumulated for the state it left), and each slab's stages start as
// soon as their planes are in.  The rate of the uploaded state is reduced on
// the way; when it equals the one dt was taken from, dt is the step's own and
// everything computed stands (the stages read the uploaded planes); when it
// differs, or the upload is not a state the fused path takes, the work is
// dropped and the step starts over from the uploaded planes.
int bx_step_host(bx_handle* h, const double* cons_in, double* cons_out, double endtime,
                 int32_t* ran) {
  CHECK_H();
  if (ran) *ran = 0;
  if (!cons_in || !cons_out) return set_err(h, BX_ERR_ARG, "cons_in and cons_out are required");
  if (!h->pa.cons) return set_err(h, BX_ERR_STATE, "the handle holds no state (lean handle)");
  if (!h->eligible || h->shape != 0) {
    // not on the fused path: the three calls it stands for
    if (int r = bx_upload_conserved(h, cons_in)) return r;
    if (int r = bx_step(h, endtime, ran)) return r;
    return bx_download(h, cons_out, nullptr, nullptr);
  }
  if (int r = host_io_setup(h)) return r;
  const Geom& g = h->g;
  const long long n = g.ng;
  cudaStream_t s = h->stream;
  cudaEvent_t ev_start = h->hev[0], ev_join = h->hev[1];
  const bool runs = h->clock.time < endtime && h->clock.step < 1000000;
  const bool spec = runs && h->clock.rate_bits != 0;
  // the uploaded state is one step boundary of the reference: sources short by one
  h->nsrc = 1;
  h->grav_step = false;
  h->p_saved = false;
  h->clock.endtime = endtime;
  h->clock.flags = 0;
  h->clock.rate_bits0 = 0;
  if (int r = push_clock(h)) return r;
  const Ctrl before = h->clock;  // rate_bits: the rate dt is taken from if spec
  if (h->io_prof) {
    if (h->io_tev.empty()) {
      h->io_tev.assign(1 + (size_t)kIoEv * h->slabs.size(), nullptr);
      for (cudaEvent_t& e : h->io_tev) CK(cudaEventCreate(&e));
    }
    CK(cudaEventRecord(h->io_tev[0], s));
  }
  CK(cudaEventRecord(ev_start, s));
  for (cudaStream_t x : h->hs) CK(cudaStreamWaitEvent(x, ev_start, 0));
  if (spec) CK(launch_dt(h->d_ctrl, 1, s));
  if (int r = host_io_enqueue(h, cons_in, cons_out, spec)) return r;
  CK(box_check_clean(g, h->buf[h->cur], n, h->nghost, h->d_dst, h->d_src2, h->d_sgn2, h->d_ctrl,
                     s));
  h->launches += 2 + (spec ? 1 : 0);
  if (int r = pull_clock(h)) return r;
  const unsigned long long actual = h->clock.rate_bits0;
  if (h->clock.flags & kFlagNotClean) {
    // the reference data flow, from the uploaded cons
    if (int r = host_io_drain(h)) return r;
    h->clock = before;
    h->clock.rate_bits = 0;
    if (int r = push_clock(h)) return r;
    CK(cudaMemcpyAsync(h->pa.cons, h->buf[h->cur], 5 * n * sizeof(double),
                       cudaMemcpyDeviceToDevice, s));
    CK(prims_from_cons(g, h->pa, s));
    h->launches += 1;
    h->mode = 0;
    if (int r = bx_adindx_fill(h)) return r;
    if (int r = bx_step(h, endtime, ran)) return r;
    return bx_download(h, cons_out, nullptr, nullptr);
  }
  h->mode = 1;
  if (!runs) {
    if (int r = host_io_drain(h)) return r;
    h->clock.rate_bits = actual;
    h->clock.flags = 0;
    if (int r = push_clock(h)) return r;
    return bx_download(h, cons_out, nullptr, nullptr);
  }
  if (!spec || actual != before.rate_bits) {
    // dt from the uploaded state's own rate: start the step over
    if (int r = host_io_drain(h)) return r;
    h->clock = before;
    h->clock.rate_bits = actual;
    if (int r = push_clock(h)) return r;
    CK(launch_dt(h->d_ctrl, 1, s));
    CK(cudaEventRecord(ev_start, s));
    for (cudaStream_t x : h->hs) CK(cudaStreamWaitEvent(x, ev_start, 0));
    if (int r = host_io_enqueue(h, nullptr, cons_out, true)) return r;
    h->launches += 1;
  }
  CK(cudaEventRecord(ev_join, h->hs[3]));
  CK(cudaStreamWaitEvent(s, ev_join, 0));
  CK(launch_end(h->d_ctrl, 1, s));
  h->launches += 1;
  // the copies (and the conversions they wait for) finish before anything else
  // may touch the staging or cons_out
  if (int r = host_io_drain(h)) return r;
  Ctrl b = before;
  b.rate_bits = actual;
  if (int r = after_fused(h, b, ran, false)) return r;
  // a step redone on the per-phase kernels: its result replaces the copies
  if (h->last_path == 0) return bx_download(h, cons_out, nullptr, nullptr);
  return BX_OK;
}

int bx_profile(bx_handle* h, int32_t enable) {
  CHECK_H();
  if (enable && !h->ev[0])
    for (int k = 0; k < 3; ++k) CK(cudaEventCreate(&h->ev[k]));
  h->prof = enable != 0;
  h->ms_stage[0] = h->ms_stage[1] = 0.0;
  h->n_stage = 0;
  h->launches = 0;
  return BX_OK;
}

int bx_step_host_profile(bx_handle* h, int32_t enable) {
  CHECK_H();
  h->io_prof = enable != 0;
  return BX_OK;
}

int bx_step_host_timeline(bx_handle* h, int32_t* nslabs, double* ms) {
  CHECK_H();
  if (!nslabs) return set_err(h, BX_ERR_ARG, "nslabs is required");
  const int ns = (int)h->slabs.size();
  if (!ms) {
    *nslabs = ns;
    return BX_OK;
  }
  if (*nslabs < ns || h->io_tev.empty())
    return set_err(h, BX_ERR_STATE, "no profiled bx_step_host, or ms too short");
  *nslabs = ns;
  for (int k = 0; k < ns; ++k)
    for (int w = 0; w < kIoEv; ++w) {
      float t = 0.f;
      const cudaError_t e =
          cudaEventElapsedTime(&t, h->io_tev[0], h->io_tev[1 + (size_t)kIoEv * k + w]);
      ms[(size_t)kIoEv * k + w] = e == cudaSuccess ? t : -1.0;
      if (e != cudaSuccess) cudaGetLastError();
    }
  return BX_OK;
}

int bx_profile_read(bx_handle* h, double* ms_stage0, double* ms_stage1, int64_t* fused_steps,
                    int64_t* launches) {
  CHECK_H();
  if (ms_stage0) *ms_stage0 = h->ms_stage[0];
  if (ms_stage1) *ms_stage1 = h->ms_stage[1];
  if (fused_steps) *fused_steps = h->n_stage;
  if (launches) *launches = h->launches;
  return BX_OK;
}

}  // extern "C"

int bx_handle_start_from_planes(bx_handle* h, const double* planes) {
  CHECK_H();
  if (!planes || !h->pa.cons) return set_err(h, BX_ERR_ARG, "no planes or no reference arrays");
  const long long n = h->g.ng;
  cudaStream_t s = h->stream;
  CK(cudaMemcpyAsync(h->pa.cons, planes, 5 * n * sizeof(double), cudaMemcpyDeviceToDevice, s));
  for (int k = 0; k < 4; ++k)
    if (int r = ghost1(h)) return r;
  CK(prims_from_cons(h->g, h->pa, s));
  h->launches += 5;
  h->mode = 0;
  return bx_adindx_fill(h);
}

int bx_handle_adopt_fused(bx_handle* h, const double* planes, long long ps, int nsrc,
                          const Ctrl& clock) {
  const long long n = h->g.ng;
  for (int q = 0; q < 5; ++q)
    CK(cudaMemcpyAsync(h->buf[h->cur] + q * n, planes + q * ps, n * sizeof(double),
                       cudaMemcpyDeviceToDevice, h->stream));
  h->nsrc = nsrc;
  h->mode = 1;
  h->grav_step = false;
  h->p_saved = false;
  h->clock = clock;
  h->clock.flags = 0;
  h->clock.active = 0;
  h->clock.tripped = 0;
  h->clock.nsrc = 0;
  if (int r = push_clock(h)) return r;
  return BX_OK;
}

extern "C" {

int bx_ghost_plan(const bx_params* params, int64_t* nghost, int32_t* dst, int32_t* src1,
                  uint8_t* sgn1, int32_t* src2, uint8_t* sgn2, int32_t* fused_ok) {
  if (!params || !nghost) return set_err(nullptr, BX_ERR_ARG, "null argument");
  const bx_params& P = *params;
  if (P.nx < 5 || P.ny < 5 || P.nz < 1) return set_err(nullptr, BX_ERR_ARG, "grid too small");
  // the plan holds int32 cell indices
  if ((long long)P.nx * P.ny * P.nz >= (1ll << 31))
    return set_err(nullptr, BX_ERR_ARG, "grid exceeds 2^31 cells");
  GhostTable T;
  build_ghost_tables(P, T);
  const size_t n = T.dst.size();
  if (dst) {
    if ((size_t)*nghost < n) return set_err(nullptr, BX_ERR_ARG, "output arrays too small");
    std::memcpy(dst, T.dst.data(), n * sizeof(int32_t));
    if (src1) std::memcpy(src1, T.src1.data(), n * sizeof(int32_t));
    if (sgn1) std::memcpy(sgn1, T.sgn1.data(), n);
    if (src2) std::memcpy(src2, T.src2.data(), n * sizeof(int32_t));
    if (sgn2) std::memcpy(sgn2, T.sgn2.data(), n);
  }
  *nghost = (int64_t)n;
  if (fused_ok)
    *fused_ok = (T.resolved2 && T.face_rule_ok && !(P.flags & BX_FLAG_PHASE_ONLY)) ? 1 : 0;
  return BX_OK;
}

// Up to kRunChunk steps on the fused form without a host round trip per step:
// the batched path's clock kernels save the clock at each step's start; a step
// whose guard fires (limiter, low density, non-finite) restores it and
// deactivates the rest of the run, its input planes untouched, and so does
// the end time.  *taken = steps committed; *tripped = a step is to be redone.
static constexpr int kRunChunk = 32;
static int fused_run(bx_handle* h, double endtime, int64_t nsteps, int64_t* taken,
                     bool* tripped) {
  *taken = 0;
  *tripped = false;
  const Geom& g = h->g;
  cudaStream_t s = h->stream;
  const int K = (int)std::min<int64_t>(nsteps, kRunChunk);
  h->clock.endtime = endtime;
  h->clock.flags = 0;
  h->clock.tripped = 0;
  h->clock.run_step = 0;
  if (int r = push_clock(h)) return r;
  const long long step0 = h->clock.step;
  const int cur0 = h->cur;
  StageArgs a{};
  a.ctrl = h->d_ctrl;
  a.geom = h->d_geom;
  a.tiles = h->d_tiles;
  a.ncells_total = g.ng;
  a.eos = h->pa.eos;
  a.U = h->pa.u;
  a.G = h->gforce_set ? h->pa.gforce : nullptr;
  a.UC = h->pa.cons_old;
  const bool p2 = g.pow2 != 0, t3 = g.threed != 0;
  auto enqueue = [&]() -> cudaError_t {
    int cur = cur0;
    for (int k = 0; k < K; ++k) {
      cudaError_t e = launch_dt_batch(h->d_ctrl, 1, s);
      a.nsrc = k == 0 ? h->nsrc : (h->gforce_set ? 1 : 2);
      a.X = h->buf[cur];
      a.Y = nullptr;
      a.out = h->buf[(cur + 1) % 3];
      if (e == cudaSuccess) e = launch_stage(0, p2, t3, a, h->ntiles, s, h->shape);
      a.Y = h->buf[(cur + 1) % 3];
      a.out = h->buf[(cur + 2) % 3];
      if (e == cudaSuccess) e = launch_stage(1, p2, t3, a, h->ntiles, s, h->shape);
      if (e == cudaSuccess) e = launch_end_batch(h->d_ctrl, 1, s);
      if (e != cudaSuccess) return e;
      cur = (cur + 2) % 3;
    }
    return cudaSuccess;
  };
  if (K == kRunChunk && !h->gforce_set) {
    // whole chunks replay a CUDA graph per (input plane set, pending sources):
    // the launches of a chunk cost less than the work of a small grid
    const int key = cur0 + 3 * (h->nsrc - 1);
    if (!h->run_graph[key]) {
      cudaGraph_t graph = nullptr;
      CK(cudaStreamBeginCapture(s, cudaStreamCaptureModeRelaxed));
      const cudaError_t e = enqueue();
      const cudaError_t e2 = cudaStreamEndCapture(s, &graph);
      CK(e);
      CK(e2);
      const cudaError_t e3 = cudaGraphInstantiate(&h->run_graph[key], graph, 0);
      cudaGraphDestroy(graph);
      CK(e3);
    }
    CK(cudaGraphLaunch(h->run_graph[key], s));
  } else {
    CK(enqueue());
  }
  h->launches += 4 * K;
  if (int r = pull_clock(h)) return r;
  const long long m = h->clock.step - step0;
  *taken = m;
  *tripped = h->clock.tripped != 0;
  if (m > 0) {
    h->cur = (int)((cur0 + 2 * m) % 3);
    h->nsrc = h->gforce_set ? 1 : 2;
    h->grav_step = h->gforce_set;
    h->p_saved = false;
    h->last_path = 1;
  }
  h->clock.flags = 0;
  h->clock.tripped = 0;
  h->clock.active = 0;
  return push_clock(h);
}

int bx_run(bx_handle* h, double endtime, int64_t nsteps, int64_t* steps_taken) {
  CHECK_H();
  int64_t n = 0;
  int rc = BX_OK;
  while (n < nsteps) {
    if (h->mode == 1 && !h->prof) {
      int64_t m = 0;
      bool tripped = false;
      rc = fused_run(h, endtime, nsteps - n, &m, &tripped);
      if (rc != BX_OK) break;
      n += m;
      if (!tripped) {
        if (m < std::min<int64_t>(nsteps - n + m, kRunChunk)) break;  // end time or step cap
        continue;
      }
      // the tripped step: bx_step takes it again (on the per-phase kernels)
    }
    int32_t ran = 0;
    rc = bx_step(h, endtime, &ran);
    if (rc != BX_OK || !ran) break;
    ++n;
  }
  if (steps_taken) *steps_taken = n;
  return rc;
}

}  // extern "C"

// bx_batch.cu -- many independent grids ("boxes") advanced together.
//
// All boxes share three pooled plane sets (each box's cells at its own offset),
// one table of per-box geometry and clocks, and one tile list that covers every
// box: TX x TY interior column tiles (z split into chunks of at most 32 planes for
// large boxes), ordered by decreasing work so that the block scheduler hands the
// longest tiles out first.  A step is four launches for the whole ensemble --
// per-box dt control, stage 0, stage 1, per-box clock advance -- the same stage
// kernels as the single-grid path, so each box evolves bit for bit as it would
// alone.  A run of n steps is captured once into a CUDA graph and replayed.
//
// Each box keeps its own dt, time and step.  A box whose step raises a guard
// (velocity limiter, low-density EOS branch, non-finite values) is frozen by
// k_end_batch with its planes holding that step's input; after the run it
// continues on a single-grid handle, which redoes the step with the per-phase
// kernels exactly as bx_step would.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <map>
#include <string>
#include <tuple>
#include <vector>

#include "bx_handle.h"
#include "bx_internal.h"

using namespace bx;


namespace {

struct Shape {
  int nghost = 0;
  int32_t *dst = nullptr, *src2 = nullptr;
  uint8_t* sgn2 = nullptr;
  bool eligible = false;
};

}  // namespace

struct bx_batch {
  int nbox = 0;
  std::vector<bx_params> P;
  std::vector<Geom> G;
  std::vector<int> shape_of;
  std::vector<Shape> shapes;
  long long N = 0;  // cells in the pool (plane stride)
  long long max_ng = 0;
  double* buf[3] = {nullptr, nullptr, nullptr};
  double* ubuf = nullptr;  // 3 planes: stage-0 velocity of every box
  int cur = 0;
  Geom* d_geom = nullptr;
  Ctrl* d_ctrl = nullptr;
  Ctrl* h_ctrl = nullptr;  // pinned, nbox
  Tile* d_tiles = nullptr;
  int ntiles = 0;
  int zc = 0;  // tile depth policy of the tile list (set_tiles)
  int shape = 0;  // tile shape of the stage kernels (Shape0: 32 x 8, Shape1: 16 x 16)
  bool pow2 = true, threed = true;
  int pm = 1;  // 1: all boxes have power-of-two spacings; 0: otherwise (cdiv, exact for any)
  PhaseArrays scratch{};  // reference arrays of the largest box (downloads)
  double* staging = nullptr;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  std::vector<bx_handle*> solo;  // boxes continuing on their own handle
  cudaGraphExec_t graph = nullptr;
  int graph_steps = -1, graph_cur = -1;
  bool graph_persistent = false;
  std::vector<int> step_x;  // X plane set of each step of the last run
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  double last_ms = 0.0;
  long long last_launches = 0;
  // persistent mode: one launch per run works through (step, stage, tile) items
  bool persistent = false;
  int* d_tiles_of_box = nullptr;
  unsigned *d_done0 = nullptr, *d_done1 = nullptr, *d_ready = nullptr;
  unsigned long long* d_head = nullptr;
  int* d_pstatus = nullptr;
  long long poll_limit = 1ll << 24;  // about 2-4 s per wait: no run waits that long
  std::string err;
};

// the message of the calling thread's last failed call made without a handle
static thread_local std::string g_batch_err;

#define BCK(expr)                                                     \
  do {                                                                \
    cudaError_t e_ = (expr);                                          \
    if (e_ != cudaSuccess) {                                          \
      b->err = std::string(#expr) + ": " + cudaGetErrorString(e_);    \
      return e_ == cudaErrorMemoryAllocation ? BX_ERR_NOMEM : BX_ERR_CUDA; \
    }                                                                 \
  } while (0)

static int berr(bx_batch* b, int code, const std::string& m) {
  if (b) b->err = m;
  else g_batch_err = m;
  return code;
}

static int pull_ctrl(bx_batch* b) {
  BCK(cudaMemcpyAsync(b->h_ctrl, b->d_ctrl, b->nbox * sizeof(Ctrl), cudaMemcpyDeviceToHost,
                      b->stream));
  BCK(cudaStreamSynchronize(b->stream));
  return BX_OK;
}
static int push_ctrl(bx_batch* b) {
  BCK(cudaMemcpyAsync(b->d_ctrl, b->h_ctrl, b->nbox * sizeof(Ctrl), cudaMemcpyHostToDevice,
                      b->stream));
  BCK(cudaStreamSynchronize(b->stream));
  return BX_OK;
}

extern "C" {

int bx_batch_destroy(bx_batch* b);

const char* bx_batch_last_error(bx_batch* b) { return b ? b->err.c_str() : g_batch_err.c_str(); }

// Tiles of every box, longest first.  zc: the z extent of a column tile
// (interior planes; capped at each box's depth), or 0 for the default rule: a
// tile marches through the whole box depth when the ensemble has enough
// columns to fill the GPU many times over (no z warm-up repeated per chunk),
// else depths are cut into chunks of 32 planes.
static std::vector<Tile> batch_tiles(const bx_batch* b, int zc_req, int shape) {
  const int TX = shape_tx(shape), TY = shape_ty(shape);
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  long long ncol = 0;
  for (int i = 0; i < b->nbox; ++i) {
    const Geom& g = b->G[i];
    ncol += (long long)((g.ax1 - g.ax0 + TX - 1) / TX) * ((g.ay1 - g.ay0 + TY - 1) / TY);
  }
  const bool whole =
      ncol >= 16ll * sms * std::max(1, stage_blocks_per_sm(1, b->pm, b->threed, shape));
  std::vector<std::pair<long long, Tile>> tl;
  for (int i = 0; i < b->nbox; ++i) {
    const Geom& g = b->G[i];
    const int NAx = g.ax1 - g.ax0, NAy = g.ay1 - g.ay0, NAz = g.az1 - g.az0;
    int zc = 1;
    if (g.threed) zc = zc_req > 0 ? std::min(NAz, zc_req) : (whole ? NAz : std::min(NAz, 32));
    for (int z = 0; z < NAz; z += zc)
      for (int y = 0; y < NAy; y += TY)
        for (int x = 0; x < NAx; x += TX) {
          const int z1 = std::min(NAz, z + zc);
          const long long work = (long long)(z1 - z + (g.threed ? 1 : 0)) *
                                 std::min(TX, NAx - x) * std::min(TY, NAy - y);
          tl.push_back({work, Tile{i, x, y, z, z1}});
        }
  }
  std::stable_sort(tl.begin(), tl.end(),
                   [](const auto& a, const auto& c) { return a.first > c.first; });
  std::vector<Tile> tiles(tl.size());
  for (size_t k = 0; k < tl.size(); ++k) tiles[k] = tl[k].second;
  return tiles;
}

// (re)build the device tile list; a captured run graph holds the old one
static int set_tiles(bx_batch* b, int zc_req, int shape) {
  const std::vector<Tile> tiles = batch_tiles(b, zc_req, shape);
  if (b->graph) {
    cudaGraphExecDestroy(b->graph);
    b->graph = nullptr;
    b->graph_steps = -1;
  }
  cudaFree(b->d_tiles);
  b->d_tiles = nullptr;
  b->ntiles = (int)tiles.size();
  BCK(cudaMalloc(&b->d_tiles, tiles.size() * sizeof(Tile)));
  BCK(cudaMemcpy(b->d_tiles, tiles.data(), tiles.size() * sizeof(Tile), cudaMemcpyHostToDevice));
  std::vector<int> per_box(b->nbox, 0);
  for (const Tile& t : tiles) per_box[t.box] += 1;
  if (!b->d_tiles_of_box) BCK(cudaMalloc(&b->d_tiles_of_box, b->nbox * sizeof(int)));
  BCK(cudaMemcpy(b->d_tiles_of_box, per_box.data(), b->nbox * sizeof(int),
                 cudaMemcpyHostToDevice));
  b->zc = zc_req;
  b->shape = shape;
  return BX_OK;
}

int bx_batch_create(int32_t nbox, const bx_params* params, bx_batch** out) {
  if (nbox <= 0 || !params || !out) return berr(nullptr, BX_ERR_ARG, "bad arguments");
  bx_batch* b = new bx_batch();
  b->nbox = nbox;
  b->P.assign(params, params + nbox);
  b->G.resize(nbox);
  b->shape_of.resize(nbox);
  b->solo.assign(nbox, nullptr);
  std::map<std::tuple<int, int, int, int>, int> shape_index;
  long long off = 0;
  for (int i = 0; i < nbox; ++i) {
    const bx_params& P = b->P[i];
    if (P.h2stat != -1 || P.fluxangmom || P.nx < 5 || P.ny < 5 || P.nz < 1 ||
        (long long)P.nx * P.ny * P.nz >= (1ll << 31) ||  // int32 cell indices of the plans
        !(P.dx >= 1e-40 && P.dx <= 1e40 && P.dy >= 1e-40 && P.dy <= 1e40 && P.dz >= 1e-40 &&
          P.dz <= 1e40 && P.gammafix > 1.0 && P.cfl > 0)) {
      bx_batch_destroy(b);
      return berr(nullptr, BX_ERR_UNSUPPORTED, "box " + std::to_string(i) +
                                                   ": unsupported or invalid parameters");
    }
    fill_geom(P, b->G[i]);
    b->G[i].base = off;
    off += b->G[i].ng;
    b->max_ng = std::max(b->max_ng, b->G[i].ng);
    b->pow2 = b->pow2 && b->G[i].pow2;
    int wbits = 0;
    for (int k = 0; k < 6; ++k) wbits |= (P.no_outflow[k] ? 1 : 0) << k;
    auto key = std::make_tuple(P.nx, P.ny, P.nz, wbits);
    auto it = shape_index.find(key);
    if (it == shape_index.end()) {
      GhostTable T;
      build_ghost_tables(P, T);
      Shape sh;
      sh.nghost = (int)T.dst.size();
      sh.eligible = T.resolved2 && T.face_rule_ok;
      if (!sh.eligible) {
        bx_batch_destroy(b);
        return berr(nullptr, BX_ERR_UNSUPPORTED,
                    "box " + std::to_string(i) +
                        ": its ghost fill does not resolve within two sweeps (reflective "
                        "walls with nz>=6); run it with bx_create");
      }
      const size_t n = std::max(1, sh.nghost);
      if (cudaMalloc(&sh.dst, n * 4) != cudaSuccess || cudaMalloc(&sh.src2, n * 4) != cudaSuccess ||
          cudaMalloc(&sh.sgn2, n) != cudaSuccess) {
        b->shapes.push_back(sh);
        bx_batch_destroy(b);
        return berr(nullptr, BX_ERR_NOMEM, "ghost tables");
      }
      cudaMemcpy(sh.dst, T.dst.data(), sh.nghost * 4, cudaMemcpyHostToDevice);
      cudaMemcpy(sh.src2, T.src2.data(), sh.nghost * 4, cudaMemcpyHostToDevice);
      cudaMemcpy(sh.sgn2, T.sgn2.data(), sh.nghost, cudaMemcpyHostToDevice);
      it = shape_index.emplace(key, (int)b->shapes.size()).first;
      b->shapes.push_back(sh);
    }
    b->shape_of[i] = it->second;
    if (b->G[i].threed != b->G[0].threed) {
      bx_batch_destroy(b);
      return berr(nullptr, BX_ERR_UNSUPPORTED, "all boxes must be 3-D (nz>=6) or all 2-D");
    }
  }
  b->threed = b->G[0].threed != 0;
  {
    int np2 = 0;
    for (int i = 0; i < nbox; ++i) np2 += b->G[i].pow2 ? 1 : 0;
    b->pm = np2 == nbox ? 1 : 0;
  }
  b->N = off;
  auto fail = [&](int code) {
    g_batch_err = b->err;
    bx_batch_destroy(b);
    return code;
  };
  int rc;
#define BCKC(expr)                 \
  do {                             \
    if ((rc = [&]() { BCK(expr); return 0; }()) != 0) return fail(rc); \
  } while (0)
  BCKC(cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking));
  b->own_stream = true;
  for (int k = 0; k < 3; ++k) BCKC(cudaMalloc(&b->buf[k], 5 * b->N * sizeof(double)));
  BCKC(cudaMalloc(&b->ubuf, 3 * b->N * sizeof(double)));
  BCKC(cudaMalloc(&b->d_geom, nbox * sizeof(Geom)));
  BCKC(cudaMemcpy(b->d_geom, b->G.data(), nbox * sizeof(Geom), cudaMemcpyHostToDevice));
  BCKC(cudaMalloc(&b->d_ctrl, nbox * sizeof(Ctrl)));
  BCKC(cudaMallocHost(&b->h_ctrl, nbox * sizeof(Ctrl)));
  std::memset(b->h_ctrl, 0, nbox * sizeof(Ctrl));
  for (int i = 0; i < nbox; ++i) {
    b->h_ctrl[i].cfl = b->P[i].cfl;
    b->h_ctrl[i].endtime = 1e300;
    b->h_ctrl[i].max_step = (1ll << 62);
    b->h_ctrl[i].nsrc = 1;
  }
  BCKC(cudaMemcpy(b->d_ctrl, b->h_ctrl, nbox * sizeof(Ctrl), cudaMemcpyHostToDevice));
  if (int r = set_tiles(b, 0, 0)) return fail(r);
  // reference arrays for downloads, sized for the largest box
  const long long m = b->max_ng;
  BCKC(cudaMalloc(&b->scratch.cons, 5 * m * sizeof(double)));
  BCKC(cudaMalloc(&b->scratch.u, 3 * m * sizeof(double)));
  BCKC(cudaMalloc(&b->scratch.p, m * sizeof(double)));
  BCKC(cudaMalloc(&b->scratch.adindx, m * sizeof(double)));
  BCKC(cudaMalloc(&b->staging, 5 * m * sizeof(double)));
  BCKC(cudaEventCreate(&b->ev0));
  BCKC(cudaEventCreate(&b->ev1));
  BCKC(cudaMalloc(&b->d_done0, nbox * sizeof(unsigned)));
  BCKC(cudaMalloc(&b->d_done1, nbox * sizeof(unsigned)));
  BCKC(cudaMalloc(&b->d_ready, nbox * sizeof(unsigned)));
  BCKC(cudaMalloc(&b->d_head, sizeof(unsigned long long)));
  BCKC(cudaMalloc(&b->d_pstatus, sizeof(int)));
  for (int sh = 0; sh < kNumShapes; ++sh) {  // sets the shared-memory attributes
    stage_blocks_per_sm(0, b->pm, b->threed, sh);
    stage_blocks_per_sm(1, b->pm, b->threed, sh);
  }
#undef BCKC
  *out = b;
  return BX_OK;
}

int bx_batch_destroy(bx_batch* b) {
  if (!b) return BX_OK;
  if (b->stream) cudaStreamSynchronize(b->stream);
  if (b->graph) cudaGraphExecDestroy(b->graph);
  for (auto* h : b->solo)
    if (h) bx_destroy(h);
  for (auto& s : b->shapes) {
    cudaFree(s.dst);
    cudaFree(s.src2);
    cudaFree(s.sgn2);
  }
  for (int k = 0; k < 3; ++k) cudaFree(b->buf[k]);
  cudaFree(b->ubuf);
  cudaFree(b->d_geom);
  cudaFree(b->d_ctrl);
  if (b->h_ctrl) cudaFreeHost(b->h_ctrl);
  cudaFree(b->d_tiles);
  cudaFree(b->d_tiles_of_box);
  cudaFree(b->d_done0);
  cudaFree(b->d_done1);
  cudaFree(b->d_ready);
  cudaFree(b->d_head);
  cudaFree(b->d_pstatus);
  cudaFree(b->scratch.cons);
  cudaFree(b->scratch.u);
  cudaFree(b->scratch.p);
  cudaFree(b->scratch.adindx);
  cudaFree(b->staging);
  if (b->ev0) cudaEventDestroy(b->ev0);
  if (b->ev1) cudaEventDestroy(b->ev1);
  if (b->own_stream && b->stream) cudaStreamDestroy(b->stream);
  delete b;
  return BX_OK;
}

int bx_batch_set_stream(bx_batch* b, void* s) {
  if (!b) return BX_ERR_ARG;
  BCK(cudaStreamSynchronize(b->stream));
  if (b->own_stream && b->stream) cudaStreamDestroy(b->stream);
  b->own_stream = false;
  if (s) {
    b->stream = (cudaStream_t)s;
  } else {
    BCK(cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking));
    b->own_stream = true;
  }
  if (b->graph) {
    cudaGraphExecDestroy(b->graph);
    b->graph = nullptr;
  }
  return BX_OK;
}

int bx_batch_upload(bx_batch* b, int32_t box, const double* cons) {
  if (!b || box < 0 || box >= b->nbox || !cons) return berr(b, BX_ERR_ARG, "bad arguments");
  if (b->solo[box]) {
    bx_destroy(b->solo[box]);
    b->solo[box] = nullptr;
  }
  const Geom& g = b->G[box];
  const Shape& sh = b->shapes[b->shape_of[box]];
  const long long n = g.ng;
  double* X = b->buf[b->cur] + g.base;
  BCK(cudaMemcpyAsync(b->staging, cons, 5 * n * sizeof(double), cudaMemcpyHostToDevice,
                      b->stream));
  // (n,5) -> five planes of n, then each plane into the pool (plane stride N)
  BCK(aos_to_soa(b->staging, b->scratch.cons, n, 5, b->stream));
  for (int q = 0; q < 5; ++q)
    BCK(cudaMemcpyAsync(X + q * b->N, b->scratch.cons + q * n, n * sizeof(double),
                        cudaMemcpyDeviceToDevice, b->stream));
  if (int r = pull_ctrl(b)) return r;
  Ctrl& c = b->h_ctrl[box];
  c.flags = 0;
  c.rate_bits = 0;
  c.tripped = 0;
  c.nsrc = 1;
  if (int r = push_ctrl(b)) return r;
  BCK(box_check_clean(g, X, b->N, sh.nghost, sh.dst, sh.src2, sh.sgn2, b->d_ctrl + box,
                      b->stream));
  BCK(box_rate(g, X, b->N, b->d_ctrl + box, b->stream));
  if (int r = pull_ctrl(b)) return r;
  if (b->h_ctrl[box].flags & kFlagNotClean)
    return berr(b, BX_ERR_STATE,
                "box " + std::to_string(box) +
                    ": not a state the fused stages start from (needs rho >= 1e-4 and finite "
                    "values in the interior and ghosts equal to the two-sweep fill)");
  return BX_OK;
}

int bx_batch_set_clock(bx_batch* b, int32_t box, double time, double dtold, int64_t step) {
  if (!b || box < 0 || box >= b->nbox) return berr(b, BX_ERR_ARG, "bad arguments");
  if (int r = pull_ctrl(b)) return r;
  b->h_ctrl[box].time = time;
  b->h_ctrl[box].dtold = dtold;
  b->h_ctrl[box].step = step;
  return push_ctrl(b);
}

int bx_batch_get_clock(bx_batch* b, int32_t box, double* time, double* dt, double* dtold,
                       int64_t* step) {
  if (!b || box < 0 || box >= b->nbox) return berr(b, BX_ERR_ARG, "bad arguments");
  if (b->solo[box]) return bx_get_clock(b->solo[box], time, dt, dtold, step);
  if (int r = pull_ctrl(b)) return r;
  const Ctrl& c = b->h_ctrl[box];
  if (time) *time = c.time;
  if (dt) *dt = c.dt;
  if (dtold) *dtold = c.dtold;
  if (step) *step = c.step;
  return BX_OK;
}

static int enqueue_steps(bx_batch* b, int nsteps) {
  StageArgs a{};
  a.ctrl = b->d_ctrl;
  a.geom = b->d_geom;
  a.tiles = b->d_tiles;
  a.ncells_total = b->N;
  a.nsrc = 0;  // per box
  a.U = b->ubuf;
  int c = b->cur;
  b->step_x.assign(nsteps, 0);
  if (b->persistent) {
    // the first step's dt, then one launch for all steps and both stages
    for (int k = 0; k < nsteps; ++k) {
      b->step_x[k] = c;
      c = (c + 2) % 3;
    }
    BCK(launch_dt_batch(b->d_ctrl, b->nbox, b->stream));
    PersistArgs p{};
    p.a = a;
    for (int k = 0; k < 3; ++k) p.buf[k] = b->buf[k];
    p.cur = b->cur;
    p.nsteps = nsteps;
    p.ntiles = b->ntiles;
    p.tiles_of_box = b->d_tiles_of_box;
    p.done0 = b->d_done0;
    p.done1 = b->d_done1;
    p.ready = b->d_ready;
    p.head = b->d_head;
    p.status = b->d_pstatus;
    p.poll_limit = b->poll_limit;
    BCK(launch_batch_persistent(p, b->pm, b->threed, b->nbox, b->stream, nullptr, b->shape));
    return BX_OK;
  }
  for (int k = 0; k < nsteps; ++k) {
    const int X = c, Y = (c + 1) % 3, Z = (c + 2) % 3;
    b->step_x[k] = X;
    BCK(launch_dt_batch(b->d_ctrl, b->nbox, b->stream));
    a.X = b->buf[X];
    a.Y = nullptr;
    a.out = b->buf[Y];
    BCK(launch_stage(0, b->pm, b->threed, a, b->ntiles, b->stream, b->shape));
    a.Y = b->buf[Y];
    a.out = b->buf[Z];
    BCK(launch_stage(1, b->pm, b->threed, a, b->ntiles, b->stream, b->shape));
    BCK(launch_end_batch(b->d_ctrl, b->nbox, b->stream));
    c = Z;
  }
  return BX_OK;
}

int bx_batch_run(bx_batch* b, int64_t nsteps, double endtime, int32_t use_graph) {
  if (!b || nsteps < 0) return berr(b, BX_ERR_ARG, "bad arguments");
  if (nsteps == 0) return BX_OK;
  if (int r = pull_ctrl(b)) return r;
  std::vector<long long> step_at_start(b->nbox);
  for (int i = 0; i < b->nbox; ++i) {
    Ctrl& c = b->h_ctrl[i];
    c.endtime = endtime;
    c.flags = 0;
    c.run_step = 0;
    c.max_step = (1ll << 62);
    step_at_start[i] = c.step;
  }
  if (int r = push_ctrl(b)) return r;
  const int ns = (int)nsteps;
  BCK(cudaEventRecord(b->ev0, b->stream));
  if (use_graph) {
    if (!b->graph || b->graph_steps != ns || b->graph_cur != b->cur ||
        b->graph_persistent != b->persistent) {
      if (b->graph) {
        cudaGraphExecDestroy(b->graph);
        b->graph = nullptr;
      }
      cudaGraph_t gr;
      BCK(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
      const int rc = enqueue_steps(b, ns);
      cudaError_t e = cudaStreamEndCapture(b->stream, &gr);
      if (rc) return rc;
      BCK(e);
      e = cudaGraphInstantiate(&b->graph, gr, 0);
      cudaGraphDestroy(gr);
      BCK(e);
      b->graph_steps = ns;
      b->graph_cur = b->cur;
      b->graph_persistent = b->persistent;
    } else {
      b->step_x.assign(ns, 0);
      int c = b->cur;
      for (int k = 0; k < ns; ++k) {
        b->step_x[k] = c;
        c = (c + 2) % 3;
      }
    }
    BCK(cudaGraphLaunch(b->graph, b->stream));
  } else {
    if (int r = enqueue_steps(b, ns)) return r;
  }
  BCK(cudaEventRecord(b->ev1, b->stream));
  BCK(cudaEventSynchronize(b->ev1));
  float ms = 0.f;
  BCK(cudaEventElapsedTime(&ms, b->ev0, b->ev1));
  b->last_ms = ms;
  b->last_launches = b->persistent ? 3 : 4ll * ns;
  if (b->persistent) {
    int st = 0;
    BCK(cudaMemcpy(&st, b->d_pstatus, sizeof(int), cudaMemcpyDeviceToHost));
    if (st)
      return berr(b, BX_ERR_STATE,
                  "persistent run: a wait on another tile's result gave up after the poll "
                  "limit; the run's results are not valid");
  }
  for (int k = 0; k < ns; ++k) b->cur = (b->cur + 2) % 3;
  if (int r = pull_ctrl(b)) return r;
  // boxes that left the fused path (or already had) continue on their own handles
  for (int i = 0; i < b->nbox; ++i) {
    Ctrl& c = b->h_ctrl[i];
    long long left = 0;
    if (!b->solo[i] && c.tripped) {
      bx_handle* h = nullptr;
      if (int r = bx_create(&b->P[i], &h)) return berr(b, r, bx_last_error(nullptr));
      const int X = b->step_x[c.trip_step];
      const int nsrc = c.nsrc;
      Ctrl clk = c;
      clk.endtime = endtime;
      if (int r = bx_handle_adopt_fused(h, b->buf[X] + b->G[i].base, b->N, nsrc, clk)) {
        std::string m = bx_last_error(h);
        bx_destroy(h);
        return berr(b, r, m);
      }
      b->solo[i] = h;
      left = ns - (c.step - step_at_start[i]);
      c.tripped = 0;
      c.active = 0;
    } else if (b->solo[i]) {
      left = ns;
    }
    if (b->solo[i] && left > 0) {
      int64_t done = 0;
      if (int r = bx_run(b->solo[i], endtime, left, &done))
        return berr(b, r, bx_last_error(b->solo[i]));
    }
  }
  return BX_OK;
}

// Run configuration of the ensemble picked by measurement.  Each candidate tile
// shape (32 x 8 and 16 x 16 columns, both in 256-thread blocks; each has its own
// compiled shared-memory layout) and tile depth (the default rule, whole box
// depths, and 64, 32, 16 and 8 planes) runs `reps` trial steps from the boxes'
// current states -- a step reads the input plane set and writes the other two,
// and the clocks are put back after every trial, so the ensemble is left as it
// was -- with four launches per step; at the fastest shape and depth the
// persistent launch is timed the same way, and the faster of the two launch
// forms stays.  The halo is the stencil's two cells (a deeper halo would fuse
// the two stages at the cost of recomputing stage 0 on a two-cell ring around
// every tile, more FP64 work for a kernel that is bound by FP64 issue, not by
// memory traffic).
static int trial_ms(bx_batch* b, const std::vector<Ctrl>& saved, int reps, double* ms_out) {
  double ms_min = 1e300;
  for (int r = 0; r < reps; ++r) {
    for (int i = 0; i < b->nbox; ++i) {
      b->h_ctrl[i] = saved[i];
      b->h_ctrl[i].endtime = 1e300;
      b->h_ctrl[i].flags = 0;
      b->h_ctrl[i].run_step = 0;
    }
    if (int rc = push_ctrl(b)) return rc;
    BCK(cudaEventRecord(b->ev0, b->stream));
    if (int rc = enqueue_steps(b, 1)) return rc;
    BCK(cudaEventRecord(b->ev1, b->stream));
    BCK(cudaEventSynchronize(b->ev1));
    float ms = 0.f;
    BCK(cudaEventElapsedTime(&ms, b->ev0, b->ev1));
    ms_min = std::min(ms_min, (double)ms);
  }
  if (b->persistent) {
    int st = 0;
    BCK(cudaMemcpy(&st, b->d_pstatus, sizeof(int), cudaMemcpyDeviceToHost));
    if (st) return berr(b, BX_ERR_STATE, "persistent trial: a wait gave up");
  }
  *ms_out = ms_min;
  return BX_OK;
}

int bx_batch_autotune(bx_batch* b, int32_t reps, int32_t* zc_out, double* ms_out) {
  if (!b || reps < 1) return berr(b, BX_ERR_ARG, "bad arguments");
  if (int r = pull_ctrl(b)) return r;
  const std::vector<Ctrl> saved(b->h_ctrl, b->h_ctrl + b->nbox);
  const int cand[] = {0, -1, 64, 32, 16, 8};
  int best = 0, best_shape = 0;
  double best_ms = 1e300;
  b->persistent = false;
  for (int sh = 0; sh < kNumShapes; ++sh) {
    for (int zc : cand) {
      // whole depths: a chunk no box exceeds
      const int zreq = zc < 0 ? (1 << 30) : zc;
      if (int r = set_tiles(b, zreq, sh)) return r;
      double ms = 0.0;
      if (int r = trial_ms(b, saved, reps, &ms)) return r;
      if (ms < best_ms) {
        best_ms = ms;
        best = zreq;
        best_shape = sh;
      }
    }
  }
  if (int r = set_tiles(b, best, best_shape)) return r;
  b->persistent = true;
  double pms = 0.0;
  if (int r = trial_ms(b, saved, reps, &pms)) return r;
  b->persistent = pms < best_ms;
  best_ms = std::min(best_ms, pms);
  std::copy(saved.begin(), saved.end(), b->h_ctrl);
  if (int r = push_ctrl(b)) return r;
  if (zc_out) *zc_out = best;
  if (ms_out) *ms_out = best_ms;
  return BX_OK;
}

int bx_batch_set_tile_shape(bx_batch* b, int32_t shape) {
  if (!b || shape < 0 || shape >= kNumShapes) return berr(b, BX_ERR_ARG, "bad arguments");
  return set_tiles(b, b->zc, shape);
}

int bx_batch_get_tile_shape(bx_batch* b, int32_t* shape, int32_t* tx, int32_t* ty,
                            int32_t* depth) {
  if (!b) return BX_ERR_ARG;
  if (shape) *shape = b->shape;
  if (tx) *tx = shape_tx(b->shape);
  if (ty) *ty = shape_ty(b->shape);
  if (depth) *depth = b->zc;
  return BX_OK;
}

int bx_batch_set_persistent(bx_batch* b, int32_t enable) {
  if (!b) return BX_ERR_ARG;
  b->persistent = enable != 0;
  if (b->graph) {
    cudaGraphExecDestroy(b->graph);
    b->graph = nullptr;
    b->graph_steps = -1;
  }
  return BX_OK;
}

int bx_batch_get_persistent(bx_batch* b, int32_t* enabled) {
  if (!b || !enabled) return BX_ERR_ARG;
  *enabled = b->persistent ? 1 : 0;
  return BX_OK;
}

int bx_batch_wait_selftest(int64_t poll_limit, int32_t* gave_up, double* ms) {
  if (poll_limit < 1 || !gave_up) return berr(nullptr, BX_ERR_ARG, "bad arguments");
  int g = 0;
  float t = 0.f;
  const cudaError_t e = persistent_wait_selftest(poll_limit, &g, &t);
  if (e != cudaSuccess) return berr(nullptr, BX_ERR_CUDA, cudaGetErrorString(e));
  *gave_up = g;
  if (ms) *ms = t;
  return BX_OK;
}

int bx_batch_download(bx_batch* b, int32_t box, double* cons, double* u, double* p) {
  if (!b || box < 0 || box >= b->nbox) return berr(b, BX_ERR_ARG, "bad arguments");
  if (b->solo[box]) return bx_download(b->solo[box], cons, u, p);
  if (int r = pull_ctrl(b)) return r;
  const Geom& g0 = b->G[box];
  Geom g = g0;
  g.base = 0;
  const Shape& sh = b->shapes[b->shape_of[box]];
  const long long n = g.ng;
  const int nsrc = b->h_ctrl[box].nsrc;
  BCK(fused_to_phase(g, b->buf[b->cur] + g0.base, nsrc, b->scratch, sh.nghost, sh.dst, sh.src2,
                     sh.sgn2, b->stream, b->N));
  if (cons) {
    BCK(soa_to_aos(b->scratch.cons, b->staging, n, 5, b->stream));
    BCK(cudaMemcpyAsync(cons, b->staging, 5 * n * sizeof(double), cudaMemcpyDeviceToHost,
                        b->stream));
  }
  if (u) {
    BCK(soa_to_aos(b->scratch.u, b->staging, n, 3, b->stream));
    BCK(cudaMemcpyAsync(u, b->staging, 3 * n * sizeof(double), cudaMemcpyDeviceToHost,
                        b->stream));
  }
  if (p)
    BCK(cudaMemcpyAsync(p, b->scratch.p, n * sizeof(double), cudaMemcpyDeviceToHost, b->stream));
  BCK(cudaStreamSynchronize(b->stream));
  return BX_OK;
}

int bx_batch_info(bx_batch* b, double* last_run_ms, int64_t* launches, int32_t* n_solo,
                  int64_t* cells) {
  if (!b) return BX_ERR_ARG;
  if (last_run_ms) *last_run_ms = b->last_ms;
  if (launches) *launches = b->last_launches;
  if (n_solo) {
    int k = 0;
    for (auto* h : b->solo) k += h ? 1 : 0;
    *n_solo = k;
  }
  if (cells) *cells = b->N;
  return BX_OK;
}

}  // extern "C"

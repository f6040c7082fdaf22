// bx_handle.h -- the handle behind the opaque bx_handle of the C ABI (private).
#pragma once
#include <cuda_runtime.h>

#include <string>
#include <vector>

#include "bx_internal.h"

// timing events per slab of a profiled bx_step_host: upload start, upload end,
// stage 0 enqueued after that upload, the slab's stage 1 end, its conversion end,
// download start, download end
constexpr int kIoEv = 7;

struct bx_handle {
  bx_params P{};
  bx::Geom g{};
  bx::GhostTable T;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  double* buf[3] = {nullptr, nullptr, nullptr};
  int cur = 0;
  int nsrc = 1;
  bx::PhaseArrays pa{};
  int nghost = 0;
  int32_t *d_dst = nullptr, *d_src1 = nullptr, *d_src2 = nullptr;
  uint8_t *d_sgn1 = nullptr, *d_sgn2 = nullptr;
  bx::Geom* d_geom = nullptr;
  bx::Tile* d_tiles = nullptr;
  int ntiles = 0;
  bx::Ctrl* d_ctrl = nullptr;
  bx::Ctrl* h_ctrl = nullptr;  // pinned mirror
  bx::Ctrl clock{};            // host copy of the clock after the last completed call
  int mode = 0;            // 0 = reference arrays current, 1 = fused planes current
  // the last fused step had a force: the planes hold the state after source(1)
  // (nsrc 1) and pa.cons_old the velocity after flux(1) that state() reads
  bool grav_step = false;
  // the planes took the reference arrays and no fused step ran since: their p
  // (kept in pa.cons_old's fourth plane) is the one to give back
  bool p_saved = false;
  bool eligible = false;
  // the grid's ghost plan and flags admit the fused kernels; eligible adds the
  // physics: with the tabulated EOS (tile shape 2) once the tables are set and
  // nz != 1, with the tabulated EOS or flux_ang (shape 3) not while a force is
  // set (update_eligible)
  bool fusable = false;
  int shape = 0;  // stage-kernel tile shape of the single-grid launches
  bool gforce_set = false;
  uint32_t status = 0;
  int last_path = 0;
  // profiling: CUDA events around the stage launches, accumulated per step
  bool prof = false;
  cudaEvent_t ev[3] = {nullptr, nullptr, nullptr};
  double ms_stage[2] = {0.0, 0.0};
  long long n_stage = 0;
  long long launches = 0;  // kernels of this library launched on the handle's stream
  double* d_eos = nullptr;  // device copy of the tabulated EOS (H2STAT >= 0)
  // avisc: the hydro namelist's avmagx, avmagy, avmagz and the qq array (3
  // planes, made by the first bx_avisc)
  double avmag[3] = {0.0, 0.0, 0.0};
  double* d_qq = nullptr;
  // bx_step_host: its tiles (thin z-chunks), the z slabs of the cell range
  // (groups of those chunks) with their ghost ranges, and the streams and
  // events that overlap the copies with the step (made on first use)
  bx::Tile* d_io_tiles = nullptr;
  struct Slab {
    long long i0, i1;  // cells [i0, i1)
    int g0, g1;        // entries [g0, g1) of the ghost plan
    int t0, nt;        // tiles [t0, t0 + nt)
    int z0, z1;        // interior-relative z range of the tiles
    int s0_after, s1_after;  // uploaded slab after which its stage 0 / stage 1 can run
  };
  std::vector<Slab> slabs;
  // upload copies, download copies, conversions, second stage-1 stream
  cudaStream_t hs[4] = {nullptr, nullptr, nullptr, nullptr};
  std::vector<cudaEvent_t> hev;  // start, join, then per slab: in, stage 0, stage 1, converted
  // bx_step_host_profile: timing events, the start and per slab the upload's
  // start and end, stage 0 enqueued after it, the slab's stage 1, conversion and
  // the download's start and end (kIoEv each)
  bool io_prof = false;
  std::vector<cudaEvent_t> io_tev;
  // bx_run: CUDA graphs of a whole chunk of force-free steps, per input plane
  // set (3) and pending sources (1 or 2)
  cudaGraphExec_t run_graph[6] = {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};
  std::string err;
};

// a handle with geometry, ghost tables, tiles, control block and stream but no
// state planes (for engines that hold their own planes)
int bx_create_lean(const bx_params* params, bx_handle** out);
// Take over a fused state held elsewhere on the device: the five conserved
// planes of one grid (plane stride `ps`), `nsrc` sources short of the
// reference state, with the given clock.  The batched path uses it to continue
// a box on a handle of its own.
int bx_handle_adopt_fused(bx_handle* h, const double* planes, long long ps, int nsrc,
                          const bx::Ctrl& clock);
// Start the reference arrays of h from the five conserved planes (plane stride
// ngrid) on the device: two calls of the ghost fill (four sweeps, so every
// ghost the sweeps reach is set from the interior, whatever the planes held
// there), u = m/rho and state()'s pressure; the handle's next step then runs on
// the per-phase kernels unless the grid takes the fused ones.
int bx_handle_start_from_planes(bx_handle* h, const double* planes);

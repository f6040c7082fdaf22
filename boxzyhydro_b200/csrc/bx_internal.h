// bx_internal.h -- device data layout and launch interfaces of the hydro step.
//
// HBM layout: every grid is held as five SoA planes of FP64 (rho, m1, m2, m3, E),
// each ng = nx*ny*nz doubles in the reference's cell order (x fastest), so a
// warp touching 32 consecutive x cells moves 256 contiguous bytes per field.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <string>
#include <vector>

#include "../../include/boxzy_gpu.h"

namespace bx {

// status bits raised on the device (BX_STATUS_* mirror these in the C header)
enum : unsigned {
  kFlagVlimit = 1u << 0,   // |u_i| > vlimit somewhere: velocity limiter rewrites cons
  kFlagLowRho = 1u << 1,   // rho < 1e-4 somewhere: low-density EOS branch
  kFlagNonFinite = 1u << 2,
  kFlagZeroWave = 1u << 3, // ap+am == 0 in an HLL face (reference divides by zero)
  kFlagNotClean = 1u << 4, // uploaded arrays are not a state the fused stages can start from
};

// main.f90 clock held on the device (time, dt, dtold, step) plus the Courant
// accumulator and guard flags of the step in flight.
struct Ctrl {
  double time;
  double dt;          // full step dt (main.f90:342)
  double dtold;       // main.f90:270-271
  double endtime;
  double rate;        // last reduced dtrate (courant.f90:22)
  unsigned long long rate_bits;  // atomicMax accumulator (bit image of a double >= 0)
  long long step;
  long long max_step;
  unsigned int flags;
  int active;         // 1 while the step in flight is to be taken
  double cfl;
  // batched path: sources the planes are short of (0 = use StageArgs::nsrc),
  // clock saved at step start, and whether the box left the fused path
  int nsrc;
  int tripped;        // 1: a guard fired; the box's planes hold the tripped step's input
  long long trip_step;  // batch step index (within the run) of the trip
  double time0, dtold0;
  long long step0;
  unsigned long long rate_bits0;
  long long run_step;   // steps launched in the current run (for trip_step)
};

// Geometry and constants of one box (one reference grid).
struct Geom {
  int nx, ny, nz;          // with ghosts
  int ax0, ax1, ay0, ay1, az0, az1;  // interior [a0,a1) per axis (0-based)
  long long sy, sz;        // strides (1, nx, nx*ny)
  long long ng;            // cells
  long long base;          // offset of this box's cells in the pooled buffers
  int wall[6];             // reflective wall flags xl,xr,yl,yr,zl,zr (after nz<6 rule)
  int threed;              // nz >= 6
  int pow2;                // dx,dy,dz all powers of two
  double dx, dy, dz, idx, idy, idz;
  double ayz, axz, axy, vol, ivol;
  double gam, gm1, small_rho, small_eps, vlimit, cfl;
  double muc, rgas;
  int ang;                 // flux_ang.f90 in place of flux.f90 (fluxangmom)
  int tab;                 // tabulated EOS (H2STAT >= 0)
  double yoff;             // yoffset of the angular-momentum transforms
};

// Work item of the tiled stage kernel: one 32x8 column tile and a z range of a box.
struct Tile {
  int box;
  int x0, y0;     // interior-relative tile origin
  int z0, z1;     // interior-relative z range [z0,z1) (for nz<6: plane range)
};

// Stage-kernel tile: TX x TY interior columns per block of NT threads (NT may
// exceed the tile: the threads without a column of their own take halo work).
// 32x8 in 256 threads measured 5 % faster on B200 than 16x14 in 256 threads
// (although the latter fits the x/y face-state and face-flux phases into two
// passes of the block instead of three: the wider rows load whole 256-byte
// segments and need fewer halo columns) and 2 % faster than 32x16 in 512
// threads (one block per SM: its barriers have no second block to hide them).
#ifndef BX_TX
#define BX_TX 32
#endif
#ifndef BX_TY
#define BX_TY 8
#endif
#ifndef BX_NT
#define BX_NT 256
#endif
constexpr int TX = BX_TX;
constexpr int TY = BX_TY;
constexpr int NT = BX_NT;
static_assert(TX * TY <= NT && NT % 32 == 0, "tile larger than the block");

// The stage kernels' tile shapes: TX_ x TY_ interior columns in a block of NT
// threads, and the shared-memory layout that follows from them (per z plane:
// primitives of the tile plus a two-cell halo, aliased with the x/y face
// fluxes; x and y face states; per-thread z-pipeline slots).  Shape 0 is the
// single-grid path's (TX x TY); the batched path's autotuner may pick shape 1.
template <int TX_, int TY_, int MODE_ = 0>
struct TileShape {
  static constexpr int TX = TX_, TY = TY_;
  static constexpr int NT = BX_NT;
  // MODE 1 (TAB): the tabulated EOS, whose gamma is a reconstructed primitive;
  // MODE 2 (ANG): angular-momentum fluxing, whose radial and angular momenta
  // are reconstructed primitives and whose x/y face fluxes of the two momentum
  // components depend on the updated cell (two versions per face)
  static constexpr bool TAB = MODE_ == 1, ANG = MODE_ == 2;
  static constexpr int NPF = TAB ? 8 : ANG ? 9 : 7;  // primitive fields
  static constexpr int NSF = TAB ? 7 : ANG ? 8 : 6;  // face-state fields
  static constexpr int NFQ = ANG ? 7 : 5;            // x/y face-flux quantities
  static constexpr int NOWN = TX * TY;               // threads with a column
  static constexpr int PW = TX + 4;          // prim plane width (x halo 2)
  static constexpr int NP = (TY + 4) * PW;   // prim plane cells
  static constexpr int NSX = TY * (TX + 2);  // x-state cells
  static constexpr int NSY = (TY + 2) * TX;  // y-state cells
  static constexpr int NFX = TY * (TX + 1);  // x faces
  static constexpr int NFY = (TY + 1) * TX;  // y faces
  // per-column z-pipeline slots (3-D): the z flux below and above the own cell
  // (5 + 5) and the plus z-state carried to the next plane (NSF), kept in
  // shared memory so the x/y phases have the registers
  static constexpr int NZS = 10 + NSF;
  // the face fluxes of the face and update phases alias the primitives
  static constexpr int NR0 = (NPF * NP > NFQ * (NFX + NFY)) ? NPF * NP : NFQ * (NFX + NFY);
  static constexpr int SMEM_DOUBLES = NR0 + 2 * NSF * NSX + 2 * NSF * NSY + NZS * NOWN;
  static_assert(TX * TY <= NT && NT % 32 == 0, "tile larger than the block");
  static_assert(4 * (TX + TY) <= NT, "one halo cell per thread and plane at most");
};
using Shape0 = TileShape<TX, TY>;
using Shape1 = TileShape<16, 16>;
// the tabulated EOS and angular-momentum fluxing (single grids only): 32 x 6
// columns, so the larger primitive and face-state sets still fit two blocks
// per SM
using Shape2 = TileShape<32, 6, 1>;
using Shape3 = TileShape<32, 6, 2>;
constexpr int kNumShapes = 2;  // the shapes the batched autotuner chooses among
// the x and y extents of tile shape `shape`
inline int shape_tx(int shape) {
  return shape == 3 ? Shape3::TX : shape == 2 ? Shape2::TX : shape == 1 ? Shape1::TX : Shape0::TX;
}
inline int shape_ty(int shape) {
  return shape == 3 ? Shape3::TY : shape == 2 ? Shape2::TY : shape == 1 ? Shape1::TY : Shape0::TY;
}

// ghost-fill tables: per ghost (index order), destination cell, source cell and
// momentum sign mask (bit0: m1, bit1: m2, bit2: m3 negated).
struct GhostTable {
  std::vector<int32_t> dst;
  std::vector<int32_t> src1;   // single fill, sources read before the fill
  std::vector<uint8_t> sgn1;
  std::vector<int32_t> src2;   // two consecutive fills, resolved to interior cells
  std::vector<uint8_t> sgn2;
  bool resolved2 = false;      // every src2 is an interior cell
  bool face_rule_ok = false;   // face ghosts follow the fixed donor rule of the stage kernels
};

void build_ghost_tables(const bx_params& P, GhostTable& T);
void fill_geom(const bx_params& P, Geom& g);
bool is_pow2(double x);

// tabulated EOS on the device (H2STAT >= 0): tables of the eos module
struct EosDev {
  int neos, neos_rho;
  double log_rho_low, drho, density_unit, tk_bgrnd;
  const double *eng2, *gam2, *muc2, *tk2;  // (neos, neos_rho), neos fastest
  const double *rho, *deng;                // (neos_rho)
  const double* log_eng1;                  // (neos_rho): log10 of each row's first energy
};
// log10 of the first energy of each density row (the value get_gamma2 needs,
// computed once with the same device function)
cudaError_t eos_log_rows(const double* eng2, long long neos, int nr, double* out,
                         cudaStream_t s);

// ---- kernels (bx_kernels.cu)
struct StageArgs {
  const double* X;   // step input planes (C2 if nsrc==2, C3 if nsrc==1)
  const double* Y;   // stage-1 input: C1
  double* out;       // stage output planes (interior cells written)
  double* U;         // 3 planes: stage 0 writes m/rho of the step input at its own
                     // cells, stage 1 reads it as the stale velocity of its EOS
  const double* G;   // 3 planes of the gravitational acceleration, or null (no force)
  double* UC;        // with G: stage 1 writes the velocity after flux(1) of its
                     // own cells (the velocity state() reads at the step's end)
  Ctrl* ctrl;        // per box control blocks
  const Geom* geom;  // per box geometry (device)
  const Tile* tiles;
  long long ncells_total;  // plane stride of the pooled buffers
  int nsrc;                // > 0: sources the input is short of; 0: per box (Ctrl::nsrc)
  EosDev eos;              // the tables of the tabulated EOS (tile shape 2 only)
};

// Raises the dynamic shared-memory limit of kernel `fn` on the current device
// to at least `bytes`.  The attribute is held per device, so it is set once per
// (kernel, device) pair, under a lock: handles on several devices and several
// host threads may launch the same kernel.
cudaError_t ensure_dyn_smem(const void* fn, size_t bytes);

// dynamic shared memory of the stage kernels of a tile shape, and their resident
// blocks per SM (sets the shared-memory attribute on the current device)
size_t stage_smem_bytes(int shape = 0);
int stage_blocks_per_sm(int stage, int pm, bool threed, int shape = 0);

// pm: 1 = every box has power-of-two spacings, 0 = otherwise
cudaError_t launch_stage(int stage, int pm, bool threed, const StageArgs& a, int ntiles,
                         cudaStream_t s, int shape = 0);
cudaError_t launch_dt(Ctrl* ctrl, int nbox, cudaStream_t s);
cudaError_t launch_end(Ctrl* ctrl, int nbox, cudaStream_t s);

// phase kernels (one reference subroutine each, full arrays)
struct PhaseArrays {
  double* cons;     // 5*ng SoA
  double* cons_old; // 5*ng
  double* u;        // 3*ng
  double* p;        // ng
  double* adindx;   // ng
  double* gforce;   // 3*ng or null (zero force)
  double* states;   // flux scratch: 42*ng face states, then 15*ng face fluxes
                    // (fixed frame); 54*ng face states with fluxangmom
  double* gtmp;     // 5*nghost scratch for the ghost fill
  double* muc;      // ng (H2STAT >= 0: muc_array of state(); else null)
  EosDev eos;       // valid when muc is set
};

cudaError_t phase_state(const Geom& g, PhaseArrays& a, Ctrl* ctrl, cudaStream_t s);
cudaError_t phase_velocity(const Geom& g, PhaseArrays& a, Ctrl* ctrl, cudaStream_t s);
cudaError_t phase_courant(const Geom& g, PhaseArrays& a, Ctrl* ctrl, cudaStream_t s);
cudaError_t phase_source(const Geom& g, PhaseArrays& a, Ctrl* ctrl, double mult, cudaStream_t s);
cudaError_t phase_calc_gforce(const Geom& g, const double* phi, double* gforce, cudaStream_t s);
cudaError_t phase_ghost(int nghost, const int32_t* dst, const int32_t* src, const uint8_t* sgn,
                        PhaseArrays& a, long long ng, cudaStream_t s);
cudaError_t phase_flux(const Geom& g, PhaseArrays& a, Ctrl* ctrl, int avg, cudaStream_t s);
cudaError_t phase_courant_finish(Ctrl* ctrl, cudaStream_t s);
// avisc.f90:13-23 into qq (3 planes of ng) from the velocity array u
cudaError_t phase_avisc(const Geom& g, const double* u, const double avmag[3], double* qq,
                        cudaStream_t s);
cudaError_t phase_copy_old(const Geom& g, PhaseArrays& a, cudaStream_t s);

// fused <-> phase representation changes
cudaError_t fused_to_cons(const Geom& g, const double* X, int nsrc, double* cons, int nghost,
                          const int32_t* dst, const int32_t* src2, const uint8_t* sgn2,
                          cudaStream_t s);
cudaError_t fused_to_phase(const Geom& g, const double* X, int nsrc, PhaseArrays& a, int nghost,
                           const int32_t* dst, const int32_t* src2, const uint8_t* sgn2,
                           cudaStream_t s, long long xps = 0);

// batched path: per-box checks on planes with stride ps (X points at the box)
cudaError_t box_check_clean(const Geom& g, const double* X, long long ps, int nghost,
                            const int32_t* dst, const int32_t* src2, const uint8_t* sgn2,
                            Ctrl* ctrl, cudaStream_t s);
cudaError_t box_rate(const Geom& g, const double* X, long long ps, Ctrl* ctrl, cudaStream_t s);
cudaError_t launch_dt_batch(Ctrl* ctrl, int nbox, cudaStream_t s);

// Persistent batched run: one launch works through a queue of items (step,
// stage, tile) in step-major order; an item waits (bounded) for what it reads:
// a stage-0 tile for its box's dt of the step, a stage-1 tile for all stage-0
// tiles of its box.  The last stage-1 tile of a box advances the box's clock
// (k_end_batch) and sets the next step's dt (k_dt_batch).
struct PersistArgs {
  StageArgs a;               // ctrl, geom, tiles (longest first), plane stride, U; nsrc 0
  double* buf[3];            // the pooled plane sets
  int cur;                   // plane set that holds the run's input
  int nsteps;
  int ntiles;
  const int* tiles_of_box;   // tiles of each box in the list
  unsigned* done0;           // per box: stage-0 tiles finished so far in the run
  unsigned* done1;           // per box: stage-1 tiles finished so far in the run
  unsigned* ready;           // per box: steps of the run whose dt is set
  unsigned long long* head;  // next queue item
  int* status;               // bit 0: a wait gave up
  long long poll_limit;      // polls before a wait gives up
};
// the launch of a run (after launch_dt_batch for its first step); blocks_out:
// the blocks launched (resident blocks per SM x SMs)
cudaError_t launch_batch_persistent(const PersistArgs& p, int pm, bool threed, int nbox,
                                    cudaStream_t s, int* blocks_out, int shape = 0);
// a wait of the persistent kernel on a counter nothing advances, with the given
// poll limit: *gave_up = 1 when it returned without the counter (the check of
// the bounded wait)
cudaError_t persistent_wait_selftest(long long poll_limit, int* gave_up, float* ms);
cudaError_t launch_end_batch(Ctrl* ctrl, int nbox, cudaStream_t s);


// does the uploaded reference state equal what the fused form reproduces
// (u == m/rho, rho >= 1e-4 everywhere, ghosts == two-sweep fill of the interior)?
cudaError_t check_clean(const Geom& g, const PhaseArrays& a, int nghost, const int32_t* dst,
                        const int32_t* src2, const uint8_t* sgn2, Ctrl* ctrl, cudaStream_t s);

// AoS host layout <-> SoA device layout
cudaError_t aos_to_soa(const double* aos, double* soa, long long n, int k, cudaStream_t s);
cudaError_t prims_from_cons(const Geom& g, PhaseArrays& a, cudaStream_t s);
// after fused_to_phase of a step with a force: the pressure from the cons and
// the velocity after flux(1) (uc, 3 planes of interior cells), ghosts as donors
cudaError_t p_after_force(const Geom& g, PhaseArrays& a, const double* uc, int nghost,
                          const int32_t* dst, const int32_t* src2, cudaStream_t s);
// host-overlapped step: AoS slab [i0, i1) -> planes; planes -> AoS reference cons
// of the slab (interior cells nsrc sources short, then the ghosts [g0, g1) of
// the resolved plan, whose donors lie in this slab or an earlier one)
cudaError_t slab_in(const double* aos, double* X, long long ps, long long i0, long long i1,
                    cudaStream_t s);
cudaError_t slab_out(const Geom& g, const double* X, long long ps, int nsrc, double* aos,
                     long long i0, long long i1, const int32_t* dst, const int32_t* src2,
                     const uint8_t* sgn2, int g0, int g1, cudaStream_t s);
// Courant rate (as box_rate) of the interior cells of [i0, i1), atomicMax into *bits
cudaError_t slab_rate(const Geom& g, const double* X, long long ps, long long i0, long long i1,
                      unsigned long long* bits, cudaStream_t s);
cudaError_t fill_const(double* a, long long n, double v, cudaStream_t s);
cudaError_t soa_to_aos(const double* soa, double* aos, long long n, int k, cudaStream_t s);

}  // namespace bx

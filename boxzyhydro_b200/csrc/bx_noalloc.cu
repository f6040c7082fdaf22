// bx_noalloc.cu -- one ghost-cell sweep that allocates nothing.
//
// bx_ghost (one set_ghost_cells sweep on a handle) gathers every ghost's new
// value into scratch memory and then scatters it, so that sources are read as
// they were before the sweep.  The handle allocates that scratch with
// cudaMalloc.  Some callers cannot allocate device memory at all: a host
// program that has reserved the device's memory for its own pool up front, or a
// runtime that runs under a device-memory budget fixed when it started, would
// see cudaMalloc fail or break the budget.  bx_ghost_fill_noalloc gives them the
// same sweep with its scratch in a fixed array compiled into the library: the
// caller passes the conserved planes and the sweep plan in device memory it
// owns, and the library takes no memory beyond that array.
//
// The array holds BX_NOALLOC_MAX_GHOSTS x 5 doubles (40 MiB).  Every GPU that
// loads the library holds it until the process exits.  Host code cannot use the
// array's name as a device address (it names a host-side stand-in), so the
// first call on each device, with that device current, looks the device
// address up with cudaGetSymbolAddress and caches it; that first call should be
// made before any stream capture begins.  The cached address belongs to the
// CUDA context that was current when it was looked up: a call that finds
// another context current on the device (after cudaDeviceReset, or with a
// context of the caller's own made current) looks the address up again, since
// the library's module, and with it the array, lives at a new address in that
// context.  All calls share the one array and it
// keeps whatever the last call left there; nothing in it needs to start at
// zero, because every slot the scatter reads was written by the gather of the
// same call.  Calls that overlap on the GPU (on different streams, or from
// different host threads) race on the array.
#include <cuda_runtime.h>

#include <cstdio>
#include <mutex>

#include "../../include/boxzy_gpu.h"

namespace {

constexpr long long kMaxGhosts = BX_NOALLOC_MAX_GHOSTS;
constexpr int kMaxDevices = 64;

__device__ __align__(256) double g_ghost_scratch[5 * kMaxGhosts];

// per device: the context the scratch address was looked up in, and the address
struct ScratchSlot {
  void* ctx = nullptr;
  double* addr = nullptr;
};
std::mutex g_scratch_mu;
ScratchSlot g_scratch[kMaxDevices];
// the message of the calling thread's last failed call
thread_local char g_noalloc_err[256];

// the driver's current context of the calling thread (cuCtxGetCurrent, found
// through the runtime so the library does not link the driver library itself)
cudaError_t current_context(void** ctx) {
  using Fn = int (*)(void**);
  static Fn fn = [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPointByVersion("cuCtxGetCurrent", &p, 12000, cudaEnableDefault, &q) !=
            cudaSuccess ||
        q != cudaDriverEntryPointSuccess)
      p = nullptr;
    return reinterpret_cast<Fn>(p);
  }();
  if (!fn) return cudaErrorNotSupported;
  return fn(ctx) == 0 ? cudaSuccess : cudaErrorDeviceUninitialized;
}

__global__ void k_noalloc_gather(long long nghost, const int32_t* __restrict__ src,
                                 const uint8_t* __restrict__ sgn, const double* __restrict__ cons,
                                 long long n, double* __restrict__ tmp) {
  const long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (k >= nghost) return;
  const long long s = src[k];
  const unsigned m = sgn[k];
  tmp[k] = cons[s];
  tmp[nghost + k] = (m & 1) ? -cons[n + s] : cons[n + s];
  tmp[2 * nghost + k] = (m & 2) ? -cons[2 * n + s] : cons[2 * n + s];
  tmp[3 * nghost + k] = (m & 4) ? -cons[3 * n + s] : cons[3 * n + s];
  tmp[4 * nghost + k] = cons[4 * n + s];
}

__global__ void k_noalloc_scatter(long long nghost, const int32_t* __restrict__ dst,
                                  const double* __restrict__ tmp, double* __restrict__ cons,
                                  long long n) {
  const long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (k >= nghost) return;
  const long long d = dst[k];
#pragma unroll
  for (int q = 0; q < 5; ++q) cons[q * n + d] = tmp[q * nghost + k];
}

int fail(int code, const char* msg) {
  std::snprintf(g_noalloc_err, sizeof(g_noalloc_err), "%s", msg);
  return code;
}

}  // namespace

extern "C" const char* bx_noalloc_last_error(void) { return g_noalloc_err; }

extern "C" int bx_ghost_fill_noalloc(double* cons_soa, int64_t ngrid, const int32_t* dst,
                                     const int32_t* src, const uint8_t* sgn, int64_t nghost,
                                     void* cuda_stream) {
  if (nghost < 0 || ngrid <= 0) return fail(BX_ERR_ARG, "ngrid must be > 0 and nghost >= 0");
  if (nghost > kMaxGhosts)
    return fail(BX_ERR_ARG,
                "nghost exceeds BX_NOALLOC_MAX_GHOSTS (1048576 ghost cells); use bx_ghost");
  if (nghost == 0) return BX_OK;
  if (!cons_soa || !dst || !src || !sgn) return fail(BX_ERR_ARG, "null device pointer");
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return fail(BX_ERR_CUDA, cudaGetErrorString(e));
  if (dev < 0 || dev >= kMaxDevices) return fail(BX_ERR_ARG, "device ordinal out of range");
  void* ctx = nullptr;
  e = current_context(&ctx);
  if (e != cudaSuccess) return fail(BX_ERR_CUDA, "cuCtxGetCurrent is not available");
  if (!ctx) {
    // no context is current on this thread yet: the runtime's symbol lookup
    // makes the device's primary context current
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_ghost_scratch);
    if (e != cudaSuccess || !p) return fail(BX_ERR_CUDA, cudaGetErrorString(e));
    e = current_context(&ctx);
    if (e != cudaSuccess || !ctx) return fail(BX_ERR_CUDA, "no current CUDA context");
  }
  double* scratch = nullptr;
  {
    std::lock_guard<std::mutex> lock(g_scratch_mu);
    ScratchSlot& slot = g_scratch[dev];
    if (slot.ctx != ctx || !slot.addr) {
      // set-up, once per device and context, with that device current: the
      // device address of the static scratch array
      void* p = nullptr;
      e = cudaGetSymbolAddress(&p, g_ghost_scratch);
      if (e != cudaSuccess || !p) return fail(BX_ERR_CUDA, cudaGetErrorString(e));
      slot.ctx = ctx;
      slot.addr = static_cast<double*>(p);
    }
    scratch = slot.addr;
  }
  cudaStream_t s = static_cast<cudaStream_t>(cuda_stream);
  const int threads = 256;
  const int blocks = (int)((nghost + threads - 1) / threads);
  k_noalloc_gather<<<blocks, threads, 0, s>>>(nghost, src, sgn, cons_soa, ngrid, scratch);
  k_noalloc_scatter<<<blocks, threads, 0, s>>>(nghost, dst, scratch, cons_soa, ngrid);
  e = cudaGetLastError();
  if (e != cudaSuccess) return fail(BX_ERR_CUDA, cudaGetErrorString(e));
  return BX_OK;
}

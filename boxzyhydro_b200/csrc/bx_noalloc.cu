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
// made before any stream capture begins.  All calls share the one array and it
// keeps whatever the last call left there; nothing in it needs to start at
// zero, because every slot the scatter reads was written by the gather of the
// same call.  Calls that overlap on the GPU (on different streams, or from
// different host threads) race on the array.
#include <cuda_runtime.h>

#include <atomic>
#include <cstdio>

#include "../../include/boxzy_gpu.h"

namespace {

constexpr long long kMaxGhosts = BX_NOALLOC_MAX_GHOSTS;
constexpr int kMaxDevices = 64;

__device__ __align__(256) double g_ghost_scratch[5 * kMaxGhosts];

std::atomic<double*> g_scratch_addr[kMaxDevices];
char g_noalloc_err[256];

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
  double* scratch = g_scratch_addr[dev].load(std::memory_order_acquire);
  if (!scratch) {
    // set-up, once per device, with that device current: the device address of
    // the static scratch array
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_ghost_scratch);
    if (e != cudaSuccess || !p) return fail(BX_ERR_CUDA, cudaGetErrorString(e));
    scratch = static_cast<double*>(p);
    g_scratch_addr[dev].store(scratch, std::memory_order_release);
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

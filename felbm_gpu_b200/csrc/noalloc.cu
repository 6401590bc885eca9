// fe_mass_weight_noalloc: the order-parameter mass reduction for callers that
// cannot allocate device memory.
//
// Some hosts own every byte of the GPU's memory through their own pool (a
// framework's caching allocator that has reserved HBM, or an application
// that sizes all buffers up front), and some run in loops that must not hit
// cudaMalloc/cudaFree, which can block on device-wide synchronization. The
// engine's own reduction (k_mass in kernels.cuh) keeps its per-block partial
// sums in memory the engine allocates. This variant keeps them in a
// fixed-size array compiled into the library instead, so a call allocates
// nothing: the caller passes the input populations and a 2-double output,
// both in its own device memory.
//
// Limits and behaviour:
//  - at most FE_NOALLOC_MAX_SITES = 16384 blocks x 2048 sites = 33,554,432
//    sites per call; larger n is rejected with FE_ERR_ARG before any launch;
//  - the scratch array (NA_SCRATCH_BYTES = 262,400 bytes) exists once per GPU
//    that loads the library and stays allocated until the process exits;
//  - every call on a device shares that one array and it keeps the previous
//    call's contents; the completion counter is cleared on the caller's stream
//    at the start of each call, but calls whose work overlaps on the GPU
//    (different streams without ordering) race on the array and give wrong
//    results: order them on one stream or with events;
//  - the first call on each device looks up the array's device address
//    (cudaGetSymbolAddress) with that device current; make that first call
//    before any stream capture is started. The address is kept for the life
//    of the process, so a cudaDeviceReset (which reloads the module and may
//    move the array) must not be followed by further calls on that device.
#include <cuda_runtime.h>

#include <cstdint>
#include <mutex>
#include <string>

#include "../../include/felbm_b200.h"
#include "fe_internal.hpp"

namespace {

constexpr int NA_THREADS = 256;
constexpr int NA_SITES_PER_THREAD = 8;
constexpr int64_t NA_SITES_PER_BLOCK = (int64_t)NA_THREADS * NA_SITES_PER_THREAD;  // 2048
constexpr int NA_MAX_BLOCKS = 16384;
constexpr int64_t NA_MAX_SITES = NA_SITES_PER_BLOCK * NA_MAX_BLOCKS;               // 33,554,432
constexpr size_t NA_HEADER = 256;                                                  // counter + padding
constexpr size_t NA_SCRATCH_BYTES = NA_HEADER + (size_t)NA_MAX_BLOCKS * 2 * sizeof(double);
static_assert(NA_MAX_SITES == FE_NOALLOC_MAX_SITES, "header limit");
static_assert(NA_SCRATCH_BYTES == 262400, "header states the scratch size");

// The scratch: [0, 4) completion counter, [256, ...) per-block {M, W} partials.
// In host code this name is only a handle for cudaGetSymbolAddress, never a
// device address.
static __device__ __align__(256) unsigned char g_noalloc_scratch[NA_SCRATCH_BYTES];

constexpr int NA_MAX_DEVICES = 64;
std::mutex g_na_mutex;
void* g_na_ptr[NA_MAX_DEVICES] = {};

__global__ void __launch_bounds__(NA_THREADS) k_mass_weight_noalloc(const double* __restrict__ h, int64_t n,
                                                                     unsigned char* __restrict__ scratch,
                                                                     double* __restrict__ out) {
  __shared__ double red[NA_THREADS / 32][2];
  __shared__ int is_last;
  unsigned int* counter = reinterpret_cast<unsigned int*>(scratch);
  double* part = reinterpret_cast<double*>(scratch + NA_HEADER);
  const int64_t begin = (int64_t)blockIdx.x * NA_SITES_PER_BLOCK;
  const int64_t end = begin + NA_SITES_PER_BLOCK < n ? begin + NA_SITES_PER_BLOCK : n;
  double m = 0.0, w = 0.0;
  for (int64_t i = begin + threadIdx.x; i < end; i += NA_THREADS) {
    double c = 0.0;
#pragma unroll
    for (int k = 0; k < 19; ++k) c += h[(int64_t)k * n + i];
    double phi = c * (1.0 - c);
    if (phi < 0.0) phi = 0.0;
    m += c;
    w += phi;
  }
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    m += __shfl_down_sync(0xffffffffu, m, o);
    w += __shfl_down_sync(0xffffffffu, w, o);
  }
  if (lane == 0) { red[wid][0] = m; red[wid][1] = w; }
  __syncthreads();
  if (threadIdx.x == 0) {
    double bm = 0.0, bw = 0.0;
    for (int q = 0; q < NA_THREADS / 32; ++q) { bm += red[q][0]; bw += red[q][1]; }
    part[2 * blockIdx.x + 0] = bm;
    part[2 * blockIdx.x + 1] = bw;
    __threadfence();
    is_last = (atomicAdd(counter, 1u) == gridDim.x - 1) ? 1 : 0;
  }
  __syncthreads();
  if (!is_last) return;
  // the last block sums the partials in a fixed order (deterministic)
  double sm = 0.0, sw = 0.0;
  for (unsigned b = threadIdx.x; b < gridDim.x; b += NA_THREADS) {
    sm += __ldcg(&part[2 * b + 0]);
    sw += __ldcg(&part[2 * b + 1]);
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    sm += __shfl_down_sync(0xffffffffu, sm, o);
    sw += __shfl_down_sync(0xffffffffu, sw, o);
  }
  __syncthreads();
  if (lane == 0) { red[wid][0] = sm; red[wid][1] = sw; }
  __syncthreads();
  if (threadIdx.x == 0) {
    double tm = 0.0, tw = 0.0;
    for (int q = 0; q < NA_THREADS / 32; ++q) { tm += red[q][0]; tw += red[q][1]; }
    out[0] = tm;
    out[1] = tw;
    *counter = 0u;
  }
}

// Device address of the scratch array on the current device, looked up once.
int scratch_address(void** ptr) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return fe_fail(FE_ERR_CUDA, std::string("fe_mass_weight_noalloc: cudaGetDevice: ") +
                                                        cudaGetErrorString(e));
  if (dev < 0 || dev >= NA_MAX_DEVICES) return fe_fail(FE_ERR_ARG, "fe_mass_weight_noalloc: device index too large");
  std::lock_guard<std::mutex> lk(g_na_mutex);
  if (!g_na_ptr[dev]) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p)
      return fe_fail(FE_ERR_CUDA, std::string("fe_mass_weight_noalloc: cudaGetSymbolAddress: ") +
                                      cudaGetErrorString(e));
    g_na_ptr[dev] = p;
  }
  *ptr = g_na_ptr[dev];
  return FE_OK;
}

}  // namespace

extern "C" int fe_mass_weight_noalloc(const double* d_h, int64_t n, double* d_out, void* stream) {
  if (!d_h || !d_out || n <= 0)
    return fe_fail(FE_ERR_ARG, "fe_mass_weight_noalloc: null pointer or n <= 0");
  if (n > NA_MAX_SITES)
    return fe_fail(FE_ERR_ARG, "fe_mass_weight_noalloc: n = " + std::to_string(n) +
                                   " exceeds the fixed scratch capacity of " + std::to_string(NA_MAX_SITES) +
                                   " sites");
  void* scratch = nullptr;
  const int rc = scratch_address(&scratch);
  if (rc) return rc;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  cudaError_t e = cudaMemsetAsync(scratch, 0, sizeof(unsigned int), st);
  if (e != cudaSuccess)
    return fe_fail(FE_ERR_CUDA, std::string("fe_mass_weight_noalloc: clearing the counter: ") + cudaGetErrorString(e));
  const int blocks = (int)((n + NA_SITES_PER_BLOCK - 1) / NA_SITES_PER_BLOCK);
  k_mass_weight_noalloc<<<blocks, NA_THREADS, 0, st>>>(d_h, n, static_cast<unsigned char*>(scratch), d_out);
  e = cudaGetLastError();
  if (e != cudaSuccess)
    return fe_fail(FE_ERR_CUDA, std::string("fe_mass_weight_noalloc: launch: ") + cudaGetErrorString(e));
  return FE_OK;
}

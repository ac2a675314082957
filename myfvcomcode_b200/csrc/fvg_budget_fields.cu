// fvg_budget_fields.cu - volume, heat and salt budgets of caller-owned device fields,
// computed without allocating any memory.
//
// fvg_budget needs a handle, and fvg_create allocates the whole model state on the device
// (several GB on a 200k-node, 40-layer mesh).  Some callers can allocate nothing at the
// point where they want a conservation check:
//   * a code that keeps its own FVCOM state on the device (a coupler, or a GPU port of the
//     rest of the model) and samples the budgets every step: cudaMalloc and cudaFree
//     synchronise the whole device, so an allocation per call would stall the caller's
//     other streams each time;
//   * a run sized to fill HBM, where even a small allocation can fail mid-run with
//     out-of-memory and end the job at the moment the check was meant to protect it.
// This entry point therefore keeps its reduction scratch in a fixed-size, file-scope
// __device__ array and calls no allocating routine (no cudaMalloc, cudaMallocAsync,
// cudaFree or library call that allocates).
//
// Limit: one 256-node tile per block with one partial triple per tile, for at most
// kMaxTiles = 16,384 tiles, i.e. M <= 4,194,304 nodes (393,240 bytes of scratch on each
// device).  Larger meshes are rejected with FVG_ERR_CAPACITY before anything is launched.
//
// Set-up: the first call on a device looks up the scratch array's device address with
// cudaGetSymbolAddress (with that device current) and caches it; later calls on that
// device reuse it.  Make one call on each device before any stream capture begins.  With
// CUDA's lazy module loading, that first call (its symbol lookup and first launches) is
// also what loads this library's device code on the device, and loading reserves device
// memory for the code and for g_budget_scratch.  "Allocates nothing" therefore holds from
// the second call on: a caller that will fill HBM makes the first call early.
//
// Every call waits for its stream and copies the result to host memory before returning.
//
// Nothing has to start at zero: the tile kernel writes every partial that the final
// kernel reads, earlier on the same stream, and the final kernel writes the result.
//
// The scratch is shared by every call on a device: two calls in flight at the same time
// on one device (from different host threads or on different streams) race on it and
// give wrong sums.  Callers must not overlap calls on the same device.
#include <cuda_runtime.h>

#include <cstdint>
#include <mutex>

#include "../../include/fvg.h"

namespace {

constexpr int kTile = 256;
constexpr int kMaxTiles = 16384;
constexpr int64_t kMaxNodes = (int64_t)kTile * kMaxTiles;  // 4,194,304
constexpr int kMaxLayers = 63;                                // KB <= 64, as fvg_create
constexpr int kMaxDevices = 64;

// Partials of tile t at [3t, 3t+3); the result at [3*kMaxTiles, 3*kMaxTiles+3).
__device__ __align__(256) double g_budget_scratch[3 * kMaxTiles + 3];

std::mutex g_scratch_mu;
double* g_scratch_ptr[kMaxDevices] = {};

// Device address of g_budget_scratch on the current device, looked up once per device.
int scratch_on_current_device(double** out) {
  int dev = -1;
  if (cudaGetDevice(&dev) != cudaSuccess) return FVG_ERR_CUDA;
  if (dev < 0 || dev >= kMaxDevices) return FVG_ERR_ARG;
  std::lock_guard<std::mutex> lock(g_scratch_mu);
  if (!g_scratch_ptr[dev]) {
    void* p = nullptr;
    if (cudaGetSymbolAddress(&p, g_budget_scratch) != cudaSuccess || !p) return FVG_ERR_CUDA;
    g_scratch_ptr[dev] = static_cast<double*>(p);
  }
  *out = g_scratch_ptr[dev];
  return FVG_OK;
}

// One thread per node, one block per 256-node tile: D*ART1 and the column sums of T1*DZ
// and S1*DZ over K = 1..KBM1 (the same per-node arithmetic as fvg_budget), then a fixed
// shared-memory tree over the tile.  Fields are Fortran-ordered with ghost row 0, leading
// dimension M+1.
__global__ void __launch_bounds__(kTile) k_budget_field_tiles(const double* __restrict__ d,
                                                              const double* __restrict__ art1,
                                                              const double* __restrict__ t1,
                                                              const double* __restrict__ s1,
                                                              const double* __restrict__ dz,
                                                              int m, int kbm1, double* part) {
  __shared__ double sv[kTile], sh[kTile], ss[kTile];
  const int tid = threadIdx.x;
  const int i = blockIdx.x * kTile + tid + 1;
  double v = 0.0, hh = 0.0, s = 0.0;
  if (i <= m) {
    const size_t ld = (size_t)m + 1;
    const double dd = d[i] * art1[i];
    double ct = 0.0, cs = 0.0;
    for (int k = 0; k < kbm1; ++k) {
      const size_t q = (size_t)k * ld + i;
      ct = ct + t1[q] * dz[q];
      cs = cs + s1[q] * dz[q];
    }
    v = dd;
    hh = ct * dd;
    s = cs * dd;
  }
  sv[tid] = v;
  sh[tid] = hh;
  ss[tid] = s;
  __syncthreads();
  for (int st = kTile / 2; st > 0; st >>= 1) {
    if (tid < st) {
      sv[tid] += sv[tid + st];
      sh[tid] += sh[tid + st];
      ss[tid] += ss[tid + st];
    }
    __syncthreads();
  }
  if (tid == 0) {
    part[3 * blockIdx.x] = sv[0];
    part[3 * blockIdx.x + 1] = sh[0];
    part[3 * blockIdx.x + 2] = ss[0];
  }
}

// One block: thread t sums tiles t, t+256, ... in order, then a fixed tree.
__global__ void __launch_bounds__(kTile) k_budget_field_final(const double* part, int ntiles,
                                                              double* out) {
  __shared__ double sv[kTile], sh[kTile], ss[kTile];
  const int tid = threadIdx.x;
  double a = 0.0, b = 0.0, c = 0.0;
  for (int t = tid; t < ntiles; t += kTile) {
    a += part[3 * t];
    b += part[3 * t + 1];
    c += part[3 * t + 2];
  }
  sv[tid] = a;
  sh[tid] = b;
  ss[tid] = c;
  __syncthreads();
  for (int st = kTile / 2; st > 0; st >>= 1) {
    if (tid < st) {
      sv[tid] += sv[tid + st];
      sh[tid] += sh[tid + st];
      ss[tid] += ss[tid + st];
    }
    __syncthreads();
  }
  if (tid == 0) {
    out[0] = sv[0];
    out[1] = sh[0];
    out[2] = ss[0];
  }
}

}  // namespace

extern "C" int fvg_budget_fields(const double* d, const double* art1, const double* t1,
                                 const double* s1, const double* dz, int32_t m, int32_t kbm1,
                                 void* stream, double out[3]) {
  if (!d || !art1 || !t1 || !s1 || !dz || !out) return FVG_ERR_ARG;
  if (m < 1 || kbm1 < 1 || kbm1 > kMaxLayers) return FVG_ERR_ARG;
  if ((int64_t)m > kMaxNodes) return FVG_ERR_CAPACITY;
  double* scratch = nullptr;
  int rc = scratch_on_current_device(&scratch);
  if (rc) return rc;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const int ntiles = (m + kTile - 1) / kTile;
  double* result = scratch + 3 * kMaxTiles;
  k_budget_field_tiles<<<ntiles, kTile, 0, s>>>(d, art1, t1, s1, dz, m, kbm1, scratch);
  k_budget_field_final<<<1, kTile, 0, s>>>(scratch, ntiles, result);
  if (cudaGetLastError() != cudaSuccess) return FVG_ERR_CUDA;
  if (cudaMemcpyAsync(out, result, 3 * sizeof(double), cudaMemcpyDeviceToHost, s) != cudaSuccess)
    return FVG_ERR_CUDA;
  if (cudaStreamSynchronize(s) != cudaSuccess) return FVG_ERR_CUDA;
  return FVG_OK;
}

// mk_noalloc.cu — FP64 statistics of a device field with no device allocation.
//
// Same two-pass warp-shuffle reduction as the diagnostics kernels (block
// partials, then one block folding the partials in a fixed order), but the
// partials live in a file-scope device array instead of memory the library
// allocates, so the entry point can be called by code that is not allowed to
// call cudaMalloc: a host application that owns the device memory through its
// own pool or has handed the rest of the HBM to another solver, or a timed
// loop in which the implicit device synchronisation of an allocation would
// stall the pipeline.  The caller passes the field and a device output.
//
// Limits and sharing:
//  * n <= MK_NOALLOC_MAX_CELLS: the scratch holds MK_NOALLOC_MAX_BLOCKS block
//    partials and each thread folds at most 64 cells.
//  * The scratch (MK_NOALLOC_MAX_BLOCKS x 5 doubles = 80 KiB) is held by every
//    GPU that loads the library until the process exits.
//  * All calls share it and it keeps the last call's contents.  Nothing in it
//    needs to start at zero: every block of a call overwrites its own slot and
//    the second pass reads only the slots of that call.  Calls that overlap on
//    the GPU (different streams, or different host threads, on one device)
//    race on the scratch; serialise them.
//  * The first call on a device looks up the scratch's device address
//    (cudaGetSymbolAddress, with that device current); make that first call
//    before any stream capture.
#include <cuda_runtime.h>

#include <cmath>
#include <mutex>
#include <string>

#include "../../include/mkb200.h"

namespace {

constexpr int kNoallocBlocks = MK_NOALLOC_MAX_BLOCKS;
constexpr int kNoallocThreads = 256;
constexpr int kNV = 5;  // sum, sum of squares, min, max, non-finite count

// Block partials of the last call.  In host code this name is only a handle
// for cudaGetSymbolAddress, never an address to pass to a kernel.
static __device__ __align__(256) double g_noalloc_partials[kNoallocBlocks * kNV];

static_assert((int64_t)kNoallocBlocks * kNoallocThreads * 64 == MK_NOALLOC_MAX_CELLS,
              "MK_NOALLOC_MAX_CELLS must match the scratch geometry");

__device__ __forceinline__ void fold(double (&v)[kNV], const double (&o)[kNV]) {
  v[0] += o[0];
  v[1] += o[1];
  v[2] = fmin(v[2], o[2]);
  v[3] = fmax(v[3], o[3]);
  v[4] += o[4];
}

__device__ __forceinline__ void block_fold(double (&v)[kNV]) {
  __shared__ double sh[kNoallocThreads / 32][kNV];
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) {
    double o[kNV];
#pragma unroll
    for (int q = 0; q < kNV; ++q) o[q] = __shfl_down_sync(0xffffffffu, v[q], off);
    fold(v, o);
  }
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (lane == 0)
#pragma unroll
    for (int q = 0; q < kNV; ++q) sh[wid][q] = v[q];
  __syncthreads();
  if (wid == 0) {
    const double init[kNV] = {0.0, 0.0, INFINITY, -INFINITY, 0.0};
#pragma unroll
    for (int q = 0; q < kNV; ++q) v[q] = lane < (int)(blockDim.x >> 5) ? sh[lane][q] : init[q];
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
      double o[kNV];
#pragma unroll
      for (int q = 0; q < kNV; ++q) o[q] = __shfl_down_sync(0xffffffffu, v[q], off);
      fold(v, o);
    }
  }
}

__global__ void __launch_bounds__(kNoallocThreads) k_noalloc_partial(const float* __restrict__ a, int64_t n,
                                                                      double* __restrict__ partials) {
  double v[kNV] = {0.0, 0.0, INFINITY, -INFINITY, 0.0};
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const double x = (double)a[i];
    if (isfinite(x)) {
      v[0] += x;
      v[1] += x * x;
      v[2] = fmin(v[2], x);
      v[3] = fmax(v[3], x);
    } else {
      v[4] += 1.0;
    }
  }
  block_fold(v);
  if (threadIdx.x == 0)
#pragma unroll
    for (int q = 0; q < kNV; ++q) partials[(int64_t)blockIdx.x * kNV + q] = v[q];
}

__global__ void __launch_bounds__(kNoallocThreads) k_noalloc_final(const double* __restrict__ partials, int nblocks,
                                                                    double* __restrict__ out) {
  double v[kNV] = {0.0, 0.0, INFINITY, -INFINITY, 0.0};
  for (int b = threadIdx.x; b < nblocks; b += blockDim.x) {
    double o[kNV];
#pragma unroll
    for (int q = 0; q < kNV; ++q) o[q] = partials[(int64_t)b * kNV + q];
    fold(v, o);
  }
  block_fold(v);
  if (threadIdx.x == 0)
#pragma unroll
    for (int q = 0; q < kNV; ++q) out[q] = v[q];
}

// Device address of the scratch, looked up once per device.
constexpr int kMaxDevices = 64;
std::mutex g_noalloc_mu;
double* g_noalloc_ptr[kMaxDevices] = {nullptr};
thread_local std::string g_noalloc_err;

mk_status noalloc_fail(mk_status s, const std::string& m) {
  g_noalloc_err = m;
  return s;
}

}  // namespace

extern "C" const char* mk_noalloc_last_error(void) { return g_noalloc_err.c_str(); }

extern "C" mk_status mk_field_stats_noalloc(const float* d_field, int64_t n, double* d_out, void* stream) {
  if (n < 0 || n > (int64_t)MK_NOALLOC_MAX_CELLS)
    return noalloc_fail(MK_ERR_ARG, "mk_field_stats_noalloc: n = " + std::to_string(n) +
                                        " is outside [0, MK_NOALLOC_MAX_CELLS = " +
                                        std::to_string((long long)MK_NOALLOC_MAX_CELLS) + "]");
  if ((!d_field && n > 0) || !d_out) return noalloc_fail(MK_ERR_ARG, "mk_field_stats_noalloc: null pointer");
  int dev = 0;
  cudaError_t st = cudaGetDevice(&dev);
  if (st != cudaSuccess) return noalloc_fail(MK_ERR_NODEVICE, std::string("no CUDA device: ") + cudaGetErrorString(st));
  if (dev < 0 || dev >= kMaxDevices) return noalloc_fail(MK_ERR_ARG, "device index out of range");
  double* scratch = nullptr;
  {
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    if (!g_noalloc_ptr[dev]) {
      // set-up on this device, which is current
      st = cudaGetSymbolAddress((void**)&g_noalloc_ptr[dev], g_noalloc_partials);
      if (st != cudaSuccess) {
        g_noalloc_ptr[dev] = nullptr;
        return noalloc_fail(MK_ERR_CUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(st));
      }
    }
    scratch = g_noalloc_ptr[dev];
  }
  const cudaStream_t s = (cudaStream_t)stream;
  int64_t nb = (n + kNoallocThreads - 1) / kNoallocThreads;
  if (nb < 1) nb = 1;
  if (nb > kNoallocBlocks) nb = kNoallocBlocks;
  k_noalloc_partial<<<(unsigned)nb, kNoallocThreads, 0, s>>>(d_field, n, scratch);
  k_noalloc_final<<<1, kNoallocThreads, 0, s>>>(scratch, (int)nb, d_out);
  st = cudaGetLastError();
  if (st != cudaSuccess) return noalloc_fail(MK_ERR_CUDA, std::string("launch: ") + cudaGetErrorString(st));
  return MK_OK;
}

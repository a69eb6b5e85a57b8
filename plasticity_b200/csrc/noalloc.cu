// noalloc.cu -- Euclidean norm of a device vector that allocates no memory.
//
// Same two-pass reduction as the library's residual norm (per-block partial
// sums, then one block sums the partials), but the partial sums live in a
// file-scope device array instead of memory obtained with cudaMalloc.  It is
// meant for callers that cannot allocate device memory themselves -- code
// running inside a framework that owns every device allocation through its
// own pool or arena, or a caller that has to stay free of cudaMalloc/cudaFree
// in its steady state -- and that already hold the input vector and a one-
// element output buffer in device memory.
#include <cuda_runtime.h>

#include <cstdio>
#include <mutex>
#include <string>

#include "../../include/pfem_b200.h"
#include "common.cuh"

namespace {

constexpr int NA_THREADS = 256;
constexpr int NA_PER_THREAD = 8;
constexpr long long NA_CHUNK = (long long)NA_THREADS * NA_PER_THREAD;  // elements per block
constexpr int NA_MAX_BLOCKS = 65536;                                    // partial-sum slots
constexpr long long NA_MAX_N = NA_CHUNK * NA_MAX_BLOCKS;                // 134,217,728 elements

// One partial sum per block of the first pass: 65,536 doubles (512 KiB),
// resident on every device that loads the library until the process exits.
// Every call overwrites the slots it uses before reading them, so nothing has
// to be cleared between calls; calls that overlap on the GPU share these
// slots and race.
static __device__ __align__(256) double g_norm_partials[NA_MAX_BLOCKS];

constexpr int NA_MAX_DEVICES = 64;
std::mutex g_setup_mu;
double* g_partials_ptr[NA_MAX_DEVICES] = {nullptr};

__device__ __forceinline__ double na_block_sum(double v, double* sh) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  if (l == 0) sh[w] = v;
  __syncthreads();
  v = (threadIdx.x < (blockDim.x >> 5)) ? sh[threadIdx.x] : 0.0;
  if (w == 0) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  }
  return v;
}

__global__ void __launch_bounds__(NA_THREADS) na_partial_kernel(const double* __restrict__ x, long long n,
                                                                double* __restrict__ part) {
  __shared__ double sh[32];
  const long long base = (long long)blockIdx.x * NA_CHUNK;
  double v = 0.0;
#pragma unroll
  for (int k = 0; k < NA_PER_THREAD; ++k) {
    const long long i = base + (long long)k * NA_THREADS + threadIdx.x;
    if (i < n) {
      const double t = x[i];
      v += t * t;
    }
  }
  v = na_block_sum(v, sh);
  if (threadIdx.x == 0) part[blockIdx.x] = v;
}

__global__ void __launch_bounds__(1024) na_final_kernel(const double* __restrict__ part, int nb,
                                                        double* __restrict__ out) {
  __shared__ double sh[32];
  double v = 0.0;
  for (int i = threadIdx.x; i < nb; i += blockDim.x) v += part[i];
  v = na_block_sum(v, sh);
  if (threadIdx.x == 0) *out = sqrt(v);
}

}  // namespace

extern "C" int pfem_norm2_noalloc(const double* x, int64_t n, double* result, void* stream) {
  if (!result || (n > 0 && !x) || n < 0) {
    pfem::set_last_error("pfem_norm2_noalloc: null pointer or negative length");
    return PFEM_ERR_BAD_ARG;
  }
  if (n > NA_MAX_N) {
    char buf[160];
    snprintf(buf, sizeof(buf), "pfem_norm2_noalloc: n = %lld exceeds the maximum of %lld elements",
             (long long)n, (long long)NA_MAX_N);
    pfem::set_last_error(buf);
    return PFEM_ERR_BAD_ARG;
  }
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) {
    pfem::set_last_error(std::string("pfem_norm2_noalloc: no usable current device: ") + cudaGetErrorString(e));
    return PFEM_ERR_CUDA;
  }
  if (dev < 0 || dev >= NA_MAX_DEVICES) {
    char buf[160];
    snprintf(buf, sizeof(buf), "pfem_norm2_noalloc: current device index %d is outside the %d devices supported",
             dev, NA_MAX_DEVICES);
    pfem::set_last_error(buf);
    return PFEM_ERR_CUDA;
  }
  double* part = nullptr;
  {
    // First call on a device (with that device current): look up the device
    // address of the scratch array.  In host code g_norm_partials names a
    // host-side stand-in, never the device memory, so the kernels must get
    // this address.
    std::lock_guard<std::mutex> lk(g_setup_mu);
    if (!g_partials_ptr[dev]) {
      void* p = nullptr;
      e = cudaGetSymbolAddress(&p, g_norm_partials);
      if (e != cudaSuccess || !p) {
        pfem::set_last_error(std::string("pfem_norm2_noalloc: cudaGetSymbolAddress failed: ") + cudaGetErrorString(e));
        return PFEM_ERR_CUDA;
      }
      g_partials_ptr[dev] = static_cast<double*>(p);
    }
    part = g_partials_ptr[dev];
  }
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const int nb = (int)((n + NA_CHUNK - 1) / NA_CHUNK);
  if (nb > 0) {
    pfem::count_launch();
    na_partial_kernel<<<nb, NA_THREADS, 0, st>>>(x, (long long)n, part);
  }
  pfem::count_launch();
  na_final_kernel<<<1, 1024, 0, st>>>(part, nb, result);
  e = cudaGetLastError();
  if (e != cudaSuccess) {
    pfem::set_last_error(std::string("pfem_norm2_noalloc: launch failed: ") + cudaGetErrorString(e));
    return PFEM_ERR_CUDA;
  }
  return PFEM_OK;
}


// Small device helpers shared by the kernels.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

namespace spops {

// Streaming load (evict-first): matrix arrays are read once per SpMV, so they
// should not push the gathered vector x out of L2.
__device__ __forceinline__ int ld_stream(const int* p) { return __ldcs(p); }
__device__ __forceinline__ int64_t ld_stream(const int64_t* p) {
  return (int64_t)__ldcs(reinterpret_cast<const long long*>(p));
}
__device__ __forceinline__ float ld_stream(const float* p) { return __ldcs(p); }
__device__ __forceinline__ double ld_stream(const double* p) { return __ldcs(p); }

// Read-only cached load for the gathered vector.
template <typename T>
__device__ __forceinline__ T ld_gather(const T* p) { return __ldg(p); }

// L2-coherent load (bypasses L1), for values written by other blocks.
__device__ __forceinline__ float ld_cg(const float* p) { return __ldcg(p); }
__device__ __forceinline__ double ld_cg(const double* p) { return __ldcg(p); }

template <typename V>
__device__ __forceinline__ V warp_sum(V v, int width = 32) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1)
    if (o < width) v += __shfl_down_sync(0xffffffffu, v, o, width);
  return v;
}

// Deterministic block-wide sum (fixed tree); result valid in thread 0.
// `red` needs blockDim.x/32 entries.
template <typename V>
__device__ __forceinline__ V block_sum(V v, V* red) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  v = warp_sum(v);
  if (lane == 0) red[wid] = v;
  __syncthreads();
  const int nw = blockDim.x >> 5;
  if (wid == 0) {
    v = lane < nw ? red[lane] : V(0);
    v = warp_sum(v);
  }
  __syncthreads();
  return v;
}

// y = alpha*sum + beta*y, with beta == 0 meaning "overwrite, do not read y".
template <typename V>
__device__ __forceinline__ void axpby_store(V* y, V sum, V alpha, V beta, bool beta_zero) {
  *y = beta_zero ? alpha * sum : alpha * sum + beta * (*y);
}

// The same with streaming (evict-first) accesses to y, for outputs that
// would otherwise push gathered operands out of L2.
template <typename V>
__device__ __forceinline__ void axpby_store_cs(V* y, V sum, V alpha, V beta, bool beta_zero) {
  __stcs(y, beta_zero ? alpha * sum : alpha * sum + beta * __ldcs(y));
}

}  // namespace spops

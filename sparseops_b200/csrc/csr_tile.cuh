// CSR tiles of 32 lanes x K consecutive entries: the helpers shared by the
// tile SpMV / SpMM kernels (spmv_csr_tile.cu) and the batch's tile items
// (batched.cu).  See spmv_csr_tile.cu for the plan (flags, tile_row, empty
// rows) and the calibration of rows that cross tiles.
#pragma once

#include <cstdint>
#include <cstring>

#include "device_util.cuh"

namespace spops {
namespace {

// last r in [0, n-1] with rp[r] <= e (the non-empty row holding entry e)
template <typename I>
__device__ __forceinline__ int64_t row_holding(const I* rp, int64_t n, int64_t e) {
  int64_t lo = 0, hi = n;
  while (hi - lo > 1) {
    const int64_t mid = (lo + hi) >> 1;
    if ((int64_t)rp[mid] <= e) lo = mid; else hi = mid;
  }
  return lo;
}

// ---- vector loads of one lane's run (32-byte aligned for 32-byte runs)
template <int BYTES>
struct RunLoad;
template <>
struct RunLoad<16> {
  static __device__ __forceinline__ void ld(const void* p, uint32_t (&w)[4]) {
    asm volatile("ld.global.nc.L1::no_allocate.v4.b32 {%0,%1,%2,%3}, [%4];"
                 : "=r"(w[0]), "=r"(w[1]), "=r"(w[2]), "=r"(w[3])
                 : "l"(p));
  }
};
template <>
struct RunLoad<32> {
  static __device__ __forceinline__ void ld(const void* p, uint32_t (&w)[8]) {
    asm volatile("ld.global.nc.L1::no_allocate.v8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
                 : "=r"(w[0]), "=r"(w[1]), "=r"(w[2]), "=r"(w[3]), "=r"(w[4]), "=r"(w[5]), "=r"(w[6]), "=r"(w[7])
                 : "l"(p));
  }
};

// K elements of T from p (aligned to min(32, K*sizeof(T)) bytes) into out.
template <typename T, int K>
__device__ __forceinline__ void load_run(const T* __restrict__ p, T (&out)[K]) {
  constexpr int BYTES = K * (int)sizeof(T);
  static_assert(BYTES == 16 || BYTES % 32 == 0, "run must be 16 bytes or a multiple of 32");
  if constexpr (BYTES == 16) {
    uint32_t w[4];
    RunLoad<16>::ld(p, w);
    memcpy(out, w, 16);
  } else {
#pragma unroll
    for (int q = 0; q < BYTES / 32; ++q) {
      uint32_t w[8];
      RunLoad<32>::ld(reinterpret_cast<const char*>(p) + 32 * q, w);
      memcpy(reinterpret_cast<char*>(out) + 32 * q, w, 32);
    }
  }
}

// Columns and values of lane `lane`'s run of tile t; entries past nnz read as
// column 0 with value 0.
template <typename I, typename V, int K>
__device__ __forceinline__ void tile_load(const I* __restrict__ ci, const V* __restrict__ val, int64_t nnz, int64_t t,
                                          int lane, I (&c)[K], V (&a)[K]) {
  const int64_t el = t * (32 * K) + (int64_t)lane * K;
  if (el + K <= nnz) {
    load_run<I, K>(ci + el, c);
    load_run<V, K>(val + el, a);
  } else {
#pragma unroll
    for (int b = 0; b < K; ++b) {
      const bool in = el + b < nnz;
      c[b] = in ? ci[el + b] : I(0);
      a[b] = in ? ld_stream(val + el + b) : V(0);
    }
  }
}

// ---- multi-RHS with k = 8 on the same tile plan (csr_tile_spmm8)
// Lane l of the warp that owns tile t takes the SpMV's 8 entries, gathers
// each entry's X row (8 values, 32-byte vector loads, four rows at a time)
// and keeps 8 running sums that are cut at every row start; the heads
// combine across lanes with the SpMV's segmented scan, and the row open at a
// tile's end goes to the 8-wide calibrator.  Every column is summed in an
// order fixed by the matrix.
template <typename V>
__device__ __forceinline__ void ld_xrow8(const V* __restrict__ p, V (&r)[8]) {
#pragma unroll
  for (int q = 0; q < (int)sizeof(V); q += 4) {
    uint32_t w[8];
    asm volatile("ld.global.nc.v8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
                 : "=r"(w[0]), "=r"(w[1]), "=r"(w[2]), "=r"(w[3]), "=r"(w[4]), "=r"(w[5]), "=r"(w[6]), "=r"(w[7])
                 : "l"(reinterpret_cast<const char*>(p) + 8 * q));
    memcpy(reinterpret_cast<char*>(r) + 8 * q, w, 32);
  }
}

template <typename V>
__device__ __forceinline__ void axpby_store8(V* __restrict__ y, const V (&v)[8], V alpha, V beta, bool bz) {
#pragma unroll
  for (int j = 0; j < 8; ++j) axpby_store(y + j, v[j], alpha, beta, bz);
}

// One tile t of a k = 8 multi-RHS product (the loop body of
// csr_tile_spmm8_kernel and of the batch's tile items).
template <typename I, typename V>
__device__ __forceinline__ void spmm8_tile(const I* __restrict__ rp, int64_t n, int64_t nnz, const I* __restrict__ ci,
                                           const V* __restrict__ val, const int64_t* __restrict__ tile_row,
                                           const uint8_t* __restrict__ flags_all, int64_t t, const V* __restrict__ X,
                                           int64_t ldx, V* __restrict__ Y, int64_t ldy, V alpha, V beta, bool bz,
                                           V* __restrict__ carry_in, V* __restrict__ open_sum,
                                           int64_t* __restrict__ open_row, int lane) {
  constexpr int K = 8;
  const unsigned lt = (1u << lane) - 1u;
  I c[K];
  V a[K];
  tile_load<I, V, K>(ci, val, nnz, t, lane, c, a);
  const uint32_t flags = flags_all[t * 32 + lane];
  const int64_t tr = tile_row[t];
  const int64_t el = t * (32 * K) + (int64_t)lane * K;
  int64_t row;
  if (tr >= 0) {
    const int cnt = __popc(flags);
    int excl = 0;
#pragma unroll
    for (int bit = 0; bit < 4; ++bit) excl += __popc(__ballot_sync(0xffffffffu, (cnt >> bit) & 1) & lt) << bit;
    const int first0 = (int)(__ballot_sync(0xffffffffu, flags & 1u) & 1u);
    row = tr + excl + (int)(flags & 1u) - first0;
  } else {
    row = row_holding(rp, n, el < nnz ? el : nnz - 1);
  }
  V acc[8], head[8];
#pragma unroll
  for (int j = 0; j < 8; ++j) acc[j] = head[j] = V(0);
  bool in_head = (flags & 1u) == 0;
#pragma unroll
  for (int h = 0; h < 2; ++h) {
    V xr[4][8];
#pragma unroll
    for (int q = 0; q < 4; ++q) ld_xrow8(X + (int64_t)c[4 * h + q] * ldx, xr[q]);
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int b = 4 * h + q;
      if (b > 0 && ((flags >> b) & 1u)) {
        if (in_head) {
#pragma unroll
          for (int j = 0; j < 8; ++j) head[j] = acc[j];
          in_head = false;
        } else {
          axpby_store8(Y + row * ldy, acc, alpha, beta, bz);
        }
#pragma unroll
        for (int j = 0; j < 8; ++j) acc[j] = V(0);
        ++row;
        if (tr < 0)
          while (row + 1 < n && rp[row] == rp[row + 1]) ++row;  // skip empty rows
      }
#pragma unroll
      for (int j = 0; j < 8; ++j) {
        const V prod = a[b] * xr[q][j];
        acc[j] += prod;
      }
    }
  }
  V tail[8];
#pragma unroll
  for (int j = 0; j < 8; ++j) {
    if (in_head) head[j] = acc[j];
    tail[j] = in_head ? V(0) : acc[j];
  }
  // segmented inclusive scan of the heads (a segment starts right after
  // every flagged lane)
  const bool has_flag = flags != 0;
  const unsigned fmask = __ballot_sync(0xffffffffu, has_flag);
  const unsigned starts = (fmask << 1) | 1u;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const unsigned span = (lane >= o) ? ((2u << lane) - 1u) & ~((2u << (lane - o)) - 1u) : 0u;
    const bool add = lane >= o && !(starts & span);
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      const V su = __shfl_up_sync(0xffffffffu, head[j], o);
      if (add) head[j] += su;
    }
  }
  const unsigned later = fmask & ~((2u << lane) - 1u);
  const int m = later ? __ffs(later) - 1 : 31;
  const int m0 = fmask ? __ffs(fmask) - 1 : 31;
  V Sm[8], cin[8];
#pragma unroll
  for (int j = 0; j < 8; ++j) {
    Sm[j] = __shfl_sync(0xffffffffu, head[j], m);
    cin[j] = __shfl_sync(0xffffffffu, head[j], m0);
  }
  if (has_flag) {
    if (later) {
#pragma unroll
      for (int j = 0; j < 8; ++j) tail[j] += Sm[j];
      axpby_store8(Y + row * ldy, tail, alpha, beta, bz);
    } else {  // the tile's last row: may continue into the next tile
#pragma unroll
      for (int j = 0; j < 8; ++j) open_sum[t * 8 + j] = tail[j] + (lane < 31 ? Sm[j] : V(0));
      open_row[t] = row;
    }
  }
  if (lane == 0) {
#pragma unroll
    for (int j = 0; j < 8; ++j) carry_in[t * 8 + j] = cin[j];
    if (!fmask) open_row[t] = -1;
  }
}

// Calibration of one tile t (t < tiles) or empty row (t - tiles < nempty)
// of a k = 8 product.
template <typename V>
__device__ __forceinline__ void spmm8_calibrate(int64_t t, int64_t tiles, const V* __restrict__ carry_in,
                                                const V* __restrict__ open_sum, const int64_t* __restrict__ open_row,
                                                const int64_t* __restrict__ empty, int64_t nempty, V* __restrict__ Y,
                                                int64_t ldy, V alpha, V beta, bool bz) {
  V tot[8];
  if (t < tiles) {
    const int64_t r = open_row[t];
    if (r < 0) return;
#pragma unroll
    for (int j = 0; j < 8; ++j) tot[j] = open_sum[t * 8 + j];
    for (int64_t u = t + 1; u < tiles; ++u) {
#pragma unroll
      for (int j = 0; j < 8; ++j) tot[j] += carry_in[u * 8 + j];
      if (open_row[u] >= 0) break;
    }
    axpby_store8(Y + r * ldy, tot, alpha, beta, bz);
  } else if (t - tiles < nempty) {
#pragma unroll
    for (int j = 0; j < 8; ++j) tot[j] = V(0);
    axpby_store8(Y + empty[t - tiles] * ldy, tot, alpha, beta, bz);
  }
}

}  // namespace
}  // namespace spops

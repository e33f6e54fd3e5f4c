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

// ---- multi-RHS with k = 8 on the SpMV's tile plan (csr_tile_spmm8 and the
// batch's tile items)
template <typename V>
__device__ __forceinline__ void axpby_store8(V* __restrict__ y, const V (&v)[8], V alpha, V beta, bool bz) {
#pragma unroll
  for (int j = 0; j < 8; ++j) axpby_store(y + j, v[j], alpha, beta, bz);
}

// Half an X row (4 values) for the lane-pair form: 32 bytes for FP64, 16 for
// FP32.
template <typename V>
__device__ __forceinline__ void ld_xhalf(const V* __restrict__ p, V (&r)[4]) {
  if constexpr (sizeof(V) == 8) {
    uint32_t w[8];
    asm volatile("ld.global.nc.v8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
                 : "=r"(w[0]), "=r"(w[1]), "=r"(w[2]), "=r"(w[3]), "=r"(w[4]), "=r"(w[5]), "=r"(w[6]), "=r"(w[7])
                 : "l"(p));
    memcpy(r, w, 32);
  } else {
    uint32_t w[4];
    asm volatile("ld.global.nc.v4.b32 {%0,%1,%2,%3}, [%4];" : "=r"(w[0]), "=r"(w[1]), "=r"(w[2]), "=r"(w[3]) : "l"(p));
    memcpy(r, w, 16);
  }
}

// One tile t of a k = 8 product with lane pairs: lanes 2p and 2p + 1 take the
// 16 consecutive entries of the plan's lanes 2p and 2p + 1, lane 2p + h
// holding columns 4h .. 4h + 3.  Both lanes of a pair gather the same X row
// in one instruction (32 bytes each), so each row costs one request.  The
// pair's row starts are the two lanes' flags; the heads combine over the 16
// pairs with the segmented scan, and the row open at the tile's end goes to
// the 8-wide calibrator.  Every column is summed in an order fixed by the
// matrix.
template <typename I, typename V>
__device__ __forceinline__ void spmm8_tile_pairs(const I* __restrict__ rp, int64_t n, int64_t nnz,
                                                 const I* __restrict__ ci, const V* __restrict__ val,
                                                 const int64_t* __restrict__ tile_row,
                                                 const uint8_t* __restrict__ flags_all, int64_t t,
                                                 const V* __restrict__ X, int64_t ldx, V* __restrict__ Y, int64_t ldy,
                                                 V alpha, V beta, bool bz, V* __restrict__ carry_in,
                                                 V* __restrict__ open_sum, int64_t* __restrict__ open_row, int lane) {
  constexpr int K = 8;
  const int pr = lane >> 1, h = lane & 1;
  const uint32_t f16 = (uint32_t)flags_all[t * 32 + 2 * pr] | ((uint32_t)flags_all[t * 32 + 2 * pr + 1] << 8);
  const int64_t tr = tile_row[t];
  const int64_t e0 = t * (32 * K) + (int64_t)pr * 2 * K;
  // pair flags as a 16-bit mask (bit p: pair p holds a row start)
  const unsigned lane_f = __ballot_sync(0xffffffffu, f16 != 0 && h == 0);
  unsigned pf = 0;
#pragma unroll
  for (int q = 0; q < 16; ++q) pf |= ((lane_f >> (2 * q)) & 1u) << q;
  int64_t row;
  if (tr >= 0) {
    const int cnt = __popc(f16);
    const unsigned below = (1u << (2 * pr)) - 1u;  // lanes of the pairs before this one
    int excl = 0;
#pragma unroll
    for (int bit = 0; bit < 5; ++bit)
      excl += __popc(__ballot_sync(0xffffffffu, ((cnt >> bit) & 1) && h == 0) & below) << bit;
    const int first0 = (int)(__ballot_sync(0xffffffffu, f16 & 1u) & 1u);
    row = tr + excl + (int)(f16 & 1u) - first0;
  } else {
    row = row_holding(rp, n, e0 < nnz ? e0 : nnz - 1);
  }
  V acc[4], head[4];
#pragma unroll
  for (int j = 0; j < 4; ++j) acc[j] = head[j] = V(0);
  bool in_head = (f16 & 1u) == 0;
  V* Yh = Y + 4 * h;
#pragma unroll
  for (int run = 0; run < 2; ++run) {  // plan lane 2p, then 2p + 1
    I c[K];
    V a[K];
    tile_load<I, V, K>(ci, val, nnz, t, 2 * pr + run, c, a);
#pragma unroll
    for (int half = 0; half < 2; ++half) {
      V xr[4][4];
#pragma unroll
      for (int q = 0; q < 4; ++q) ld_xhalf(X + (int64_t)c[4 * half + q] * ldx + 4 * h, xr[q]);
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const int b = run * K + 4 * half + q;
        if (b > 0 && ((f16 >> b) & 1u)) {
          if (in_head) {
#pragma unroll
            for (int j = 0; j < 4; ++j) head[j] = acc[j];
            in_head = false;
          } else {
#pragma unroll
            for (int j = 0; j < 4; ++j) axpby_store(Yh + row * ldy + j, acc[j], alpha, beta, bz);
          }
#pragma unroll
          for (int j = 0; j < 4; ++j) acc[j] = V(0);
          ++row;
          if (tr < 0)
            while (row + 1 < n && rp[row] == rp[row + 1]) ++row;  // skip empty rows
        }
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          const V prod = a[4 * half + q] * xr[q][j];
          acc[j] += prod;
        }
      }
    }
  }
  V tail[4];
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    if (in_head) head[j] = acc[j];
    tail[j] = in_head ? V(0) : acc[j];
  }
  const bool has_flag = f16 != 0;
  const unsigned starts = (pf << 1) | 1u;  // pair p starts a segment if pair p - 1 is flagged (or p == 0)
#pragma unroll
  for (int o = 1; o < 16; o <<= 1) {
    const unsigned span = (pr >= o) ? ((2u << pr) - 1u) & ~((2u << (pr - o)) - 1u) : 0u;
    const bool add = pr >= o && !(starts & span);
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const V su = __shfl_up_sync(0xffffffffu, head[j], 2 * o);
      if (add) head[j] += su;
    }
  }
  const unsigned later = pf & ~((2u << pr) - 1u);
  const int m = later ? __ffs(later) - 1 : 15;
  const int m0 = pf ? __ffs(pf) - 1 : 15;
  V Sm[4], cin[4];
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    Sm[j] = __shfl_sync(0xffffffffu, head[j], 2 * m + h);
    cin[j] = __shfl_sync(0xffffffffu, head[j], 2 * m0 + h);
  }
  if (has_flag) {
    if (later) {
#pragma unroll
      for (int j = 0; j < 4; ++j) axpby_store(Yh + row * ldy + j, tail[j] + Sm[j], alpha, beta, bz);
    } else {  // the tile's last row: may continue into the next tile
#pragma unroll
      for (int j = 0; j < 4; ++j) open_sum[t * 8 + 4 * h + j] = tail[j] + (pr < 15 ? Sm[j] : V(0));
      if (h == 0) open_row[t] = row;
    }
  }
  if (pr == 0) {
#pragma unroll
    for (int j = 0; j < 4; ++j) carry_in[t * 8 + 4 * h + j] = cin[j];
    if (h == 0 && !pf) open_row[t] = -1;
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

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

// K elements of T to p (32-byte aligned) with 256-bit stores: a lane's run
// is written as whole 32-byte sectors.
template <typename T, int K>
__device__ __forceinline__ void store_run(T* __restrict__ p, const T (&v)[K]) {
  constexpr int BYTES = K * (int)sizeof(T);
  static_assert(BYTES % 32 == 0, "run must be a multiple of 32 bytes");
  unsigned long long w[BYTES / 8];
  memcpy(w, v, BYTES);
#pragma unroll
  for (int q = 0; q < BYTES / 32; ++q)
    asm volatile("st.global.v4.b64 [%0], {%1, %2, %3, %4};" ::"l"(reinterpret_cast<char*>(p) + 32 * q),
                 "l"(w[4 * q]), "l"(w[4 * q + 1]), "l"(w[4 * q + 2]), "l"(w[4 * q + 3])
                 : "memory");
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

// Given the products p of the lane's run: rows complete inside the lane go to
// y, the heads combine across lanes, the tile's open row and carry go to the
// calibrator arrays.
template <typename I, typename V, int K>
__device__ __forceinline__ void tile_finish(const I* __restrict__ rp, int64_t n, int64_t nnz, int64_t t, int lane,
                                            uint32_t flags, int64_t tr, const V (&p)[K], V* __restrict__ y, V alpha,
                                            V beta, bool bz, V* __restrict__ carry_in, V* __restrict__ open_sum,
                                            int64_t* __restrict__ open_row) {
  const unsigned lt = (1u << lane) - 1u;  // lanes below this one
  const int64_t el = t * (32 * K) + (int64_t)lane * K;
  // ---- row of the lane's first entry
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
  // ---- in-lane segments
  V head = V(0), acc = V(0);
  bool in_head = (flags & 1u) == 0;
#pragma unroll
  for (int b = 0; b < K; ++b) {
    if (b > 0 && ((flags >> b) & 1u)) {
      if (in_head) {
        head = acc;
        in_head = false;
      } else {
        axpby_store(y + row, acc, alpha, beta, bz);
      }
      acc = V(0);
      ++row;
      if (tr < 0)
        while (row + 1 < n && rp[row] == rp[row + 1]) ++row;  // skip empty rows
    }
    acc += p[b];
  }
  V tail = V(0);
  if (in_head) head = acc; else tail = acc;
  // ---- cross-lane: segmented inclusive scan of the heads, a segment
  // starting right after every flagged lane
  const bool has_flag = flags != 0;
  const unsigned fmask = __ballot_sync(0xffffffffu, has_flag);
  const unsigned starts = (fmask << 1) | 1u;  // lane l starts a segment if lane l-1 is flagged (or l == 0)
  V S = head;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const V su = __shfl_up_sync(0xffffffffu, S, o);
    // add lane (l - o)'s sum unless a segment starts in lanes l-o+1 .. l
    const unsigned span = (lane >= o) ? ((2u << lane) - 1u) & ~((2u << (lane - o)) - 1u) : 0u;
    if (lane >= o && !(starts & span)) S += su;
  }
  const unsigned later = fmask & ~((2u << lane) - 1u);  // flagged lanes after this one
  const int m = later ? __ffs(later) - 1 : 31;
  const V Sm = __shfl_sync(0xffffffffu, S, m);
  const int m0 = fmask ? __ffs(fmask) - 1 : 31;
  const V cin = __shfl_sync(0xffffffffu, S, m0);
  if (has_flag) {
    if (later) {
      axpby_store(y + row, tail + Sm, alpha, beta, bz);
    } else {  // the tile's last row: may continue into the next tile
      open_sum[t] = tail + (lane < 31 ? Sm : V(0));
      open_row[t] = row;
    }
  }
  if (lane == 0) {
    carry_in[t] = cin;
    if (!fmask) open_row[t] = -1;
  }
}

// Calibration of one tile t (t < tiles) or empty row (t - tiles < nempty)
// of a single-vector product: the row open at tile t's end receives the heads
// of the following tiles up to the first one that starts a row.
template <typename V>
__device__ __forceinline__ void spmv_calibrate1(int64_t t, int64_t tiles, const V* __restrict__ carry_in,
                                                const V* __restrict__ open_sum, const int64_t* __restrict__ open_row,
                                                const int64_t* __restrict__ empty, int64_t nempty, V* __restrict__ y,
                                                V alpha, V beta, bool bz) {
  if (t < tiles) {
    const int64_t r = open_row[t];
    if (r < 0) return;
    V tot = open_sum[t];
    for (int64_t u = t + 1; u < tiles; ++u) {
      tot += carry_in[u];
      if (open_row[u] >= 0) break;
    }
    axpby_store(y + r, tot, alpha, beta, bz);
  } else if (t - tiles < nempty) {
    axpby_store(y + empty[t - tiles], V(0), alpha, beta, bz);
  }
}

// ---- multi-RHS with k = 8, 16, 32 on the SpMV's tile plan (csr_tile_spmm
// and the batch's tile items)
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

// One tile t of a multi-RHS product with k = 4G columns, G lanes per entry:
// group q (lanes qG .. qG + G - 1) takes the 8G consecutive entries of the
// plan's lanes qG .. qG + G - 1, lane qG + h holding columns 4h .. 4h + 3.
// The group's lanes gather an entry's whole X row in one instruction (32
// bytes each for FP64), so a row costs one L2 request per 128 bytes.  The
// group's row starts are its G lanes' flags; the heads combine over the 32/G
// groups with the segmented scan, and the row open at the tile's end goes to
// the k-wide calibrator.  Every column is summed in an order fixed by the
// matrix.
template <typename I, typename V, int G>
__device__ __forceinline__ void spmm_tile_groups(const I* __restrict__ rp, int64_t n, int64_t nnz,
                                                 const I* __restrict__ ci, const V* __restrict__ val,
                                                 const int64_t* __restrict__ tile_row,
                                                 const uint8_t* __restrict__ flags_all, int64_t t,
                                                 const V* __restrict__ X, int64_t ldx, V* __restrict__ Y, int64_t ldy,
                                                 V alpha, V beta, bool bz, V* __restrict__ carry_in,
                                                 V* __restrict__ open_sum, int64_t* __restrict__ open_row, int lane) {
  constexpr int K = 8, NG = 32 / G, KC = 4 * G;
  static_assert(G == 2 || G == 4 || G == 8, "2, 4 or 8 lanes per entry");
  const int gq = lane / G, h = lane % G;
  uint64_t fl = 0;  // bit b: entry b of the group's 8G starts a row
#pragma unroll
  for (int r = 0; r < G; ++r) fl |= (uint64_t)flags_all[t * 32 + gq * G + r] << (8 * r);
  const int64_t tr = tile_row[t];
  const int64_t e0 = t * (32 * K) + (int64_t)gq * G * K;
  // group flags as an NG-bit mask (bit q: group q holds a row start)
  const unsigned lane_f = __ballot_sync(0xffffffffu, fl != 0 && h == 0);
  unsigned gf = 0;
#pragma unroll
  for (int q = 0; q < NG; ++q) gf |= ((lane_f >> (G * q)) & 1u) << q;
  int64_t row;
  if (tr >= 0) {
    const int cnt = __popcll(fl);
    const unsigned below = (gq * G >= 32) ? 0xffffffffu : ((1u << (gq * G)) - 1u);  // lanes of earlier groups
    int excl = 0;
#pragma unroll
    for (int bit = 0; bit < 7; ++bit)
      excl += __popc(__ballot_sync(0xffffffffu, ((cnt >> bit) & 1) && h == 0) & below) << bit;
    const int first0 = (int)(__ballot_sync(0xffffffffu, fl & 1u) & 1u);
    row = tr + excl + (int)(fl & 1u) - first0;
  } else {
    row = row_holding(rp, n, e0 < nnz ? e0 : nnz - 1);
  }
  V acc[4], head[4];
#pragma unroll
  for (int j = 0; j < 4; ++j) acc[j] = head[j] = V(0);
  bool in_head = (fl & 1u) == 0;
  V* Yh = Y + 4 * h;
#pragma unroll 1
  for (int run = 0; run < G; ++run) {  // plan lanes qG, qG + 1, ...
    I c[K];
    V a[K];
    tile_load<I, V, K>(ci, val, nnz, t, gq * G + run, c, a);
#pragma unroll
    for (int half = 0; half < 2; ++half) {
      V xr[4][4];
#pragma unroll
      for (int q = 0; q < 4; ++q) ld_xhalf(X + (int64_t)c[4 * half + q] * ldx + 4 * h, xr[q]);
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const int b = run * K + 4 * half + q;
        if (b > 0 && ((fl >> b) & 1u)) {
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
  const bool has_flag = fl != 0;
  const unsigned starts = (gf << 1) | 1u;  // group q starts a segment if group q - 1 is flagged (or q == 0)
#pragma unroll
  for (int o = 1; o < NG; o <<= 1) {
    const unsigned span = (gq >= o) ? ((2u << gq) - 1u) & ~((2u << (gq - o)) - 1u) : 0u;
    const bool add = gq >= o && !(starts & span);
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const V su = __shfl_up_sync(0xffffffffu, head[j], G * o);
      if (add) head[j] += su;
    }
  }
  const unsigned later = gf & ~((2u << gq) - 1u);
  const int m = later ? __ffs(later) - 1 : NG - 1;
  const int m0 = gf ? __ffs(gf) - 1 : NG - 1;
  V Sm[4], cin[4];
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    Sm[j] = __shfl_sync(0xffffffffu, head[j], G * m + h);
    cin[j] = __shfl_sync(0xffffffffu, head[j], G * m0 + h);
  }
  if (has_flag) {
    if (later) {
#pragma unroll
      for (int j = 0; j < 4; ++j) axpby_store(Yh + row * ldy + j, tail[j] + Sm[j], alpha, beta, bz);
    } else {  // the tile's last row: may continue into the next tile
#pragma unroll
      for (int j = 0; j < 4; ++j) open_sum[t * KC + 4 * h + j] = tail[j] + (gq < NG - 1 ? Sm[j] : V(0));
      if (h == 0) open_row[t] = row;
    }
  }
  if (gq == 0) {
#pragma unroll
    for (int j = 0; j < 4; ++j) carry_in[t * KC + 4 * h + j] = cin[j];
    if (h == 0 && !gf) open_row[t] = -1;
  }
}

// Calibration of one tile t (t < tiles) or empty row (t - tiles < nempty)
// of a product with KC columns (8 at a time).
template <typename V, int KC>
__device__ __forceinline__ void spmm_calibrate(int64_t t, int64_t tiles, const V* __restrict__ carry_in,
                                               const V* __restrict__ open_sum, const int64_t* __restrict__ open_row,
                                               const int64_t* __restrict__ empty, int64_t nempty, V* __restrict__ Y,
                                               int64_t ldy, V alpha, V beta, bool bz) {
  V tot[8];
  if (t < tiles) {
    const int64_t r = open_row[t];
    if (r < 0) return;
    for (int c0 = 0; c0 < KC; c0 += 8) {
#pragma unroll
      for (int j = 0; j < 8; ++j) tot[j] = open_sum[t * KC + c0 + j];
      for (int64_t u = t + 1; u < tiles; ++u) {
#pragma unroll
        for (int j = 0; j < 8; ++j) tot[j] += carry_in[u * KC + c0 + j];
        if (open_row[u] >= 0) break;
      }
      axpby_store8(Y + r * ldy + c0, tot, alpha, beta, bz);
    }
  } else if (t - tiles < nempty) {
#pragma unroll
    for (int j = 0; j < 8; ++j) tot[j] = V(0);
    for (int c0 = 0; c0 < KC; c0 += 8) axpby_store8(Y + empty[t - tiles] * ldy + c0, tot, alpha, beta, bz);
  }
}

}  // namespace
}  // namespace spops

// Warp-level units of SpMV work shared by the single-matrix kernels
// (spmv_csr.cu, formats.cu) and the batched persistent kernel (batched.cu).
#pragma once

#include "device_util.cuh"
#include "spops_internal.h"

namespace spops {

// CSR segments: a short segment holds < 2*kCsrCap entries of at most
// kCsrRowCap rows; a long row is cut into chunks of kCsrCap entries.
constexpr int kCsrCap = 256;
constexpr int kCsrRowCap = 32;
// Largest half-width of the x window a segment stages in shared memory
// (csr_segment_spmv with band > 0): rows [r0, r0 + nr) read x[r0 - band,
// r0 + nr + band) from the window, every other column from global memory.
constexpr int kBandMax = 64;
constexpr int kBandWin = kCsrRowCap + 2 * kBandMax;

// Padded rows (SELL / ELL): stored rows longer than kPadLong slots are summed
// by pieces of kPadPiece slots, one warp per piece.
constexpr int kPadLong = 2048;
constexpr int kPadPiece = 2048;

__device__ __forceinline__ int lanes_per_row(int nr) {
  const int t = 32 / (nr > 0 ? nr : 1);
  return t >= 32 ? 32 : t >= 16 ? 16 : t >= 8 ? 8 : t >= 4 ? 4 : t >= 2 ? 2 : 1;
}

// Sum of the chunk sums of one long row, by the last chunk to finish (fixed
// order, so deterministic).  `first` is the row's first chunk slot.  Returns
// true (in all lanes) on the warp that wrote y.
template <typename V>
__device__ __forceinline__ void warp_chunk_finish(V sum, int64_t slot, int64_t first, int nchunks, V* __restrict__ yrow,
                                                  V* __restrict__ partial, int* __restrict__ counter, V alpha,
                                                  V beta, bool bz, int lane) {
  int last = 0;
  if (lane == 0) {
    partial[slot] = sum;
    __threadfence();
    last = (atomicAdd(counter + first, 1) == nchunks - 1);
  }
  last = __shfl_sync(0xffffffffu, last, 0);
  if (last) {
    __threadfence();
    V tot = V(0);
    for (int q = lane; q < nchunks; q += 32) tot += ld_cg(partial + first + q);
    tot = warp_sum(tot);
    if (lane == 0) {
      axpby_store(yrow, tot, alpha, beta, bz);
      counter[first] = 0;
    }
  }
}

// One CSR segment j (descriptor d) with a whole warp.  prod: the warp's
// 2*kCsrCap shared-memory slice.  Short segment: coalesced evict-first loads
// of kItems entries per lane per round, every gather of the round issued
// before use, products to shared memory, then t lanes reduce each row.  Long
// chunk: register sum, warp reduction, chunk combine.
//
// band > 0 (x window staging): the warp first copies x[r0 - band, r0 + nr +
// band) (coalesced, out-of-range slots zero) into xs, its kBandWin-entry
// shared-memory slice; a column inside the window is read from there, any
// other with a global gather.  The products and their order are unchanged.
template <typename I, typename V, int kItems>
__device__ __forceinline__ void csr_segment_spmv(const CsrSeg& d, int64_t j, const I* __restrict__ ci,
                                                 const V* __restrict__ val, const I* __restrict__ rp,
                                                 const V* __restrict__ x, V* __restrict__ y, V alpha, V beta,
                                                 bool bz, V* __restrict__ prod, V* __restrict__ partial,
                                                 int* __restrict__ counter, int lane, int band = 0,
                                                 int64_t ncols = 0, V* __restrict__ xs = nullptr) {
  const int m = (int)(d.p1 - d.p0);
  const bool is_long = d.chunk >= 0;
  const I* cseg = ci + d.p0;
  const V* vseg = val + d.p0;
  V lsum = V(0);
  const int64_t w0 = (int64_t)d.r0 - band;
  int W = 0;
  if (band > 0) {
    W = (is_long ? 1 : d.nr) + 2 * band;
    __syncwarp();  // the previous item's reads of xs are done
    for (int t = lane; t < W; t += 32) {
      const int64_t c = w0 + t;
      xs[t] = (c >= 0 && c < ncols) ? ld_gather(x + c) : V(0);
    }
    __syncwarp();
  }
  for (int base = 0; base < m; base += 32 * kItems) {
    I c[kItems];
    V a[kItems];
#pragma unroll
    for (int it = 0; it < kItems; ++it) {
      const int k = base + lane + 32 * it;
      if (k < m) {
        c[it] = ld_stream(cseg + k);
        a[it] = ld_stream(vseg + k);
      }
    }
#pragma unroll
    for (int it = 0; it < kItems; ++it) {
      const int k = base + lane + 32 * it;
      if (k < m) {
        const int64_t o = (int64_t)c[it] - w0;
        const V p = a[it] * ((o >= 0 && o < W) ? xs[o] : ld_gather(x + c[it]));
        if (is_long) lsum += p; else prod[k] = p;
      }
    }
  }
  if (!is_long) {
    __syncwarp();
    const int nr = d.nr;
    const int t = lanes_per_row(nr);
    const int groups = 32 / t, g = lane / t, sub = lane % t;
    for (int rb = 0; rb < nr; rb += groups) {
      const int rr = rb + g;
      V s0 = V(0), s1 = V(0);
      if (rr < nr) {
        const int s = (int)((int64_t)rp[d.r0 + rr] - d.p0), e = (int)((int64_t)rp[d.r0 + rr + 1] - d.p0);
        int k = s + sub;
        for (; k + t < e; k += 2 * t) {
          s0 += prod[k];
          s1 += prod[k + t];
        }
        if (k < e) s0 += prod[k];
      }
      const V sum = warp_sum(s0 + s1, t);
      if (rr < nr && sub == 0) axpby_store(y + d.r0 + rr, sum, alpha, beta, bz);
    }
    __syncwarp();
  } else {
    lsum = warp_sum(lsum);
    warp_chunk_finish(lsum, j, j - d.chunk, d.nr, y + d.r0, partial, counter, alpha, beta, bz, lane);
  }
}

// Multi-RHS CSR segment: Y[r, 0:k] = alpha * A[r,:] X[:, 0:k] + beta * Y[r, 0:k]
// (row-major X [cols x ldx], Y [rows x ldy]).  The segment's X row offsets
// (column * ldx), values and row starts are first staged in the warp's
// SpmmStage (one coalesced pass), so the gathers need no dependent global
// loads.  The warp is 32/KT groups of KT lanes; lane rl of a group owns RHS
// column t0 + rl.  A short segment gives each group a run of whole rows
// holding about a 32/KT-th of its entries; the group streams that run in
// batches of U entries (U gathers per lane in flight) that cross row
// boundaries, storing each row as its last entry passes.  A long-row chunk is
// split between the groups, whose sums combine with xor shuffles; chunk sums
// then combine through partial[slot * k + r].  Every sum is taken in a fixed
// order, so results are bit-reproducible.
template <typename I, typename V>
struct SpmmStage {
  int64_t off[2 * kCsrCap];  // column * ldx
  V a[2 * kCsrCap];
  int rs[kCsrRowCap + 1];
};

// Entries [e0, e1) of the stage, rows [r, r_end) with starts rs (rs[r_end] >=
// e1): Y[row] = alpha * sum + beta * Y[row] per row as the stream passes it.
// With rs == nullptr the range is one row's chunk and its sum is returned.
template <typename I, typename V, int U>
__device__ __forceinline__ V spmm_stream(const SpmmStage<I, V>& S, const V* __restrict__ X, int e0, int e1,
                                         const int* rs, int r, int r_end, int64_t col0, bool rok,
                                         V* __restrict__ Yrow0, int64_t ldy, V alpha, V beta, bool bz) {
  V acc = V(0);
  int next = rs ? (r < r_end ? rs[r + 1] : e1) : e1;
  if (rs)
    while (r < r_end && next <= e0) {  // empty rows before the first entry
      if (rok) axpby_store_cs(Yrow0 + (int64_t)r * ldy + col0, acc, alpha, beta, bz);
      ++r;
      next = r < r_end ? rs[r + 1] : e1;
    }
  for (int eb = e0; eb < e1; eb += U) {
    V xv[U];
#pragma unroll
    for (int q = 0; q < U; ++q) {
      const int e = eb + q;
      xv[q] = (e < e1 && rok) ? ld_gather(X + S.off[e] + col0) : V(0);
    }
#pragma unroll
    for (int q = 0; q < U; ++q) {
      const int e = eb + q;
      if (e < e1) {
        if (rs)
          while (e >= next) {  // rows that end before entry e
            if (rok) axpby_store_cs(Yrow0 + (int64_t)r * ldy + col0, acc, alpha, beta, bz);
            acc = V(0);
            ++r;
            next = rs[r + 1];
          }
        acc += S.a[e] * xv[q];
      }
    }
  }
  if (rs)
    while (r < r_end) {
      if (rok) axpby_store_cs(Yrow0 + (int64_t)r * ldy + col0, acc, alpha, beta, bz);
      acc = V(0);
      ++r;
    }
  return acc;
}

template <typename I, typename V, int KT>
__device__ __forceinline__ void csr_segment_spmm(const CsrSeg& d, int64_t j, const I* __restrict__ ci,
                                                 const V* __restrict__ val, const I* __restrict__ rp,
                                                 const V* __restrict__ X, int64_t ldx, V* __restrict__ Y,
                                                 int64_t ldy, int64_t k, V alpha, V beta, bool bz,
                                                 V* __restrict__ partial, int* __restrict__ counter,
                                                 SpmmStage<I, V>& S, int lane) {
  constexpr int P = 32 / KT;
  constexpr int U = KT == 32 ? 16 : 8;
  const int grp = lane / KT, rl = lane % KT;
  const int m = (int)(d.p1 - d.p0);
  const bool is_long = d.chunk >= 0;
  // stage: all loads of a round issued before any store (8 entries per lane
  // in flight), the row starts in the first round
  constexpr int kStageItems = 8;
  __syncwarp();  // the previous segment's reads of the stage are done
  for (int base = 0; base < m || base == 0; base += 32 * kStageItems) {
    I c[kStageItems];
    V a[kStageItems];
#pragma unroll
    for (int u = 0; u < kStageItems; ++u) {
      const int e = base + lane + 32 * u;
      if (e < m) {
        c[u] = ld_stream(ci + d.p0 + e);
        a[u] = ld_stream(val + d.p0 + e);
      }
    }
    I r0v = 0, r1v = 0;
    if (base == 0 && !is_long) {
      if (lane <= d.nr) r0v = rp[d.r0 + lane];
      if (lane + 32 <= d.nr) r1v = rp[d.r0 + lane + 32];
    }
#pragma unroll
    for (int u = 0; u < kStageItems; ++u) {
      const int e = base + lane + 32 * u;
      if (e < m) {
        S.off[e] = (int64_t)c[u] * ldx;
        S.a[e] = a[u];
      }
    }
    if (base == 0 && !is_long) {
      if (lane <= d.nr) S.rs[lane] = (int)((int64_t)r0v - d.p0);
      if (lane + 32 <= d.nr) S.rs[lane + 32] = (int)((int64_t)r1v - d.p0);
    }
  }
  __syncwarp();
  if (!is_long) {
    // rows of this group: those starting in [m*grp/P, m*(grp+1)/P)
    auto first_row = [&](int g) {
      if (g >= P) return d.nr;
      const int target = (int)((int64_t)m * g / P);
      int lo = 0, hi = d.nr;  // first r in [0, nr] with rs[r] >= target
      while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (S.rs[mid] < target) lo = mid + 1; else hi = mid;
      }
      return g == 0 ? 0 : lo;
    };
    const int rb = first_row(grp), re = first_row(grp + 1);
    if (rb < re)
      for (int64_t t0 = 0; t0 < k; t0 += KT)
        spmm_stream<I, V, U>(S, X, S.rs[rb], S.rs[re], S.rs, rb, re, t0 + rl, t0 + rl < k, Y + d.r0 * ldy, ldy,
                             alpha, beta, bz);
    __syncwarp();
  } else {
    // chunk sums per RHS column; the last chunk of the row adds them in order
    const int e0 = (int)((int64_t)m * grp / P), e1 = (int)((int64_t)m * (grp + 1) / P);
    for (int64_t t0 = 0; t0 < k; t0 += KT) {
      const bool rok = t0 + rl < k;
      V s = spmm_stream<I, V, U>(S, X, e0, e1, nullptr, 0, 0, t0 + rl, rok, nullptr, 0, alpha, beta, bz);
      __syncwarp();
#pragma unroll
      for (int o = KT; o < 32; o <<= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
      if (grp == 0 && rok) partial[j * k + t0 + rl] = s;
    }
    __threadfence();
    __syncwarp();
    const int64_t first = j - d.chunk;
    int last = 0;
    if (lane == 0) last = (atomicAdd(counter + first, 1) == d.nr - 1);
    last = __shfl_sync(0xffffffffu, last, 0);
    if (last) {
      __threadfence();
      for (int64_t t = lane; t < k; t += 32) {
        V tot = V(0);
        for (int q = 0; q < d.nr; ++q) tot += ld_cg(partial + (first + q) * k + t);
        axpby_store(Y + d.r0 * ldy + t, tot, alpha, beta, bz);
      }
      __syncwarp();
      if (lane == 0) counter[first] = 0;
    }
  }
}

// Padded rows: stored rows [i0, i0+32) with one warp (see formats.cu).
// Sum of one lane's row in a column-major chunk: slots [0, len) at base +
// k * stride.  Eight slots at a time: their columns and values are loaded,
// then their eight x gathers issued, before any is added, so each lane keeps
// eight gathers in flight.  Even slots go to one sum and odd slots to the
// other, in slot order (padding columns, -1, are skipped).
template <typename I, typename V>
__device__ __forceinline__ V colmajor_row_sum(const I* __restrict__ col, const V* __restrict__ val,
                                              const V* __restrict__ x, int64_t base, int len, int64_t stride) {
  V s0 = V(0), s1 = V(0);
  int k = 0;
  for (; k + 8 <= len; k += 8) {
    I c[8];
    V a[8], p[8];
#pragma unroll
    for (int u = 0; u < 8; ++u) {
      const int64_t e = base + (int64_t)(k + u) * stride;
      c[u] = ld_stream(col + e);
      a[u] = ld_stream(val + e);
    }
#pragma unroll
    for (int u = 0; u < 8; ++u) p[u] = c[u] >= 0 ? a[u] * ld_gather(x + c[u]) : V(0);
#pragma unroll
    for (int u = 0; u < 8; ++u)
      if (c[u] >= 0) {
        if (u & 1) s1 += p[u]; else s0 += p[u];
      }
  }
  for (; k + 1 < len; k += 2) {
    const int64_t a = base + (int64_t)k * stride, b = a + stride;
    const I ca = ld_stream(col + a), cb = ld_stream(col + b);
    if (ca >= 0) s0 += ld_stream(val + a) * ld_gather(x + ca);
    if (cb >= 0) s1 += ld_stream(val + b) * ld_gather(x + cb);
  }
  if (k < len) {
    const int64_t a = base + (int64_t)k * stride;
    const I ca = ld_stream(col + a);
    if (ca >= 0) s0 += ld_stream(val + a) * ld_gather(x + ca);
  }
  return s0 + s1;
}

template <typename I, typename V, bool kColMajor>
__device__ __forceinline__ void padded_rows32(int64_t i0, const I* __restrict__ col, const V* __restrict__ val,
                                              const I* __restrict__ chunk_len,
                                              const int64_t* __restrict__ chunk_off,
                                              const int* __restrict__ row_len, const I* __restrict__ reorder,
                                              int64_t n, int64_t C, const V* __restrict__ x, V* __restrict__ y,
                                              V alpha, V beta, bool bz, int lane) {
  const int64_t i = i0 + lane;
  int len = 0;
  int64_t base = 0;
  if (i < n) {
    len = row_len[i];
    if (len > kPadLong) len = -1;  // long row: summed by pieces
    const int64_t c = i / C;
    base = chunk_off[c] + (kColMajor ? (i - c * C) : (i - c * C) * (int64_t)chunk_len[c]);
  }
  if (kColMajor) {
    const V s = colmajor_row_sum<I, V>(col, val, x, base, len, C);
    if (i < n && len >= 0) axpby_store(y + (reorder ? (int64_t)reorder[i] : i), s, alpha, beta, bz);
  } else {
    const unsigned ml = __reduce_max_sync(0xffffffffu, (unsigned)(len > 0 ? len : 0));
    int t = 1;
    while (t < 32 && (unsigned)(t * 4) < ml) t <<= 1;
    const int per = 32 / t, sub = lane % t;
    for (int p = 0; p < t; ++p) {
      const int jj = p * per + lane / t;
      const int L = __shfl_sync(0xffffffffu, len, jj);
      const int64_t b = __shfl_sync(0xffffffffu, base, jj);
      V s0 = V(0), s1 = V(0);
      int k = sub;
      for (; k + t < L; k += 2 * t) {
        const I ca = ld_stream(col + b + k), cb = ld_stream(col + b + k + t);
        if (ca >= 0) s0 += ld_stream(val + b + k) * ld_gather(x + ca);
        if (cb >= 0) s1 += ld_stream(val + b + k + t) * ld_gather(x + cb);
      }
      if (k < L) {
        const I ca = ld_stream(col + b + k);
        if (ca >= 0) s0 += ld_stream(val + b + k) * ld_gather(x + ca);
      }
      const V sum = warp_sum(s0 + s1, t);
      const int64_t row = i0 + jj;
      if (sub == 0 && row < n && L >= 0) axpby_store(y + (reorder ? (int64_t)reorder[row] : row), sum, alpha, beta, bz);
    }
  }
}

// Steps (slots per row) of a 32-row column-major chunk that one warp takes:
// chunks with longer rows are cut into windows of kPadWindow steps, each its
// own warp, whose per-row partial sums the last window to finish adds up.
constexpr int kPadWindow = 128;

// Window [k0, k0 + kPadWindow) of a column-major chunk of exactly 32 rows,
// with one warp; emit(r, sum) receives the sum of row i0 + r over the window,
// exactly once per row.  The window's rows are ranked by length (longest
// first, one bitonic sort across the warp); in phase p = 0..5 the 32 >> p
// longest unfinished rows get 1 << p lanes each, which take every (1 << p)-th
// slot, until the row of rank (32 >> p) / 2 runs out; rows that finish in a
// phase are reduced over their lanes and emitted.  So a window whose rows
// differ in length (SELL-C-sigma with a small sigma) keeps its lanes busy
// instead of idling on padding; balanced windows keep one lane per row, as
// every phase costs a memory round trip.  `len` is the row's slot count
// (0 for rows handled elsewhere).
template <typename I, typename V, typename Emit>
__device__ __forceinline__ void padded_window32(int64_t base, int len, int k0, const I* __restrict__ col,
                                                const V* __restrict__ val, const V* __restrict__ x, int lane,
                                                Emit&& emit) {
  len = len - k0;
  len = len < 0 ? 0 : (len > kPadWindow ? kPadWindow : len);
  base += 32 * (int64_t)k0;
  const unsigned total = __reduce_add_sync(0xffffffffu, (unsigned)len);
  const unsigned longest = __reduce_max_sync(0xffffffffu, (unsigned)len);
  if (32u * longest <= total + total / 4 + 32u * 8u) {
    emit(lane, colmajor_row_sum<I, V>(col, val, x, base + lane, len, 32));
    return;
  }
  // rank rows by length, descending (ties: lower row first)
  uint32_t key = ((uint32_t)len << 5) | (uint32_t)(31 - lane);
#pragma unroll
  for (int kk = 2; kk <= 32; kk <<= 1) {
#pragma unroll
    for (int jj = kk >> 1; jj > 0; jj >>= 1) {
      const uint32_t other = __shfl_xor_sync(0xffffffffu, key, jj);
      const bool first_half = (lane & kk) == 0, lower = (lane & jj) == 0;
      key = (lower == first_half) ? (key > other ? key : other) : (key < other ? key : other);
    }
  }
  const int rank_len = (int)(key >> 5), rank_row = 31 - (int)(key & 31u);
  V sum = V(0);
  int kbeg = 0;
#pragma unroll 1
  for (int p = 0; p < 6; ++p) {
    const int R = 32 >> p, g = 1 << p;
    const int q = lane & (R - 1), sub = lane >> (5 - p);
    const int L = __shfl_sync(0xffffffffu, rank_len, q);
    const int r = __shfl_sync(0xffffffffu, rank_row, q);
    const int kend = __shfl_sync(0xffffffffu, rank_len, R > 1 ? R / 2 : 0);
    const int lim = L < kend ? L : kend;
    const int64_t rb = base + r;
    V s0 = V(0), s1 = V(0);
    int k = kbeg + sub;
    for (; k + g < lim; k += 2 * g) {
      const int64_t a = rb + 32 * (int64_t)k, b = a + 32 * (int64_t)g;
      const I ca = ld_stream(col + a), cb = ld_stream(col + b);
      const V va = ld_stream(val + a), vb = ld_stream(val + b);
      if (ca >= 0) s0 += va * ld_gather(x + ca);
      if (cb >= 0) s1 += vb * ld_gather(x + cb);
    }
    if (k < lim) {
      const int64_t a = rb + 32 * (int64_t)k;
      const I ca = ld_stream(col + a);
      const V va = ld_stream(val + a);
      if (ca >= 0) s0 += va * ld_gather(x + ca);
    }
    sum += s0 + s1;
    // rows of rank [R/2, R) end in this phase (rank 0 in the last one)
    V tot = sum;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1)
      if (o >= R) tot += __shfl_xor_sync(0xffffffffu, tot, o);
    if (q >= (R > 1 ? R / 2 : 0)) {
      if (sub == 0) emit(r, tot);
      sum = V(0);
    }
    kbeg = kend;
  }
}

// One piece q of a long padded row, with one warp.
template <typename I, typename V, bool kColMajor>
__device__ __forceinline__ void padded_piece(int64_t q, const PadPiece& pc, const I* __restrict__ col,
                                             const V* __restrict__ val, const I* __restrict__ chunk_len,
                                             const int64_t* __restrict__ chunk_off, const int* __restrict__ row_len,
                                             const I* __restrict__ reorder, int64_t C, const V* __restrict__ x,
                                             V* __restrict__ y, V alpha, V beta, bool bz, V* __restrict__ partial,
                                             int* __restrict__ counter, int lane) {
  const int64_t i = pc.row;
  const int len = row_len[i];
  const int64_t c = i / C;
  const int64_t base = chunk_off[c] + (kColMajor ? (i - c * C) : (i - c * C) * (int64_t)chunk_len[c]);
  const int64_t stride = kColMajor ? C : 1;
  const int64_t k0 = (int64_t)pc.piece * kPadPiece;
  const int64_t k1 = (k0 + kPadPiece < len) ? k0 + kPadPiece : len;
  V s0 = V(0), s1 = V(0);
  int64_t k = k0 + lane;
  for (; k + 32 < k1; k += 64) {
    const int64_t a = base + k * stride, b = base + (k + 32) * stride;
    const I ca = ld_stream(col + a), cb = ld_stream(col + b);
    if (ca >= 0) s0 += ld_stream(val + a) * ld_gather(x + ca);
    if (cb >= 0) s1 += ld_stream(val + b) * ld_gather(x + cb);
  }
  if (k < k1) {
    const int64_t a = base + k * stride;
    const I ca = ld_stream(col + a);
    if (ca >= 0) s0 += ld_stream(val + a) * ld_gather(x + ca);
  }
  const V sum = warp_sum(s0 + s1);
  warp_chunk_finish(sum, q, q - pc.piece, pc.npieces, y + (reorder ? (int64_t)reorder[i] : i), partial, counter,
                    alpha, beta, bz, lane);
}

}  // namespace spops

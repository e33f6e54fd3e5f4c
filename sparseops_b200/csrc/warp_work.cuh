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
template <typename I, typename V, int kItems>
__device__ __forceinline__ void csr_segment_spmv(const CsrSeg& d, int64_t j, const I* __restrict__ ci,
                                                 const V* __restrict__ val, const I* __restrict__ rp,
                                                 const V* __restrict__ x, V* __restrict__ y, V alpha, V beta,
                                                 bool bz, V* __restrict__ prod, V* __restrict__ partial,
                                                 int* __restrict__ counter, int lane) {
  const int m = (int)(d.p1 - d.p0);
  const bool is_long = d.chunk >= 0;
  const I* cseg = ci + d.p0;
  const V* vseg = val + d.p0;
  V lsum = V(0);
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
        const V p = a[it] * ld_gather(x + c[it]);
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
// (row-major X [cols x ldx], Y [rows x ldy]).  Lanes = KT RHS columns x
// 32/KT entry groups; rows of the segment one after another; the entry-group
// partial sums combine with xor shuffles (fixed order).  Long chunks combine
// through partial[slot * k + r].
template <typename I, typename V, int KT>
__device__ __forceinline__ void csr_segment_spmm(const CsrSeg& d, int64_t j, const I* __restrict__ ci,
                                                 const V* __restrict__ val, const I* __restrict__ rp,
                                                 const V* __restrict__ X, int64_t ldx, V* __restrict__ Y,
                                                 int64_t ldy, int64_t k, V alpha, V beta, bool bz,
                                                 V* __restrict__ partial, int* __restrict__ counter, int lane) {
  constexpr int P = 32 / KT;
  const int grp = lane / KT, rl = lane % KT;
  auto row_dot = [&](int64_t e0, int64_t e1, int64_t t0) {
    const bool rok = t0 + rl < k;
    V s0 = V(0), s1 = V(0);
    int64_t e = e0 + grp;
    for (; e + P < e1; e += 2 * P) {
      const V a0 = val[e], a1 = val[e + P];
      const I c0 = ci[e], c1 = ci[e + P];
      if (rok) {
        s0 += a0 * ld_gather(X + (int64_t)c0 * ldx + t0 + rl);
        s1 += a1 * ld_gather(X + (int64_t)c1 * ldx + t0 + rl);
      }
    }
    if (e < e1 && rok) s0 += val[e] * ld_gather(X + (int64_t)ci[e] * ldx + t0 + rl);
    V s = s0 + s1;
#pragma unroll
    for (int o = KT; o < 32; o <<= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    return s;
  };
  if (d.chunk < 0) {
    for (int rr = 0; rr < d.nr; ++rr) {
      const int64_t r = d.r0 + rr;
      const int64_t e0 = rp[r], e1 = rp[r + 1];
      for (int64_t t0 = 0; t0 < k; t0 += KT) {
        const V s = row_dot(e0, e1, t0);
        if (grp == 0 && t0 + rl < k) axpby_store(Y + r * ldy + t0 + rl, s, alpha, beta, bz);
      }
    }
  } else {
    // chunk sums per RHS column; the last chunk of the row adds them in order
    for (int64_t t0 = 0; t0 < k; t0 += KT) {
      const V s = row_dot(d.p0, d.p1, t0);
      if (grp == 0 && t0 + rl < k) partial[j * k + t0 + rl] = s;
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
    V s0 = V(0), s1 = V(0);
    int k = 0;
    for (; k + 1 < len; k += 2) {
      const int64_t a = base + (int64_t)k * C, b = a + C;
      const I ca = ld_stream(col + a), cb = ld_stream(col + b);
      if (ca >= 0) s0 += ld_stream(val + a) * ld_gather(x + ca);
      if (cb >= 0) s1 += ld_stream(val + b) * ld_gather(x + cb);
    }
    if (k < len) {
      const int64_t a = base + (int64_t)k * C;
      const I ca = ld_stream(col + a);
      if (ca >= 0) s0 += ld_stream(val + a) * ld_gather(x + ca);
    }
    if (i < n && len >= 0) axpby_store(y + (reorder ? (int64_t)reorder[i] : i), s0 + s1, alpha, beta, bz);
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
    V s0 = V(0), s1 = V(0);
    const int64_t rb = base + lane;
    int k = 0;
    for (; k + 1 < len; k += 2) {
      const int64_t a = rb + 32 * (int64_t)k, b = a + 32;
      const I ca = ld_stream(col + a), cb = ld_stream(col + b);
      const V va = ld_stream(val + a), vb = ld_stream(val + b);
      if (ca >= 0) s0 += va * ld_gather(x + ca);
      if (cb >= 0) s1 += vb * ld_gather(x + cb);
    }
    if (k < len) {
      const int64_t a = rb + 32 * (int64_t)k;
      const I ca = ld_stream(col + a);
      const V va = ld_stream(val + a);
      if (ca >= 0) s0 += va * ld_gather(x + ca);
    }
    emit(lane, s0 + s1);
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

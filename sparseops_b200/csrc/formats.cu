// Device format conversions and SpMV kernels for the non-CSR formats.
//
// Conversions (replace the host loops of reference include/sparse_conversion.h):
//   SELL-C-sigma  csr_to_sell_c_sigma  344-487: rows of every sigma-slice sorted by
//                 the pair (nnz, row) DESCENDING -- one stable radix sort of
//                 (slice, ~len) keys over rows enumerated from the last row
//                 down, which reproduces std::greater on the pairs bit for bit;
//                 chunk_len = longest row of the chunk rounded up to alignment.
//   SELL-C-R      csr_to_sell_c_R 490-606: the same with one slice.
//   S-ELL         csr_to_sell 265-342: chunks of C consecutive rows, unsorted.
//   ELL           csr_to_ell 194-256: one chunk of all rows, width = longest row.
//   DIA           csr_to_dia 619-774: diagonals numbered by first appearance in
//                 a row-major scan (atomicMin of the entry index per diagonal,
//                 then a sort of the present diagonals by that index).
//   BSR           csr_to_bsr 776-934: block columns of a block row ascending
//                 (sort + unique of block keys); blocks row-major.
//   COO           csr_to_coo 152-176 (row indices expanded per entry).
// SpMV kernels (replace SpOps_<fmt>, src/spmv_*.cpp):
//   padded rows (SELL-C-sigma / SELL-C-R / S-ELL / ELL): one warp per 32
//     stored rows; row-major layout: t lanes per row (t from the warp's
//     longest row), coalesced along the row, padding never read past a row's
//     last entry; col-major layout: one lane per row, consecutive lanes read
//     consecutive slots.  Rows longer than kPadLong slots: block per piece of
//     kPadPiece slots, combined in piece order by the last piece to finish.
//   DIA: one thread per row, diagonal offsets staged in shared memory, every
//     diagonal read coalesced along the rows.
//   BSR: one warp per block row, lanes over the br*bc block elements.
//   COO: sorted by row on the device once, then the CSR kernel.
#include <cub/cub.cuh>

#include <algorithm>
#include <vector>

#include "device_util.cuh"
#include "spops_internal.h"
#include "warp_work.cuh"

namespace spops {

namespace {


template <typename I>
__device__ __forceinline__ int64_t row_length(const I* rp, int64_t r) {
  return (int64_t)rp[r + 1] - (int64_t)rp[r];
}

// ----------------------------------------------------------- SELL sort
template <typename I>
__global__ void sell_keys_kernel(const I* __restrict__ rp, int64_t n, int64_t sigma, int lbits,
                                 uint64_t* __restrict__ keys, I* __restrict__ vals) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int64_t r = n - 1 - i;  // enumerate rows from the last: stable sort keeps larger rows first
  const uint64_t len = (uint64_t)row_length(rp, r);
  const uint64_t lmask = (lbits >= 64) ? ~0ULL : ((1ULL << lbits) - 1);
  keys[i] = ((uint64_t)(r / sigma) << lbits) | (lmask - (len & lmask));
  vals[i] = (I)r;
}

template <typename I>
__global__ void stored_len_kernel(const I* __restrict__ rp, const I* __restrict__ reorder, int64_t n,
                                  int* __restrict__ row_len) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int64_t r = reorder ? (int64_t)reorder[i] : i;
  row_len[i] = (int)row_length(rp, r);
}

// chunk_max[c] = max row_len over the chunk's stored rows (chunk_max zeroed).
__global__ void chunk_max_kernel(const int* __restrict__ row_len, int64_t n, int64_t C, int* __restrict__ cmax) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  const int lane = threadIdx.x & 31;
  const int64_t c = i < n ? i / C : -1;
  const int v = i < n ? row_len[i] : 0;
  const int64_t c0 = __shfl_sync(0xffffffffu, c, 0);
  const int64_t c31 = __shfl_sync(0xffffffffu, c, 31);
  if (c0 == c31 && c0 >= 0) {
    const unsigned m = __reduce_max_sync(0xffffffffu, (unsigned)v);
    if (lane == 0) atomicMax(cmax + c0, (int)m);
  } else if (i < n) {
    atomicMax(cmax + c, v);
  }
}

template <typename I>
__global__ void chunk_len_kernel(const int* __restrict__ cmax, int64_t nchunks, int64_t C, int64_t align,
                                 I* __restrict__ chunk_len, int64_t* __restrict__ elems) {
  const int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (c >= nchunks) return;
  const int64_t L = ((int64_t)cmax[c] + align - 1) / align * align;
  chunk_len[c] = (I)L;
  elems[c] = L * C;
}

// Copy every row's entries into its padded slots (one warp per stored row).
template <typename I, typename V, bool kColMajor>
__global__ void pad_fill_kernel(const I* __restrict__ rp, const I* __restrict__ ci, const V* __restrict__ v,
                                const I* __restrict__ reorder, int64_t n, int64_t C,
                                const I* __restrict__ chunk_len, const int64_t* __restrict__ chunk_off,
                                I* __restrict__ col, V* __restrict__ val) {
  const int64_t i = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (i >= n) return;
  const int64_t r = reorder ? (int64_t)reorder[i] : i;
  const int64_t s = rp[r], e = rp[r + 1];
  const int64_t c = i / C;
  const int64_t base = chunk_off[c] + (kColMajor ? (i - c * C) : (i - c * C) * (int64_t)chunk_len[c]);
  for (int64_t k = lane; k < e - s; k += 32) {
    const int64_t dst = base + (kColMajor ? k * C : k);
    col[dst] = ci[s + k];
    val[dst] = v[s + k];
  }
}

// Row lengths of an uploaded padded matrix: slots up to the last real entry.
template <typename I, bool kColMajor>
__global__ void pad_rowlen_kernel(const I* __restrict__ col, int64_t n, int64_t C, const I* __restrict__ chunk_len,
                                  const int64_t* __restrict__ chunk_off, int* __restrict__ row_len) {
  const int64_t i = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (i >= n) return;
  const int64_t c = i / C;
  const int64_t L = chunk_len[c];
  const int64_t base = chunk_off[c] + (kColMajor ? (i - c * C) : (i - c * C) * L);
  int last = 0;
  for (int64_t k = lane; k < L; k += 32)
    if (col[base + (kColMajor ? k * C : k)] >= 0) last = (int)k + 1;
  last = (int)__reduce_max_sync(0xffffffffu, (unsigned)last);
  if (lane == 0) row_len[i] = last;
}

__global__ void pad_npieces_kernel(const int* __restrict__ row_len, int64_t n, int64_t* __restrict__ np) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int L = row_len[i];
  np[i] = L > kPadLong ? (L + kPadPiece - 1) / kPadPiece : 0;
}

__global__ void pad_pieces_kernel(const int64_t* __restrict__ np, const int64_t* __restrict__ off, int64_t n,
                                  PadPiece* __restrict__ pieces) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int64_t k = np[i];
  for (int64_t q = 0; q < k; ++q) pieces[off[i] + q] = PadPiece{i, (int32_t)q, (int32_t)k};
}

__global__ void minmax_kernel(const int* __restrict__ a, int64_t n, int* __restrict__ mm) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  int mx = 0, mn = INT32_MAX;
  if (i < n) mx = mn = a[i];
  mx = (int)__reduce_max_sync(0xffffffffu, (unsigned)mx);
  mn = (int)__reduce_min_sync(0xffffffffu, (unsigned)mn);
  if ((threadIdx.x & 31) == 0) {
    atomicMax(mm, mx);
    atomicMin(mm + 1, mn);
  }
}

// -------------------------------------------------------- padded SpMV
template <typename I, typename V, bool kColMajor>
__global__ void __launch_bounds__(256) padded_kernel(
    const I* __restrict__ col, const V* __restrict__ val, const I* __restrict__ chunk_len,
    const int64_t* __restrict__ chunk_off, const int* __restrict__ row_len, const I* __restrict__ reorder,
    int64_t n, int64_t C, const V* __restrict__ x, V* __restrict__ y, V alpha, V beta, bool bz,
    int64_t main_warps, int64_t npieces, const PadPiece* __restrict__ pieces, V* __restrict__ partial,
    int* __restrict__ counter) {
  const int lane = threadIdx.x & 31;
  const int64_t w = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  if (w < main_warps)
    padded_rows32<I, V, kColMajor>(w * 32, col, val, chunk_len, chunk_off, row_len, reorder, n, C, x, y, alpha, beta,
                                   bz, lane);
  else if (w - main_warps < npieces)
    padded_piece<I, V, kColMajor>(w - main_warps, pieces[w - main_warps], col, val, chunk_len, chunk_off, row_len,
                                  reorder, C, x, y, alpha, beta, bz, partial, counter, lane);
}

// Column-major SELL with C = 32: one warp per step window of a chunk
// (padded_window32); windows of one chunk combine their per-row partial sums
// in window order on the last one to finish.  Long rows go to pieces.
template <typename I, typename V>
__global__ void __launch_bounds__(256) padded_win_kernel(
    const I* __restrict__ col, const V* __restrict__ val, const int64_t* __restrict__ chunk_off,
    const int* __restrict__ row_len, const I* __restrict__ reorder, int64_t n, const V* __restrict__ x,
    V* __restrict__ y, V alpha, V beta, bool bz, const PadWin* __restrict__ wins, int64_t nwin,
    V* __restrict__ wpartial, int* __restrict__ wcounter, int64_t npieces, const PadPiece* __restrict__ pieces,
    V* __restrict__ partial, int* __restrict__ counter, const int* __restrict__ head, const I* __restrict__ tcol,
    const V* __restrict__ tval) {
  const int lane = threadIdx.x & 31;
  const int64_t w = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  if (w >= nwin) {
    if (w - nwin < npieces)
      padded_piece<I, V, true>(w - nwin, pieces[w - nwin], col, val, nullptr, chunk_off, row_len, reorder, 32, x, y,
                               alpha, beta, bz, partial, counter, lane);
    return;
  }
  const PadWin W = wins[w];
  const int64_t i0 = W.chunk * 32, i = i0 + lane;
  int len = 0;
  if (i < n) {
    len = row_len[i];
    if (len > kPadLong || len < 0) len = 0;  // long rows: pieces
    const int h = head[W.chunk];
    if (len > h) len = h;  // the slots beyond the head are tail entries
  }
  auto store = [&](int r, V s) {
    const int64_t row = i0 + r;
    if (row < n && row_len[row] <= kPadLong)
      axpby_store(y + (reorder ? (int64_t)reorder[row] : row), s, alpha, beta, bz);
  };
  if (W.nw == 1) {
    padded_window32<I, V>(chunk_off[W.chunk], len, 0, col, val, x, lane, store);
    return;
  }
  V* part = wpartial + (W.first + W.widx) * 32;
  if (W.tail >= 0) {  // one row's tail entries, read contiguously, 4 per lane per step
    V s0 = V(0), s1 = V(0), s2 = V(0), s3 = V(0);
    const I* tc = tcol + W.tail;
    const V* tv = tval + W.tail;
    int e = lane;
    for (; e + 96 < W.tlen; e += 128) {
      const I c0 = ld_stream(tc + e), c1 = ld_stream(tc + e + 32), c2 = ld_stream(tc + e + 64),
              c3 = ld_stream(tc + e + 96);
      const V v0 = ld_stream(tv + e), v1 = ld_stream(tv + e + 32), v2 = ld_stream(tv + e + 64),
              v3 = ld_stream(tv + e + 96);
      s0 += v0 * ld_gather(x + c0);
      s1 += v1 * ld_gather(x + c1);
      s2 += v2 * ld_gather(x + c2);
      s3 += v3 * ld_gather(x + c3);
    }
    for (; e < W.tlen; e += 32) s0 += ld_stream(tv + e) * ld_gather(x + ld_stream(tc + e));
    const V s = __shfl_sync(0xffffffffu, warp_sum((s0 + s1) + (s2 + s3)), 0);  // the sum is in lane 0
    part[lane] = lane == W.tlane ? s : V(0);
  } else {
    padded_window32<I, V>(chunk_off[W.chunk], len, W.widx * kPadWindow, col, val, x, lane,
                          [&](int r, V s) { part[r] = s; });
  }
  __syncwarp();
  int last = 0;
  if (lane == 0) {
    __threadfence();
    last = atomicAdd(wcounter + W.chunk, 1) == W.nw - 1;
  }
  last = __shfl_sync(0xffffffffu, last, 0);
  if (last) {
    __threadfence();
    V tot = V(0);
    for (int q = 0; q < W.nw; ++q) tot += ld_cg(wpartial + (W.first + q) * 32 + lane);
    store(lane, tot);
    __syncwarp();
    if (lane == 0) wcounter[W.chunk] = 0;
  }
}

// Entries of one tail window (a longer tail is cut into several).
constexpr int kTailWin = 1024;

// Per 32-row chunk (a warp): the head width h (the fourth-longest row's
// length, rows longer than kPadLong left to pieces), the tail rows (longer
// than h, at most three), their entries, and the chunk's windows: head
// windows of kPadWindow slots (at least one) and tail windows of kTailWin
// entries.
__global__ void pad_head_kernel(const int* __restrict__ row_len, int64_t n, int64_t nchunks, bool tails,
                                int* __restrict__ head, int64_t* __restrict__ ntr, int64_t* __restrict__ nte,
                                int64_t* __restrict__ nw, uint32_t* __restrict__ order_key) {
  const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  const int64_t c = t >> 5;
  const int lane = threadIdx.x & 31;
  if (c >= nchunks) return;
  const int64_t i = c * 32 + lane;
  int len = i < n ? row_len[i] : 0;
  if (len > kPadLong || len < 0) len = 0;
  unsigned key = (unsigned)len;  // descending across the lanes
#pragma unroll
  for (int kk = 2; kk <= 32; kk <<= 1) {
#pragma unroll
    for (int jj = kk >> 1; jj > 0; jj >>= 1) {
      const unsigned other = __shfl_xor_sync(0xffffffffu, key, jj);
      const bool first_half = (lane & kk) == 0, lower = (lane & jj) == 0;
      key = (lower == first_half) ? (key > other ? key : other) : (key < other ? key : other);
    }
  }
  const int h = (int)__shfl_sync(0xffffffffu, key, tails ? 3 : 0);
  const int tl = len > h ? len - h : 0;
  const unsigned rows = __reduce_add_sync(0xffffffffu, tl > 0 ? 1u : 0u);
  const unsigned ents = __reduce_add_sync(0xffffffffu, (unsigned)tl);
  const unsigned twin = __reduce_add_sync(0xffffffffu, (unsigned)((tl + kTailWin - 1) / kTailWin));
  if (lane == 0) {
    head[c] = h;
    order_key[c] = ~key;  // key is the longest row here: longest chunks first
    ntr[c] = rows;
    nte[c] = ents;
    nw[c] = (h > kPadWindow ? ((int64_t)h + kPadWindow - 1) / kPadWindow : 1) + twin;
  }
}

__global__ void iota_i32_kernel(int32_t* __restrict__ a, int64_t m) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i < m) a[i] = (int32_t)i;
}

// Window offsets in the order the chunks are taken (order[i]: the i-th
// chunk): the counts gathered into that order, scanned, and scattered back.
__global__ void pad_gather_nw_kernel(const int32_t* __restrict__ order, const int64_t* __restrict__ nw, int64_t nch,
                                     int64_t* __restrict__ nw_sorted) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i < nch) nw_sorted[i] = nw[order[i]];
  if (i == nch) nw_sorted[i] = 0;
}

__global__ void pad_scatter_woff_kernel(const int32_t* __restrict__ order, const int64_t* __restrict__ woff_sorted,
                                        int64_t nch, int64_t* __restrict__ woff) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i < nch) woff[order[i]] = woff_sorted[i];
  if (i == nch) woff[nch] = woff_sorted[nch];
}

// The chunk's window list and tail records (offsets from exclusive scans of
// pad_head_kernel's counts).
__global__ void pad_win_fill_kernel(const int* __restrict__ row_len, int64_t n, int64_t nchunks,
                                    const int* __restrict__ head, const int64_t* __restrict__ woff,
                                    const int64_t* __restrict__ nw, const int64_t* __restrict__ troff,
                                    const int64_t* __restrict__ teoff, PadWin* __restrict__ wins,
                                    PadTail* __restrict__ tails) {
  const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  const int64_t c = t >> 5;
  const int lane = threadIdx.x & 31;
  if (c >= nchunks) return;
  const int64_t i = c * 32 + lane;
  int len = i < n ? row_len[i] : 0;
  if (len > kPadLong || len < 0) len = 0;
  const int h = head[c];
  const int tl = len > h ? len - h : 0;
  const int tw = (tl + kTailWin - 1) / kTailWin;
  // exclusive prefixes over the lanes: tail rows, entries, tail windows
  int pr = tl > 0 ? 1 : 0, pe = tl, pw = tw;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int ur = __shfl_up_sync(0xffffffffu, pr, o), ue = __shfl_up_sync(0xffffffffu, pe, o),
              uw = __shfl_up_sync(0xffffffffu, pw, o);
    if (lane >= o) {
      pr += ur;
      pe += ue;
      pw += uw;
    }
  }
  pr -= tl > 0 ? 1 : 0;
  pe -= tl;
  pw -= tw;
  const int nh = h > kPadWindow ? (h + kPadWindow - 1) / kPadWindow : 1;
  const int64_t first = woff[c];
  const int32_t total = (int32_t)nw[c];
  for (int q = lane; q < nh; q += 32) wins[first + q] = PadWin{c, first, q, total, -1, 0, 0};
  if (tl > 0) {
    const int64_t start = teoff[c] + pe;
    tails[troff[c] + pr] = PadTail{i, start, h, tl};
    for (int m = 0; m < tw; ++m) {
      const int32_t len_m = tl - m * kTailWin < kTailWin ? tl - m * kTailWin : kTailWin;
      wins[first + nh + pw + m] = PadWin{c, first, nh + pw + m, total, start + (int64_t)m * kTailWin, len_m, lane};
    }
  }
}

// Copy every tail's slots from the column-major chunks (warp per tail).
template <typename I, typename V>
__global__ void pad_tail_copy_kernel(const PadTail* __restrict__ tails, int64_t ntails,
                                     const int64_t* __restrict__ chunk_off, const I* __restrict__ col,
                                     const V* __restrict__ val, I* __restrict__ tcol, V* __restrict__ tval) {
  const int64_t t = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (t >= ntails) return;
  const PadTail T = tails[t];
  const int64_t c = T.row >> 5;
  const int64_t base = chunk_off[c] + (T.row - c * 32);
  for (int e = lane; e < T.len; e += 32) {
    const int64_t src = base + 32 * (int64_t)(T.from + e);
    tcol[T.start + e] = col[src];
    tval[T.start + e] = val[src];
  }
}

// ------------------------------------------------------------------ DIA
template <typename I>
__global__ void dia_first_kernel(const I* __restrict__ rp, const I* __restrict__ ci, int64_t n,
                                 unsigned long long* __restrict__ first) {
  const int64_t r = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (r >= n) return;
  for (int64_t k = (int64_t)rp[r] + lane; k < (int64_t)rp[r + 1]; k += 32) {
    const int64_t d = n - r + (int64_t)ci[k];
    atomicMin(first + d, (unsigned long long)k);
  }
}

__global__ void dia_select_kernel(const unsigned long long* __restrict__ first, int64_t nd_all,
                                  unsigned long long* __restrict__ keys, int64_t* __restrict__ ids,
                                  int64_t* __restrict__ count) {
  const int64_t d = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (d >= nd_all) return;
  if (first[d] != ~0ULL) {
    const int64_t slot = (int64_t)atomicAdd((unsigned long long*)count, 1ULL);
    keys[slot] = first[d];
    ids[slot] = d;
  }
}

__global__ void dia_index_kernel(const int64_t* __restrict__ ids_sorted, int64_t ndiag, int64_t n,
                                 int64_t* __restrict__ offsets, int* __restrict__ diag_index) {
  const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (t >= ndiag) return;
  const int64_t d = ids_sorted[t];
  offsets[t] = d - n;
  diag_index[d] = (int)t;
}

template <typename I, typename V>
__global__ void dia_fill_kernel(const I* __restrict__ rp, const I* __restrict__ ci, const V* __restrict__ v,
                                int64_t n, const int* __restrict__ diag_index, int64_t stride,
                                V* __restrict__ data) {
  const int64_t r = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (r >= n) return;
  for (int64_t k = (int64_t)rp[r] + lane; k < (int64_t)rp[r + 1]; k += 32) {
    const int64_t d = n - r + (int64_t)ci[k];
    data[(int64_t)diag_index[d] * stride + r] = v[k];
  }
}

template <typename V>
__global__ void __launch_bounds__(256) dia_kernel(const int64_t* __restrict__ offsets, const V* __restrict__ data,
                                                  int64_t ndiag, int64_t stride, int64_t n, int64_t ncols,
                                                  const V* __restrict__ x, V* __restrict__ y, V alpha, V beta,
                                                  bool bz) {
  __shared__ int64_t soff[1024];
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  V s0 = V(0), s1 = V(0);
  for (int64_t d0 = 0; d0 < ndiag; d0 += 1024) {
    const int nd = (int)((ndiag - d0) < 1024 ? (ndiag - d0) : 1024);
    __syncthreads();
    for (int t = threadIdx.x; t < nd; t += blockDim.x) soff[t] = offsets[d0 + t];
    __syncthreads();
    if (i < n) {
      for (int d = 0; d < nd; ++d) {
        const int64_t j = i + soff[d];
        if (j >= 0 && j < ncols) {
          const V p = ld_stream(data + (d0 + d) * stride + i) * ld_gather(x + j);
          if (d & 1) s1 += p; else s0 += p;
        }
      }
    }
  }
  if (i < n) axpby_store(y + i, s0 + s1, alpha, beta, bz);
}

// DIA with x staged in shared memory: the block's 256 rows reach x only in
// [i0 + lo, i0 + 255 + hi], so that window (win = 256 + hi - lo entries) is
// read once, coalesced, and every diagonal's gathers come from shared memory.
// Used when the window fits (dia_spmv_t); the products are summed in the same
// order as dia_kernel, so both give the same bits.
constexpr int kDiaStageMaxDiags = 1024;
constexpr int64_t kDiaStageMaxWin = 4096;

template <typename V>
__global__ void __launch_bounds__(256) dia_staged_kernel(const int64_t* __restrict__ offsets,
                                                         const V* __restrict__ data, int64_t ndiag, int64_t stride,
                                                         int64_t n, int64_t ncols, const V* __restrict__ x,
                                                         V* __restrict__ y, V alpha, V beta, bool bz, int64_t lo,
                                                         int64_t win) {
  extern __shared__ __align__(16) unsigned char dia_sm[];
  V* xs = reinterpret_cast<V*>(dia_sm);
  __shared__ int64_t soff[kDiaStageMaxDiags];
  const int64_t i0 = blockIdx.x * 256LL;
  const int64_t w0 = i0 + lo;  // x index held by xs[0]
  for (int t = threadIdx.x; t < ndiag; t += blockDim.x) soff[t] = offsets[t];
  for (int64_t t = threadIdx.x; t < win; t += blockDim.x) {
    const int64_t j = w0 + t;
    xs[t] = (j >= 0 && j < ncols) ? ld_gather(x + j) : V(0);
  }
  __syncthreads();
  const int64_t i = i0 + threadIdx.x;
  if (i >= n) return;
  V s0 = V(0), s1 = V(0);
  for (int d = 0; d < (int)ndiag; ++d) {
    const int64_t j = i + soff[d];
    if (j >= 0 && j < ncols) {
      const V p = ld_stream(data + d * stride + i) * xs[j - w0];
      if (d & 1) s1 += p; else s0 += p;
    }
  }
  axpby_store(y + i, s0 + s1, alpha, beta, bz);
}

// ------------------------------------------------------------------ BSR
template <typename I>
__global__ void bsr_keys_kernel(const I* __restrict__ rp, const I* __restrict__ ci, int64_t n, int64_t br,
                                int64_t bc, int64_t nb, int64_t* __restrict__ keys) {
  const int64_t r = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (r >= n) return;
  for (int64_t k = (int64_t)rp[r] + lane; k < (int64_t)rp[r + 1]; k += 32)
    keys[k] = (r / br) * nb + (int64_t)ci[k] / bc;
}

template <typename I>
__global__ void bsr_struct_kernel(const int64_t* __restrict__ ukeys, int64_t nnzb, int64_t nb,
                                  I* __restrict__ bcol, unsigned long long* __restrict__ cnt) {
  const int64_t b = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (b >= nnzb) return;
  bcol[b] = (I)(ukeys[b] % nb);
  atomicAdd(cnt + ukeys[b] / nb, 1ULL);
}

template <typename I>
__global__ void bsr_rowptr_kernel(const int64_t* __restrict__ scan, int64_t mb, I* __restrict__ row_ptr) {
  const int64_t b = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (b > mb) return;
  row_ptr[b] = (I)scan[b];
}

template <typename I, typename V>
__global__ void bsr_fill_kernel(const I* __restrict__ rp, const I* __restrict__ ci, const V* __restrict__ v,
                                int64_t n, int64_t br, int64_t bc, int64_t nb, const int64_t* __restrict__ ukeys,
                                int64_t nnzb, V* __restrict__ data) {
  const int64_t r = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (r >= n) return;
  for (int64_t k = (int64_t)rp[r] + lane; k < (int64_t)rp[r + 1]; k += 32) {
    const int64_t key = (r / br) * nb + (int64_t)ci[k] / bc;
    int64_t lo = 0, hi = nnzb;  // lower_bound in the sorted unique keys
    while (lo < hi) {
      const int64_t mid = (lo + hi) >> 1;
      if (ukeys[mid] < key) lo = mid + 1; else hi = mid;
    }
    data[lo * br * bc + (r % br) * bc + (int64_t)ci[k] % bc] = v[k];
  }
}

template <typename I, typename V>
__global__ void __launch_bounds__(256) bsr_kernel(const I* __restrict__ row_ptr, const I* __restrict__ bcol,
                                                  const V* __restrict__ data, int64_t mb, int br, int bc, int64_t n,
                                                  int64_t ncols, const V* __restrict__ x, V* __restrict__ y, V alpha,
                                                  V beta, bool bz) {
  extern __shared__ __align__(16) unsigned char bsr_smem[];
  V* acc_all = reinterpret_cast<V*>(bsr_smem);
  const int B = br * bc;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  V* acc = acc_all + (int64_t)w * B;
  const int64_t brow = (int64_t)blockIdx.x * 8 + w;
  if (brow >= mb) return;  // whole warp; the kernel has no block barrier
  for (int e = lane; e < B; e += 32) acc[e] = V(0);
  const int64_t b0 = row_ptr[brow], b1 = row_ptr[brow + 1];
  for (int64_t b = b0; b < b1; ++b) {
    const int64_t cbase = (int64_t)bcol[b] * bc;
    const V* blk = data + b * B;
    for (int e = lane; e < B; e += 32) {
      const int64_t cx = cbase + (e % bc);
      if (cx < ncols) acc[e] += ld_stream(blk + e) * ld_gather(x + cx);
    }
  }
  __syncwarp();
  for (int r = lane; r < br; r += 32) {
    const int64_t row = brow * br + r;
    if (row < n) {
      V s = V(0);
      for (int c = 0; c < bc; ++c) s += acc[r * bc + c];
      axpby_store(y + row, s, alpha, beta, bz);
    }
  }
}

// ------------------------------------------------------------------ COO
template <typename I>
__global__ void coo_check_kernel(const I* __restrict__ row, const I* __restrict__ col, int64_t nnz, int64_t n,
                                 int64_t ncols, int* __restrict__ flags, unsigned long long* __restrict__ cnt) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < nnz; k += stride) {
    const int64_t r = row[k], c = col[k];
    if (r < 0 || r >= n || c < 0 || c >= ncols) {
      atomicOr(flags, 2);
      continue;
    }
    if (k + 1 < nnz && (int64_t)row[k + 1] < r) atomicOr(flags, 1);  // not sorted by row
    atomicAdd(cnt + r, 1ULL);
  }
}

template <typename I, typename V>
__global__ void gather_kernel(const int64_t* __restrict__ perm, const I* __restrict__ col, const V* __restrict__ val,
                              int64_t nnz, I* __restrict__ col_out, V* __restrict__ val_out) {
  const int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (k >= nnz) return;
  const int64_t p = perm[k];
  col_out[k] = col[p];
  val_out[k] = val[p];
}

template <typename I>
__global__ void csr_expand_rows_kernel(const I* __restrict__ rp, int64_t n, I* __restrict__ row) {
  const int64_t r = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (r >= n) return;
  for (int64_t k = (int64_t)rp[r] + lane; k < (int64_t)rp[r + 1]; k += 32) row[k] = (I)r;
}

template <typename I>
__global__ void to_index_kernel(const unsigned long long* __restrict__ in, int64_t m, I* __restrict__ out) {
  const int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (k < m) out[k] = (I)in[k];
}

__global__ void iota_kernel(int64_t* __restrict__ a, int64_t m) {
  const int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (k < m) a[k] = k;
}

template <typename I>
__global__ void validate_cols_kernel(const I* __restrict__ col, int64_t m, int64_t ncols, bool allow_pad,
                                     int* __restrict__ bad) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < m; k += stride) {
    const int64_t c = col[k];
    if (c >= ncols || (c < 0 && !(allow_pad && c == -1))) atomicOr(bad, 1);
  }
}

inline unsigned grid_for(int64_t work, int threads = 256) {
  int64_t g = (work + threads - 1) / threads;
  return (unsigned)(g < 1 ? 1 : g);
}

inline int bits_for(uint64_t v) {
  int b = 1;
  while (b < 64 && (v >> b) != 0) ++b;
  return b;
}

// Host scratch helper: carve 256-byte aligned pieces out of ctx->scratch.
struct Carve {
  char* base;
  size_t off = 0;
  explicit Carve(char* b) : base(b) {}
  template <typename T> T* take(size_t n) {
    T* p = reinterpret_cast<T*>(base + off);
    off += (n * sizeof(T) + 255) & ~(size_t)255;
    return p;
  }
};

template <typename T>
spops_status_t download(Context* ctx, T* host, const void* dev, size_t n) {
  if (n == 0) return SPOPS_OK;
  SPOPS_CUDA(cudaMemcpyAsync(host, dev, n * sizeof(T), cudaMemcpyDeviceToHost, ctx->stream));
  SPOPS_CUDA(cudaStreamSynchronize(ctx->stream));
  return SPOPS_OK;
}

// ----------------------------------------------------- padded conversion
template <typename I, typename V>
spops_status_t to_padded(Context* ctx, Matrix* A, spops_format_t fmt, const spops_format_params_t& p, Matrix* M) {
  const int64_t n = A->rows;
  cudaStream_t st = ctx->stream;
  const I* rp = A->row.as<I>();
  PaddedData& P = M->pad;
  int64_t C, sigma;
  bool sort;
  const int64_t align_default = 32 / (int64_t)sizeof(V);  // reference SIMD_WIDTH(256)/8/sizeof(V)
  int64_t align = p.alignment > 0 ? p.alignment : align_default;
  if (fmt == SPOPS_FMT_ELL) {
    C = n > 0 ? n : 1;
    sigma = 0;
    sort = false;
    align = 1;  // the reference pads ELL rows to the longest row exactly
  } else {
    C = p.chunk > 0 ? p.chunk : 4;
    if (fmt == SPOPS_FMT_SELL_C_SIGMA) {
      sigma = p.sigma > 0 ? p.sigma : 16384;
      if (sigma % C) return fail(SPOPS_ERR_INVALID, "SELL-C-sigma: sigma (%lld) must be a multiple of C (%lld)",
                                 (long long)sigma, (long long)C);
      sort = true;
    } else if (fmt == SPOPS_FMT_SELL_C_R) {
      sigma = n > 0 ? n : 1;
      sort = true;
    } else {
      sigma = 0;
      sort = false;
    }
  }
  M->layout = (p.layout == SPOPS_COL_MAJOR) ? SPOPS_COL_MAJOR : SPOPS_ROW_MAJOR;
  P.C = C;
  P.sigma = sigma;
  P.align = align;
  P.sorted = sort;
  P.nchunks = n > 0 ? (n + C - 1) / C : 0;

  // scratch: keys in/out (u64), vals in (I), chunk max (int), elems/off (int64), cub temp
  size_t cub_sort = 0, cub_scan = 0;
  {
    uint64_t* k = nullptr;
    I* v = nullptr;
    int64_t* e = nullptr;
    SPOPS_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, cub_sort, k, k, v, v, (int64_t)(n > 0 ? n : 1), 0, 64, st));
    SPOPS_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, cub_scan, e, e, (int64_t)(P.nchunks + 1), st));
  }
  const size_t nn = (size_t)(n > 0 ? n : 1), nc = (size_t)P.nchunks + 1;
  SPOPS_TRY(ctx->scratch_reserve(2 * nn * 8 + nn * sizeof(I) + nc * 4 + 2 * nc * 8 + std::max(cub_sort, cub_scan) +
                                 8 * 256));
  Carve cv(ctx->scratch.as<char>());
  uint64_t* keys_in = cv.take<uint64_t>(nn);
  uint64_t* keys_out = cv.take<uint64_t>(nn);
  I* vals_in = cv.take<I>(nn);
  int* cmax = cv.take<int>(nc);
  int64_t* elems = cv.take<int64_t>(nc);
  void* cub_tmp = cv.take<char>(std::max(cub_sort, cub_scan));

  SPOPS_TRY(P.row_len.alloc(nn * sizeof(int)));
  if (sort) {
    SPOPS_TRY(P.reorder.alloc(nn * sizeof(I)));
    if (n > 0) {
      // key bits: slice id above, (max_len - len) below
      int mm_h[2];
      int64_t maxlen = 0;
      {
        int* mm = reinterpret_cast<int*>(elems);  // reuse as temp
        int init[2] = {0, INT32_MAX};
        SPOPS_CUDA(cudaMemcpyAsync(mm, init, sizeof(init), cudaMemcpyHostToDevice, st));
        stored_len_kernel<I><<<grid_for(n), 256, 0, st>>>(rp, nullptr, n, P.row_len.as<int>());
        minmax_kernel<<<grid_for(n), 256, 0, st>>>(P.row_len.as<int>(), n, mm);
        SPOPS_LAUNCH_CHECK();
        SPOPS_TRY(download(ctx, mm_h, mm, 2));
        maxlen = mm_h[0];
      }
      const int lbits = bits_for((uint64_t)maxlen);
      const int sbits = bits_for((uint64_t)((n - 1) / sigma));
      sell_keys_kernel<I><<<grid_for(n), 256, 0, st>>>(rp, n, sigma, lbits, keys_in, vals_in);
      SPOPS_LAUNCH_CHECK();
      SPOPS_CUDA(cub::DeviceRadixSort::SortPairs(cub_tmp, cub_sort, keys_in, keys_out, vals_in, P.reorder.as<I>(), n,
                                                 0, std::min(64, lbits + sbits), st));
    }
  }
  if (n > 0) {
    stored_len_kernel<I><<<grid_for(n), 256, 0, st>>>(rp, sort ? P.reorder.as<I>() : nullptr, n,
                                                      P.row_len.as<int>());
    SPOPS_CUDA(cudaMemsetAsync(cmax, 0, nc * sizeof(int), st));
    chunk_max_kernel<<<grid_for(n), 256, 0, st>>>(P.row_len.as<int>(), n, C, cmax);
    SPOPS_LAUNCH_CHECK();
  }
  SPOPS_TRY(P.chunk_len.alloc((size_t)(P.nchunks > 0 ? P.nchunks : 1) * sizeof(I)));
  SPOPS_TRY(P.chunk_off.alloc(nc * sizeof(int64_t)));
  SPOPS_CUDA(cudaMemsetAsync(elems, 0, nc * sizeof(int64_t), st));
  if (P.nchunks > 0) {
    chunk_len_kernel<I><<<grid_for(P.nchunks), 256, 0, st>>>(cmax, P.nchunks, C, align, P.chunk_len.as<I>(), elems);
    SPOPS_LAUNCH_CHECK();
  }
  SPOPS_CUDA(cub::DeviceScan::ExclusiveSum(cub_tmp, cub_scan, elems, P.chunk_off.as<int64_t>(), (int64_t)nc, st));
  int64_t stored = 0;
  SPOPS_TRY(download(ctx, &stored, P.chunk_off.as<int64_t>() + P.nchunks, 1));
  P.stored = stored;
  // refuse storage that cannot fit (the reference's ELL of a power-law matrix
  // needs hundreds of GB): keep 10% of free memory
  size_t free_b = 0, total_b = 0;
  SPOPS_CUDA(cudaMemGetInfo(&free_b, &total_b));
  const double need = (double)stored * (double)(sizeof(I) + sizeof(V));
  if (need > 0.9 * (double)free_b)
    return fail(SPOPS_ERR_TOO_LARGE, "%s needs %.1f GB of padded storage (%lld slots for %lld entries); %.1f GB free",
                fmt == SPOPS_FMT_ELL ? "ELL" : "SELL", need / 1e9, (long long)stored, (long long)A->nnz,
                free_b / 1e9);
  SPOPS_TRY(M->col.alloc((size_t)stored * sizeof(I)));
  SPOPS_TRY(M->val.alloc((size_t)stored * sizeof(V)));
  SPOPS_CUDA(cudaMemsetAsync(M->col.p, 0xff, M->col.bytes, st));
  SPOPS_CUDA(cudaMemsetAsync(M->val.p, 0, M->val.bytes, st));
  if (n > 0) {
    const unsigned g = grid_for(n * 32);
    if (M->layout == SPOPS_COL_MAJOR)
      pad_fill_kernel<I, V, true><<<g, 256, 0, st>>>(rp, A->col.as<I>(), A->val.as<V>(),
                                                     sort ? P.reorder.as<I>() : nullptr, n, C, P.chunk_len.as<I>(),
                                                     P.chunk_off.as<int64_t>(), M->col.as<I>(), M->val.as<V>());
    else
      pad_fill_kernel<I, V, false><<<g, 256, 0, st>>>(rp, A->col.as<I>(), A->val.as<V>(),
                                                      sort ? P.reorder.as<I>() : nullptr, n, C, P.chunk_len.as<I>(),
                                                      P.chunk_off.as<int64_t>(), M->col.as<I>(), M->val.as<V>());
    SPOPS_LAUNCH_CHECK();
  }
  return padded_finish(ctx, M);
}

template <typename I, typename V>
spops_status_t padded_finish_t(Context* ctx, Matrix* M) {
  PaddedData& P = M->pad;
  const int64_t n = M->rows;
  cudaStream_t st = ctx->stream;
  const size_t nn = (size_t)(n > 0 ? n : 1);
  if (!P.row_len.p) {
    SPOPS_TRY(P.row_len.alloc(nn * sizeof(int)));
    if (n > 0) {
      if (M->layout == SPOPS_COL_MAJOR)
        pad_rowlen_kernel<I, true><<<grid_for(n * 32), 256, 0, st>>>(M->col.as<I>(), n, P.C, P.chunk_len.as<I>(),
                                                                   P.chunk_off.as<int64_t>(), P.row_len.as<int>());
      else
        pad_rowlen_kernel<I, false><<<grid_for(n * 32), 256, 0, st>>>(M->col.as<I>(), n, P.C, P.chunk_len.as<I>(),
                                                                    P.chunk_off.as<int64_t>(), P.row_len.as<int>());
      SPOPS_LAUNCH_CHECK();
    }
  }
  size_t cub_scan = 0;
  int64_t* e = nullptr;
  SPOPS_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, cub_scan, e, e, (int64_t)nn, st));
  SPOPS_TRY(ctx->scratch_reserve(2 * nn * 8 + cub_scan + 3 * 256 + 8));
  Carve cv(ctx->scratch.as<char>());
  int64_t* np = cv.take<int64_t>(nn);
  int64_t* off = cv.take<int64_t>(nn);
  int* mm = cv.take<int>(2);
  void* cub_tmp = cv.take<char>(cub_scan);
  int64_t npieces = 0;
  int mm_h[2] = {0, 0};
  if (n > 0) {
    int init[2] = {0, INT32_MAX};
    SPOPS_CUDA(cudaMemcpyAsync(mm, init, sizeof(init), cudaMemcpyHostToDevice, st));
    minmax_kernel<<<grid_for(n), 256, 0, st>>>(P.row_len.as<int>(), n, mm);
    pad_npieces_kernel<<<grid_for(n), 256, 0, st>>>(P.row_len.as<int>(), n, np);
    SPOPS_LAUNCH_CHECK();
    SPOPS_CUDA(cub::DeviceScan::ExclusiveSum(cub_tmp, cub_scan, np, off, n, st));
    int64_t h[2];
    SPOPS_TRY(download(ctx, &h[0], off + n - 1, 1));
    SPOPS_TRY(download(ctx, &h[1], np + n - 1, 1));
    npieces = h[0] + h[1];
    SPOPS_TRY(download(ctx, mm_h, mm, 2));
  }
  P.max_row = mm_h[0];
  P.min_row = n > 0 ? mm_h[1] : 0;
  P.npieces = npieces;
  const size_t npc = (size_t)(npieces > 0 ? npieces : 1);
  SPOPS_TRY(P.piece.alloc(npc * sizeof(PadPiece)));
  SPOPS_TRY(P.partial.alloc(npc * sizeof(double)));
  SPOPS_TRY(P.counter.alloc(npc * sizeof(int)));
  SPOPS_CUDA(cudaMemsetAsync(P.counter.p, 0, P.counter.bytes, st));
  if (npieces > 0) {
    pad_pieces_kernel<<<grid_for(n), 256, 0, st>>>(np, off, n, P.piece.as<PadPiece>());
    SPOPS_LAUNCH_CHECK();
  }
  SPOPS_CUDA(cudaStreamSynchronize(st));
  if (P.C == 32 && M->layout == SPOPS_COL_MAJOR && n > 0) {
    // heads, tails and windows of the 32-row chunks
    const int64_t nch = (n + 31) / 32;
    PoolBuf cnt(ctx), offs(ctx), tmp(ctx);
    SPOPS_TRY(cnt.alloc((size_t)(nch + 1) * 3 * 8));
    SPOPS_TRY(offs.alloc((size_t)(nch + 1) * 3 * 8));
    int64_t* ntr = cnt.as<int64_t>();
    int64_t* nte = ntr + (nch + 1);
    int64_t* nwc = nte + (nch + 1);
    int64_t* troff = offs.as<int64_t>();
    int64_t* teoff = troff + (nch + 1);
    int64_t* woff = teoff + (nch + 1);
    SPOPS_CUDA(cudaMemsetAsync(cnt.p, 0, cnt.bytes, st));
    SPOPS_TRY(P.head.alloc((size_t)nch * 4));
    PoolBuf okey(ctx), okey_s(ctx), ord_in(ctx), ord(ctx), nws(ctx), woffs(ctx);
    SPOPS_TRY(okey.alloc((size_t)nch * 4));
    pad_head_kernel<<<grid_for(nch * 32), 256, 0, st>>>(P.row_len.as<int>(), n, nch, ctx->sell_tails != 0,
                                                         P.head.as<int>(), ntr, nte, nwc, okey.as<uint32_t>());
    SPOPS_LAUNCH_CHECK();
    size_t cs = 0, cso = 0;
    SPOPS_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, cs, ntr, troff, nch + 1, st));
    if (ctx->sell_order)
      SPOPS_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, cso, okey.as<uint32_t>(), okey.as<uint32_t>(),
                                                 ord.as<int32_t>(), ord.as<int32_t>(), nch, 0, 32, st));
    SPOPS_TRY(tmp.alloc(std::max(cs, cso) + 256));
    SPOPS_CUDA(cub::DeviceScan::ExclusiveSum(tmp.p, cs, ntr, troff, nch + 1, st));
    SPOPS_CUDA(cub::DeviceScan::ExclusiveSum(tmp.p, cs, nte, teoff, nch + 1, st));
    if (ctx->sell_order) {  // windows of chunks of like length side by side in the list: longest first
      SPOPS_TRY(okey_s.alloc((size_t)nch * 4));
      SPOPS_TRY(ord_in.alloc((size_t)nch * 4));
      SPOPS_TRY(ord.alloc((size_t)nch * 4));
      SPOPS_TRY(nws.alloc((size_t)(nch + 1) * 8));
      SPOPS_TRY(woffs.alloc((size_t)(nch + 1) * 8));
      iota_i32_kernel<<<grid_for(nch), 256, 0, st>>>(ord_in.as<int32_t>(), nch);
      SPOPS_CUDA(cub::DeviceRadixSort::SortPairs(tmp.p, cso, okey.as<uint32_t>(), okey_s.as<uint32_t>(),
                                                 ord_in.as<int32_t>(), ord.as<int32_t>(), nch, 0, 32, st));
      pad_gather_nw_kernel<<<grid_for(nch + 1), 256, 0, st>>>(ord.as<int32_t>(), nwc, nch, nws.as<int64_t>());
      SPOPS_CUDA(cub::DeviceScan::ExclusiveSum(tmp.p, cs, nws.as<int64_t>(), woffs.as<int64_t>(), nch + 1, st));
      pad_scatter_woff_kernel<<<grid_for(nch + 1), 256, 0, st>>>(ord.as<int32_t>(), woffs.as<int64_t>(), nch, woff);
      SPOPS_LAUNCH_CHECK();
    } else {
      SPOPS_CUDA(cub::DeviceScan::ExclusiveSum(tmp.p, cs, nwc, woff, nch + 1, st));
    }
    int64_t h[3];
    SPOPS_TRY(download(ctx, &h[0], troff + nch, 1));
    SPOPS_TRY(download(ctx, &h[1], teoff + nch, 1));
    SPOPS_TRY(download(ctx, &h[2], woff + nch, 1));
    P.ntails = h[0];
    P.ntail_entries = h[1];
    P.nwin = h[2];
    SPOPS_TRY(P.win.alloc((size_t)P.nwin * sizeof(PadWin)));
    SPOPS_TRY(P.win_partial.alloc((size_t)P.nwin * 32 * sizeof(double)));
    SPOPS_TRY(P.win_counter.alloc((size_t)nch * sizeof(int)));
    SPOPS_TRY(P.tails.alloc((size_t)std::max<int64_t>(P.ntails, 1) * sizeof(PadTail)));
    SPOPS_TRY(P.tcol.alloc((size_t)std::max<int64_t>(P.ntail_entries, 1) * sizeof(I)));
    SPOPS_TRY(P.tval.alloc((size_t)std::max<int64_t>(P.ntail_entries, 1) * sizeof(V)));
    SPOPS_CUDA(cudaMemsetAsync(P.win_counter.p, 0, P.win_counter.bytes, st));
    pad_win_fill_kernel<<<grid_for(nch * 32), 256, 0, st>>>(P.row_len.as<int>(), n, nch, P.head.as<int>(), woff, nwc,
                                                             troff, teoff, P.win.as<PadWin>(), P.tails.as<PadTail>());
    SPOPS_LAUNCH_CHECK();
    if (P.ntails > 0) {
      pad_tail_copy_kernel<I, V><<<grid_for(P.ntails * 32), 256, 0, st>>>(
          P.tails.as<PadTail>(), P.ntails, P.chunk_off.as<int64_t>(), M->col.as<I>(), M->val.as<V>(),
          P.tcol.as<I>(), P.tval.as<V>());
      SPOPS_LAUNCH_CHECK();
    }
    P.tails_fresh = true;
    SPOPS_CUDA(cudaStreamSynchronize(st));
  }
  return SPOPS_OK;
}

template <typename I, typename V>
spops_status_t padded_spmv_t(Context* ctx, Matrix* A, double alpha, const void* x, double beta, void* y) {
  const PaddedData& P = A->pad;
  const int64_t n = A->rows;
  if (n == 0) return SPOPS_OK;
  const int64_t main_warps = (n + 31) / 32;
  const int64_t grid = (main_warps + P.npieces + 7) / 8;
  if (grid > INT32_MAX) return fail(SPOPS_ERR_TOO_LARGE, "padded SpMV grid");
  const I* ro = P.sorted ? P.reorder.as<I>() : nullptr;
  if (P.nwin > 0) {
    const int64_t g = (P.nwin + P.npieces + 7) / 8;
    if (g > INT32_MAX) return fail(SPOPS_ERR_TOO_LARGE, "padded SpMV grid");
    if (!P.tails_fresh && P.ntails > 0) {  // values changed: copy the tails again
      PaddedData& Pw = A->pad;
      pad_tail_copy_kernel<I, V><<<grid_for(P.ntails * 32), 256, 0, ctx->stream>>>(
          P.tails.as<PadTail>(), P.ntails, P.chunk_off.as<int64_t>(), A->col.as<I>(), A->val.as<V>(),
          Pw.tcol.as<I>(), Pw.tval.as<V>());
      SPOPS_LAUNCH_CHECK();
      Pw.tails_fresh = true;
    }
    padded_win_kernel<I, V><<<(unsigned)g, 256, 0, ctx->stream>>>(
        A->col.as<I>(), A->val.as<V>(), P.chunk_off.as<int64_t>(), P.row_len.as<int>(), ro, n,
        static_cast<const V*>(x), static_cast<V*>(y), (V)alpha, (V)beta, beta == 0.0, P.win.as<PadWin>(), P.nwin,
        P.win_partial.as<V>(), P.win_counter.as<int>(), P.npieces, P.piece.as<PadPiece>(), P.partial.as<V>(),
        P.counter.as<int>(), P.head.as<int>(), P.tcol.as<I>(), P.tval.as<V>());
    SPOPS_LAUNCH_CHECK();
    return SPOPS_OK;
  }
  if (A->layout == SPOPS_COL_MAJOR)
    padded_kernel<I, V, true><<<(unsigned)grid, 256, 0, ctx->stream>>>(
        A->col.as<I>(), A->val.as<V>(), P.chunk_len.as<I>(), P.chunk_off.as<int64_t>(), P.row_len.as<int>(), ro, n,
        P.C, static_cast<const V*>(x), static_cast<V*>(y), (V)alpha, (V)beta, beta == 0.0, main_warps, P.npieces,
        P.piece.as<PadPiece>(), P.partial.as<V>(), P.counter.as<int>());
  else
    padded_kernel<I, V, false><<<(unsigned)grid, 256, 0, ctx->stream>>>(
        A->col.as<I>(), A->val.as<V>(), P.chunk_len.as<I>(), P.chunk_off.as<int64_t>(), P.row_len.as<int>(), ro, n,
        P.C, static_cast<const V*>(x), static_cast<V*>(y), (V)alpha, (V)beta, beta == 0.0, main_warps, P.npieces,
        P.piece.as<PadPiece>(), P.partial.as<V>(), P.counter.as<int>());
  SPOPS_LAUNCH_CHECK();
  return SPOPS_OK;
}

// ------------------------------------------------------- DIA conversion
template <typename I, typename V>
spops_status_t to_dia(Context* ctx, Matrix* A, const spops_format_params_t& p, Matrix* M) {
  const int64_t n = A->rows, nc = A->cols;
  cudaStream_t st = ctx->stream;
  const int64_t max_diags = p.max_diags > 0 ? p.max_diags : 10240;
  const int64_t align = p.alignment > 0 ? p.alignment : 32 / (int64_t)sizeof(V);
  const int64_t nd_all = n + nc + 1;
  size_t cub_sort = 0;
  {
    unsigned long long* k = nullptr;
    int64_t* v = nullptr;
    SPOPS_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, cub_sort, k, k, v, v, nd_all, 0, 64, st));
  }
  const size_t na = (size_t)nd_all;
  SPOPS_TRY(ctx->scratch_reserve(na * (8 + 8 + 8 + 8 + 8 + 4) + cub_sort + 8 * 256));
  Carve cv(ctx->scratch.as<char>());
  unsigned long long* first = cv.take<unsigned long long>(na);
  unsigned long long* kin = cv.take<unsigned long long>(na);
  unsigned long long* kout = cv.take<unsigned long long>(na);
  int64_t* ids_in = cv.take<int64_t>(na);
  int64_t* ids_out = cv.take<int64_t>(na);
  int* dindex = cv.take<int>(na);
  int64_t* count = cv.take<int64_t>(1);
  void* cub_tmp = cv.take<char>(cub_sort);
  SPOPS_CUDA(cudaMemsetAsync(first, 0xff, na * 8, st));
  SPOPS_CUDA(cudaMemsetAsync(count, 0, 8, st));
  if (n > 0) {
    dia_first_kernel<I><<<grid_for(n * 32), 256, 0, st>>>(A->row.as<I>(), A->col.as<I>(), n, first);
    dia_select_kernel<<<grid_for(nd_all), 256, 0, st>>>(first, nd_all, kin, ids_in, count);
    SPOPS_LAUNCH_CHECK();
  }
  int64_t ndiag = 0;
  SPOPS_TRY(download(ctx, &ndiag, count, 1));
  if (ndiag > max_diags)
    return fail(SPOPS_ERR_TOO_LARGE, "DIA: %lld diagonals exceed the limit %lld", (long long)ndiag,
                (long long)max_diags);
  M->dia.ndiag = ndiag;
  M->dia.stride = n > 0 ? (n + align - 1) / align * align : 0;
  SPOPS_TRY(M->dia.offsets.alloc((size_t)(ndiag > 0 ? ndiag : 1) * sizeof(int64_t)));
  const double need = (double)ndiag * (double)M->dia.stride * sizeof(V);
  size_t free_b = 0, total_b = 0;
  SPOPS_CUDA(cudaMemGetInfo(&free_b, &total_b));
  if (need > 0.9 * (double)free_b) return fail(SPOPS_ERR_TOO_LARGE, "DIA needs %.1f GB", need / 1e9);
  SPOPS_TRY(M->dia.data.alloc((size_t)(ndiag * M->dia.stride > 0 ? ndiag * M->dia.stride : 1) * sizeof(V)));
  SPOPS_CUDA(cudaMemsetAsync(M->dia.data.p, 0, M->dia.data.bytes, st));
  if (ndiag > 0) {
    SPOPS_CUDA(cub::DeviceRadixSort::SortPairs(cub_tmp, cub_sort, kin, kout, ids_in, ids_out, ndiag, 0, 64, st));
    dia_index_kernel<<<grid_for(ndiag), 256, 0, st>>>(ids_out, ndiag, n, M->dia.offsets.as<int64_t>(), dindex);
    dia_fill_kernel<I, V><<<grid_for(n * 32), 256, 0, st>>>(A->row.as<I>(), A->col.as<I>(), A->val.as<V>(), n,
                                                            dindex, M->dia.stride, M->dia.data.as<V>());
    SPOPS_LAUNCH_CHECK();
  }
  SPOPS_CUDA(cudaStreamSynchronize(st));
  return SPOPS_OK;
}

// ------------------------------------------------------- BSR conversion
template <typename I, typename V>
spops_status_t to_bsr(Context* ctx, Matrix* A, const spops_format_params_t& p, Matrix* M) {
  const int64_t n = A->rows, nc = A->cols, nnz = A->nnz;
  cudaStream_t st = ctx->stream;
  BsrData& B = M->bsr;
  B.br = p.block_rows > 0 ? p.block_rows : 16;
  B.bc = p.block_cols > 0 ? p.block_cols : 32 / (int64_t)sizeof(V);
  if (B.br * B.bc > 1024) return fail(SPOPS_ERR_UNSUPPORTED, "BSR blocks larger than 1024 elements");
  B.mb = (n + B.br - 1) / B.br;
  B.nb = (nc + B.bc - 1) / B.bc;
  size_t cub_sort = 0, cub_uniq = 0, cub_scan = 0;
  {
    int64_t* k = nullptr;
    unsigned long long* u = nullptr;
    int64_t* cnt = nullptr;
    SPOPS_CUDA(cub::DeviceRadixSort::SortKeys(nullptr, cub_sort, k, k, (int64_t)(nnz > 0 ? nnz : 1), 0, 64, st));
    SPOPS_CUDA(cub::DeviceSelect::Unique(nullptr, cub_uniq, k, k, cnt, (int64_t)(nnz > 0 ? nnz : 1), st));
    SPOPS_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, cub_scan, u, u, (int64_t)(B.mb + 1), st));
  }
  const size_t nz = (size_t)(nnz > 0 ? nnz : 1), nmb = (size_t)B.mb + 1;
  SPOPS_TRY(ctx->scratch_reserve(3 * nz * 8 + 2 * nmb * 8 + std::max({cub_sort, cub_uniq, cub_scan}) + 8 * 256));
  Carve cv(ctx->scratch.as<char>());
  int64_t* keys = cv.take<int64_t>(nz);
  int64_t* skeys = cv.take<int64_t>(nz);
  int64_t* ukeys = cv.take<int64_t>(nz);
  unsigned long long* cnt = cv.take<unsigned long long>(nmb);
  unsigned long long* scan = cv.take<unsigned long long>(nmb);
  int64_t* nuniq = cv.take<int64_t>(1);
  void* cub_tmp = cv.take<char>(std::max({cub_sort, cub_uniq, cub_scan}));
  SPOPS_CUDA(cudaMemsetAsync(nuniq, 0, 8, st));
  if (nnz > 0) {
    bsr_keys_kernel<I><<<grid_for(n * 32), 256, 0, st>>>(A->row.as<I>(), A->col.as<I>(), n, B.br, B.bc, B.nb, keys);
    SPOPS_LAUNCH_CHECK();
    SPOPS_CUDA(cub::DeviceRadixSort::SortKeys(cub_tmp, cub_sort, keys, skeys, nnz, 0, 64, st));
    SPOPS_CUDA(cub::DeviceSelect::Unique(cub_tmp, cub_uniq, skeys, ukeys, nuniq, nnz, st));
  }
  int64_t nnzb = 0;
  SPOPS_TRY(download(ctx, &nnzb, nuniq, 1));
  B.nnzb = nnzb;
  const int64_t blk = B.br * B.bc;
  SPOPS_TRY(B.row_ptr.alloc(nmb * sizeof(I)));
  SPOPS_TRY(B.bcol.alloc((size_t)(nnzb > 0 ? nnzb : 1) * sizeof(I)));
  SPOPS_TRY(B.data.alloc((size_t)(nnzb > 0 ? nnzb * blk : 1) * sizeof(V)));
  SPOPS_CUDA(cudaMemsetAsync(B.data.p, 0, B.data.bytes, st));
  SPOPS_CUDA(cudaMemsetAsync(cnt, 0, nmb * 8, st));
  if (nnzb > 0) {
    bsr_struct_kernel<I><<<grid_for(nnzb), 256, 0, st>>>(ukeys, nnzb, B.nb, B.bcol.as<I>(), cnt);
    SPOPS_LAUNCH_CHECK();
  }
  SPOPS_CUDA(cub::DeviceScan::ExclusiveSum(cub_tmp, cub_scan, cnt, scan, (int64_t)nmb, st));
  bsr_rowptr_kernel<I><<<grid_for((int64_t)nmb), 256, 0, st>>>(reinterpret_cast<const int64_t*>(scan), B.mb,
                                                               B.row_ptr.as<I>());
  if (nnzb > 0)
    bsr_fill_kernel<I, V><<<grid_for(n * 32), 256, 0, st>>>(A->row.as<I>(), A->col.as<I>(), A->val.as<V>(), n, B.br,
                                                            B.bc, B.nb, ukeys, nnzb, B.data.as<V>());
  SPOPS_LAUNCH_CHECK();
  SPOPS_CUDA(cudaStreamSynchronize(st));
  return SPOPS_OK;
}

// ------------------------------------------------------- COO conversion
template <typename I, typename V>
spops_status_t to_coo(Context* ctx, Matrix* A, Matrix* M) {
  cudaStream_t st = ctx->stream;
  const int64_t nz = A->nnz;
  SPOPS_TRY(M->row.alloc((size_t)(nz > 0 ? nz : 1) * sizeof(I)));
  SPOPS_TRY(M->col.alloc((size_t)(nz > 0 ? nz : 1) * sizeof(I)));
  SPOPS_TRY(M->val.alloc((size_t)(nz > 0 ? nz : 1) * sizeof(V)));
  if (nz > 0) {
    csr_expand_rows_kernel<I><<<grid_for(A->rows * 32), 256, 0, st>>>(A->row.as<I>(), A->rows, M->row.as<I>());
    SPOPS_LAUNCH_CHECK();
    SPOPS_CUDA(cudaMemcpyAsync(M->col.p, A->col.p, nz * sizeof(I), cudaMemcpyDeviceToDevice, st));
    SPOPS_CUDA(cudaMemcpyAsync(M->val.p, A->val.p, nz * sizeof(V), cudaMemcpyDeviceToDevice, st));
  }
  return coo_analyse(ctx, M);
}

template <typename I, typename V>
spops_status_t coo_analyse_t(Context* ctx, Matrix* A) {
  cudaStream_t st = ctx->stream;
  const int64_t n = A->rows, nz = A->nnz;
  size_t cub_sort = 0, cub_scan = 0;
  {
    I* k = nullptr;
    int64_t* v = nullptr;
    unsigned long long* u = nullptr;
    SPOPS_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, cub_sort, k, k, v, v, (int64_t)(nz > 0 ? nz : 1), 0,
                                               8 * (int)sizeof(I), st));
    SPOPS_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, cub_scan, u, u, (int64_t)(n + 1), st));
  }
  const size_t nzz = (size_t)(nz > 0 ? nz : 1), n1 = (size_t)n + 1;
  SPOPS_TRY(ctx->scratch_reserve(nzz * (sizeof(I) + 16) + 2 * n1 * 8 + std::max(cub_sort, cub_scan) + 8 * 256));
  Carve cv(ctx->scratch.as<char>());
  I* skeys = cv.take<I>(nzz);
  int64_t* perm_in = cv.take<int64_t>(nzz);
  int64_t* perm = cv.take<int64_t>(nzz);
  unsigned long long* cnt = cv.take<unsigned long long>(n1);
  unsigned long long* scan = cv.take<unsigned long long>(n1);
  int* flags = cv.take<int>(1);
  void* cub_tmp = cv.take<char>(std::max(cub_sort, cub_scan));
  SPOPS_CUDA(cudaMemsetAsync(cnt, 0, n1 * 8, st));
  SPOPS_CUDA(cudaMemsetAsync(flags, 0, 4, st));
  if (nz > 0) {
    coo_check_kernel<I><<<std::min<unsigned>(grid_for(nz), 4096u), 256, 0, st>>>(A->row.as<I>(), A->col.as<I>(), nz,
                                                                                  n, A->cols, flags, cnt);
    SPOPS_LAUNCH_CHECK();
  }
  int hflags = 0;
  SPOPS_TRY(download(ctx, &hflags, flags, 1));
  if (hflags & 2) return fail(SPOPS_ERR_INVALID, "COO: row or column index out of range");
  Matrix* C = new Matrix();
  C->ctx = ctx;
  C->format = SPOPS_FMT_CSR;
  C->itype = A->itype;
  C->vtype = A->vtype;
  C->rows = n;
  C->cols = A->cols;
  C->nnz = nz;
  spops_status_t s = C->row.alloc(n1 * sizeof(I));
  if (s == SPOPS_OK) {
    SPOPS_CUDA(cub::DeviceScan::ExclusiveSum(cub_tmp, cub_scan, cnt, scan, (int64_t)n1, st));
    to_index_kernel<I><<<grid_for((int64_t)n1), 256, 0, st>>>(scan, (int64_t)n1, C->row.as<I>());
    if (!(hflags & 1)) {  // already sorted by row: borrow the arrays
      C->col.borrow(A->col.p, A->col.bytes);
      C->val.borrow(A->val.p, A->val.bytes);
    } else {
      s = C->col.alloc(nzz * sizeof(I));
      if (s == SPOPS_OK) s = C->val.alloc(nzz * sizeof(V));
      if (s == SPOPS_OK) {
        iota_kernel<<<grid_for(nz), 256, 0, st>>>(perm_in, nz);
        SPOPS_CUDA(cub::DeviceRadixSort::SortPairs(cub_tmp, cub_sort, A->row.as<I>(), skeys, perm_in, perm, nz, 0,
                                                   8 * (int)sizeof(I), st));
        gather_kernel<I, V><<<grid_for(nz), 256, 0, st>>>(perm, A->col.as<I>(), A->val.as<V>(), nz, C->col.as<I>(),
                                                          C->val.as<V>());
        SPOPS_LAUNCH_CHECK();
      }
    }
  }
  if (s == SPOPS_OK) s = csr_analyse(ctx, C);
  if (s != SPOPS_OK) {
    C->release_all();
    delete C;
    return s;
  }
  if (A->csr_view) {
    A->csr_view->release_all();
    delete A->csr_view;
  }
  A->csr_view = C;
  return SPOPS_OK;
}

template <typename I, typename V>
spops_status_t dia_spmv_t(Context* ctx, Matrix* A, double alpha, const void* x, double beta, void* y) {
  if (A->rows == 0) return SPOPS_OK;
  DiaData& D = A->dia;
  if (!D.span_known) {
    std::vector<int64_t> off((size_t)D.ndiag);
    if (D.ndiag > 0) SPOPS_TRY(download(ctx, off.data(), D.offsets.as<int64_t>(), D.ndiag));
    D.lo = D.ndiag > 0 ? *std::min_element(off.begin(), off.end()) : 0;
    D.hi = D.ndiag > 0 ? *std::max_element(off.begin(), off.end()) : 0;
    D.span_known = true;
  }
  const int64_t win = 256 + D.hi - D.lo;
  if (D.ndiag > 0 && D.ndiag <= kDiaStageMaxDiags && win <= kDiaStageMaxWin) {
    dia_staged_kernel<V><<<grid_for(A->rows), 256, (size_t)win * sizeof(V), ctx->stream>>>(
        D.offsets.as<int64_t>(), D.data.as<V>(), D.ndiag, D.stride, A->rows, A->cols, static_cast<const V*>(x),
        static_cast<V*>(y), (V)alpha, (V)beta, beta == 0.0, D.lo, win);
    SPOPS_LAUNCH_CHECK();
    return SPOPS_OK;
  }
  dia_kernel<V><<<grid_for(A->rows), 256, 0, ctx->stream>>>(
      A->dia.offsets.as<int64_t>(), A->dia.data.as<V>(), A->dia.ndiag, A->dia.stride, A->rows, A->cols,
      static_cast<const V*>(x), static_cast<V*>(y), (V)alpha, (V)beta, beta == 0.0);
  SPOPS_LAUNCH_CHECK();
  return SPOPS_OK;
}

template <typename I, typename V>
spops_status_t bsr_spmv_t(Context* ctx, Matrix* A, double alpha, const void* x, double beta, void* y) {
  const BsrData& B = A->bsr;
  if (B.mb == 0) return SPOPS_OK;
  const size_t smem = (size_t)8 * B.br * B.bc * sizeof(V);
  if (smem > 48 * 1024)
    SPOPS_CUDA(cudaFuncSetAttribute(bsr_kernel<I, V>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  bsr_kernel<I, V><<<grid_for(B.mb, 8), 256, smem, ctx->stream>>>(
      B.row_ptr.as<I>(), B.bcol.as<I>(), B.data.as<V>(), B.mb, (int)B.br, (int)B.bc, A->rows, A->cols,
      static_cast<const V*>(x), static_cast<V*>(y), (V)alpha, (V)beta, beta == 0.0);
  SPOPS_LAUNCH_CHECK();
  return SPOPS_OK;
}

template <typename I, typename V>
spops_status_t convert_t(Context* ctx, Matrix* A, spops_format_t fmt, const spops_format_params_t& p, Matrix* M) {
  switch (fmt) {
    case SPOPS_FMT_SELL_C_SIGMA:
    case SPOPS_FMT_SELL_C_R:
    case SPOPS_FMT_SELL:
    case SPOPS_FMT_ELL: return to_padded<I, V>(ctx, A, fmt, p, M);
    case SPOPS_FMT_DIA: return to_dia<I, V>(ctx, A, p, M);
    case SPOPS_FMT_BSR: return to_bsr<I, V>(ctx, A, p, M);
    case SPOPS_FMT_COO: return to_coo<I, V>(ctx, A, M);
    case SPOPS_FMT_CSR5: return csr5_build(ctx, A, M);
    default: return fail(SPOPS_ERR_UNSUPPORTED, "conversion CSR -> format %d", (int)fmt);
  }
}

#define SPOPS_DISPATCH(A, FN, ...)                                                              \
  (((A)->itype == SPOPS_INDEX_I32)                                                              \
       ? (((A)->vtype == SPOPS_VALUE_F64) ? FN<int32_t, double>(__VA_ARGS__) : FN<int32_t, float>(__VA_ARGS__)) \
       : (((A)->vtype == SPOPS_VALUE_F64) ? FN<int64_t, double>(__VA_ARGS__) : FN<int64_t, float>(__VA_ARGS__)))

}  // namespace

void Matrix::release_all() {
  row.release();
  col.release();
  val.release();
  plan.release();
  pad.release();
  dia.release();
  bsr.release();
  tr.release();
  csr5.release();
  spmm_partial.release();
  cl_sz.release();
  cl_rpv.release();
  cl_off.release();
  if (csr_view) {
    csr_view->release_all();
    delete csr_view;
    csr_view = nullptr;
  }
}

spops_status_t convert_from_csr(Context* ctx, Matrix* A, spops_format_t fmt, const spops_format_params_t& p,
                                Matrix** out) {
  if (A->format != SPOPS_FMT_CSR) return fail(SPOPS_ERR_INVALID, "conversion source must be a CSR matrix");
  if (!A->plan.ready) SPOPS_TRY(csr_analyse(ctx, A));  // validates the pattern
  Matrix* M = new spops_matrix_s();
  M->ctx = ctx;
  M->format = fmt;
  M->itype = A->itype;
  M->vtype = A->vtype;
  M->rows = A->rows;
  M->cols = A->cols;
  M->nnz = A->nnz;
  spops_status_t s = SPOPS_DISPATCH(A, convert_t, ctx, A, fmt, p, M);
  if (s != SPOPS_OK) {
    M->release_all();
    delete static_cast<spops_matrix_s*>(M);
    return s;
  }
  *out = M;
  return SPOPS_OK;
}

spops_status_t padded_finish(Context* ctx, Matrix* M) { return SPOPS_DISPATCH(M, padded_finish_t, ctx, M); }

spops_status_t padded_spmv(Context* ctx, Matrix* A, double alpha, const void* x, double beta, void* y) {
  return SPOPS_DISPATCH(A, padded_spmv_t, ctx, A, alpha, x, beta, y);
}

spops_status_t dia_spmv(Context* ctx, Matrix* A, double alpha, const void* x, double beta, void* y) {
  return SPOPS_DISPATCH(A, dia_spmv_t, ctx, A, alpha, x, beta, y);
}

spops_status_t bsr_spmv(Context* ctx, Matrix* A, double alpha, const void* x, double beta, void* y) {
  return SPOPS_DISPATCH(A, bsr_spmv_t, ctx, A, alpha, x, beta, y);
}

spops_status_t coo_analyse(Context* ctx, Matrix* A) { return SPOPS_DISPATCH(A, coo_analyse_t, ctx, A); }

spops_status_t validate_columns(Context* ctx, const void* col, int64_t count, spops_index_t it, int64_t ncols,
                                bool allow_pad) {
  if (count <= 0) return SPOPS_OK;
  SPOPS_TRY(ctx->scratch_reserve(256));
  int* bad = ctx->scratch.as<int>();
  SPOPS_CUDA(cudaMemsetAsync(bad, 0, 4, ctx->stream));
  const unsigned g = std::min<unsigned>(grid_for(count), 4096u);
  if (it == SPOPS_INDEX_I32)
    validate_cols_kernel<int32_t><<<g, 256, 0, ctx->stream>>>(static_cast<const int32_t*>(col), count, ncols,
                                                              allow_pad, bad);
  else
    validate_cols_kernel<int64_t><<<g, 256, 0, ctx->stream>>>(static_cast<const int64_t*>(col), count, ncols,
                                                              allow_pad, bad);
  SPOPS_LAUNCH_CHECK();
  int h = 0;
  SPOPS_TRY(download(ctx, &h, bad, 1));
  if (h) return fail(SPOPS_ERR_INVALID, "column index outside [0, cols)%s", allow_pad ? " (and not padding -1)" : "");
  return SPOPS_OK;
}

}  // namespace spops

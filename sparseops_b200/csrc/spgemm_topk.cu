// Row-wise SpGEMM (LeSpGEMM kernels 1-3) and the top-k Jaccard similarity
// product (HashSpGEMMTopK) on the device.
//
// Row-wise: replaces LeSpGEMM (reference src/spgemm.cpp:683-706) with its
// hash (44-110), array (113-175) and sparse-accumulator (178-235) row
// kernels.  All three compute C = A*B with every structural entry of the
// product kept -- exact zeros included, no small-value drop -- and differ only
// in the order of a row's columns when unsorted (hash-slot order for kernel 1
// with sortOutput = false, ascending otherwise).  Here every row comes out
// with ascending columns (a valid order for all of them): the cluster-wise
// pipeline of spgemm.cu runs with one cluster per row and the row-wise output
// rules.
//
// Top-k: replaces HashSpGEMMTopK (src/spgemm.cpp:708-842) with
// spgemm_hash_numeric_topk_omp_lb and sort_and_store_table2mat_topk_jaccard
// (src/spgemm_hash.cpp:168-318):
//   1. the binary pattern of A (values 1) times its transpose (built on the
//      device, rows in ascending original row as csr_transpose orders them)
//      gives |A_i n A_j| for every structural pair (i, j);
//   2. per entry j != i: u = |A_i| + |A_j| - inter (row lengths of A),
//      jacc = u == 0 ? 0 : (V)1 * inter / (V)u in the value type;
//   3. per row, entries ranked by (jacc descending, column ascending) and
//      the first top_k kept, the diagonal excluded, by one stable segmented
//      radix sort of a descending key with the columns in ascending order as
//      payload.  Rows of the result are in that order, as the reference's.
// For top_k <= 32 the counts are not materialised: each row's counts build up
// in a hash table of its own and the best k are selected from the table (the
// fused path below, steps 1-3 in one kernel per row size).
#include <cub/cub.cuh>

#include <numeric>
#include <vector>

#include "spops_internal.h"

namespace spops {
namespace {

inline unsigned grid_for(int64_t work, int threads = 256) {
  int64_t g = (work + threads - 1) / threads;
  return (unsigned)(g < 1 ? 1 : g);
}

template <typename V>
__global__ void fill_kernel(V* __restrict__ a, int64_t n, V v) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i < n) a[i] = v;
}

// Descending sort key of a non-negative similarity; the diagonal sorts last.
__device__ __forceinline__ uint64_t desc_key(double v) {
  const uint64_t b = (uint64_t)__double_as_longlong(v);  // v >= 0: bits ordered as values
  return b == 0 ? ~(uint64_t)1 : ~b;                      // ~b; +0.0 just before the diagonal
}
__device__ __forceinline__ uint64_t desc_key(float v) { return (uint64_t)(0xffffffffu - __float_as_uint(v)); }
__device__ __forceinline__ double from_key(uint64_t k, double) {
  return k == ~(uint64_t)1 ? 0.0 : __longlong_as_double((long long)~k);
}
__device__ __forceinline__ float from_key(uint64_t k, float) { return __uint_as_float(0xffffffffu - (uint32_t)k); }

constexpr uint64_t kDiagKey = ~(uint64_t)0;

// One warp per row i of the intersection counts C: the key of every entry
// and whether the row holds its diagonal.
template <typename I, typename V>
__global__ void jaccard_key_kernel(const I* __restrict__ crp, const I* __restrict__ cci, const V* __restrict__ cval,
                                   const I* __restrict__ arp, int64_t n, uint64_t* __restrict__ key,
                                   I* __restrict__ col, int64_t* __restrict__ has_diag) {
  const int64_t i = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (i >= n) return;
  const int64_t e0 = crp[i], e1 = crp[i + 1];
  const int64_t li = (int64_t)arp[i + 1] - (int64_t)arp[i];
  int diag = 0;
  for (int64_t e = e0 + lane; e < e1; e += 32) {
    const int64_t j = cci[e];
    col[e] = (I)j;
    if (j == i) {
      key[e] = kDiagKey;
      diag = 1;
      continue;
    }
    const V inter = cval[e];
    const int64_t u = li + ((int64_t)arp[j + 1] - (int64_t)arp[j]) - (int64_t)inter;
    const V jacc = u == 0 ? V(0) : V(1) * inter / (V)u;
    key[e] = desc_key(jacc);
  }
  diag = __any_sync(0xffffffffu, diag);
  if (lane == 0) has_diag[i] = diag;
}

template <typename I>
__global__ void kept_kernel(const I* __restrict__ crp, const int64_t* __restrict__ has_diag, int64_t n, int64_t k,
                            int64_t* __restrict__ kept) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i > n) return;
  if (i == n) {
    kept[n] = 0;
    return;
  }
  const int64_t avail = (int64_t)crp[i + 1] - (int64_t)crp[i] - has_diag[i];
  kept[i] = avail < k ? avail : k;
}

template <typename I, typename V>
__global__ void topk_write_kernel(const I* __restrict__ crp, const uint64_t* __restrict__ skey,
                                  const I* __restrict__ scol, const int64_t* __restrict__ orp, int64_t n,
                                  I* __restrict__ out_rp, I* __restrict__ oci, V* __restrict__ ov) {
  const int64_t i = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (i > n) return;
  if (lane == 0) out_rp[i] = (I)orp[i];
  if (i == n) return;
  const int64_t s = crp[i], o = orp[i], m = orp[i + 1] - orp[i];
  for (int64_t t = lane; t < m; t += 32) {  // the first m keys of the row are its best non-diagonal entries
    oci[o + t] = scol[s + t];
    ov[o + t] = from_key(skey[s + t], V(0));
  }
}

// (key, column) order of the ranking: key ascending (similarity descending),
// then column ascending -- the order the stable segmented sort gives.
__device__ __forceinline__ bool rank_less(uint64_t ka, int64_t ca, uint64_t kb, int64_t cb) {
  return ka < kb || (ka == kb && ca < cb);
}

// One compare-exchange step of a warp-wide bitonic network over one
// (key, column) per lane; `up` says whether this lane's block ascends.
__device__ __forceinline__ void warp_cx(uint64_t& k, int64_t& c, int j, bool up) {
  const int lane = threadIdx.x & 31;
  const uint64_t pk = __shfl_xor_sync(0xffffffffu, k, j);
  const int64_t pc = __shfl_xor_sync(0xffffffffu, c, j);
  const bool keep_min = ((lane & j) == 0) == up;
  const bool take = keep_min ? rank_less(pk, pc, k, c) : rank_less(k, c, pk, pc);
  if (take) {
    k = pk;
    c = pc;
  }
}

__device__ __forceinline__ void warp_sort32(uint64_t& k, int64_t& c) {
  const int lane = threadIdx.x & 31;
  for (int b = 2; b <= 32; b <<= 1)
    for (int j = b >> 1; j > 0; j >>= 1) warp_cx(k, c, j, (lane & b) == 0);
}

// The best 32 (key, column) pairs a warp has been offered, sorted across the
// lanes (lane l holds the l-th best), for a top-k with k <= 32.  Only pairs
// that rank before the current k-th best are kept as candidates, compacted
// into a 64-slot buffer in shared memory; each time 32 are there they are
// sorted and merged into the best 32 (lane l keeps the better of best[l] and
// cand[31 - l], which leaves the best 32 of both as a bitonic sequence; five
// steps sort it) and the k-th best moves up.  A pair that does not beat the
// k-th best when it is offered ranks after k pairs already seen, so the
// filter drops nothing of the result.  A random order of m pairs brings about
// k ln(m / k) candidates, so most offers cost a ballot.
struct WarpTop {
  uint64_t* buf_k;
  int64_t* buf_c;
  int k, lane, nbuf;
  uint64_t bk, tk;  // the lane's entry of the best 32; the k-th best
  int64_t bc, tc;
  __device__ __forceinline__ WarpTop(uint64_t* bkey, int64_t* bcol, int k_, int lane_)
      : buf_k(bkey), buf_c(bcol), k(k_), lane(lane_), nbuf(0), bk(kDiagKey), tk(kDiagKey), bc(INT64_MAX),
        tc(INT64_MAX) {}  // padding sorts after every entry, the diagonal included
  // merge 32 pairs sorted ascending across the lanes
  __device__ __forceinline__ void merge_sorted(uint64_t ck, int64_t cc) {
    const uint64_t rk = __shfl_sync(0xffffffffu, ck, 31 - lane);
    const int64_t rc = __shfl_sync(0xffffffffu, cc, 31 - lane);
    if (rank_less(rk, rc, bk, bc)) {
      bk = rk;
      bc = rc;
    }
    for (int j = 16; j > 0; j >>= 1) warp_cx(bk, bc, j, true);
    tk = __shfl_sync(0xffffffffu, bk, k - 1);
    tc = __shfl_sync(0xffffffffu, bc, k - 1);
  }
  __device__ __forceinline__ void merge(uint64_t ck, int64_t cc) {
    warp_sort32(ck, cc);
    merge_sorted(ck, cc);
  }
  __device__ __forceinline__ void offer(uint64_t key, int64_t col, bool ok) {
    const bool cand = ok && rank_less(key, col, tk, tc);
    const unsigned m = __ballot_sync(0xffffffffu, cand);
    if (cand) {
      const int p = nbuf + __popc(m & ((1u << lane) - 1u));  // nbuf <= 31 before, so p <= 62
      buf_k[p] = key;
      buf_c[p] = col;
    }
    nbuf += __popc(m);
    if (nbuf >= 32) {
      __syncwarp();
      const uint64_t ck = buf_k[lane];
      const int64_t cc = buf_c[lane];
      const int rest = nbuf - 32;
      uint64_t rk = 0;
      int64_t rc = 0;
      if (lane < rest) {
        rk = buf_k[32 + lane];
        rc = buf_c[32 + lane];
      }
      __syncwarp();
      if (lane < rest) {
        buf_k[lane] = rk;
        buf_c[lane] = rc;
      }
      nbuf = rest;
      merge(ck, cc);
    }
  }
  __device__ __forceinline__ void flush() {
    if (nbuf > 0) {
      __syncwarp();
      const uint64_t ck = lane < nbuf ? buf_k[lane] : kDiagKey;
      const int64_t cc = lane < nbuf ? buf_c[lane] : INT64_MAX;
      nbuf = 0;
      merge(ck, cc);
    }
  }
};

// ---- fused top-k for k <= 32: the intersection counts are never written.
// Row i's counts |A_i n A_j| accumulate in a hash table (one warp's, or one
// block's of W warps; in shared memory, or in global memory for rows of more
// than 8192 products): every pair of a column c of row i and a row j holding
// c (row c of the pattern's transpose) adds one to j's count.  The counts are
// integers, so the order of the additions does not matter, and the
// transpose's rows need no order either.  Each new key also goes to a list of
// the occupied slots; the listed slots go to WarpTop as a materialised row
// would (warp 0 of a block merges the other warps' best 32) and are then
// cleared, so a table is cleared in full only once per kernel.  j = i is not
// counted; it is in C's row whenever row i has an entry, which is all the
// exclusion of the diagonal needs.
constexpr uint32_t kEmptySlot = 0xffffffffu;
constexpr int kHashBins = 5;  // products <= 128, 512, 2048, 8192, more

__host__ __device__ constexpr int64_t hash_bin_max(int bin) { return (int64_t)128 << (2 * bin); }

// adds one to j's count; returns the slot, plus kFreshSlot when j was not in
// the table before, or -1 when the table is full (it has at least twice as
// many slots as the row has products, so this does not happen)
constexpr int64_t kFreshSlot = (int64_t)1 << 40;

__device__ __forceinline__ int64_t slot_add(uint32_t* keys, uint32_t* cnts, uint32_t j, int log_s) {
  const uint32_t mask = (uint32_t)(((uint64_t)1 << log_s) - 1u);
  uint32_t h = (j * 2654435761u) >> (32 - log_s);
  for (uint32_t probe = 0; probe <= mask; ++probe) {
    const uint32_t cur = *reinterpret_cast<volatile uint32_t*>(keys + h);
    if (cur == j) {
      atomicAdd(cnts + h, 1u);
      return h;
    }
    if (cur == kEmptySlot) {
      const uint32_t prev = atomicCAS(keys + h, kEmptySlot, j);
      if (prev == kEmptySlot || prev == j) {
        atomicAdd(cnts + h, 1u);
        return (int64_t)h + (prev == kEmptySlot ? kFreshSlot : 0);
      }
    }
    h = (h + 1) & mask;
  }
  return -1;
}

// Per warp of a row group: the B row starts and product offsets of 32 of the
// row's columns, and the WarpTop candidate buffer (which also carries the
// warp's best 32 to warp 0 of the group).
struct HashWarpSmem {
  int64_t st[32];
  int32_t off[33];
  uint64_t bkey[64];
  int64_t bcol[64];
};

template <int W>
__device__ __forceinline__ void group_sync() {
  if constexpr (W == 1) __syncwarp(); else __syncthreads();
}

// One row with a group of W warps (wg = this warp's index in the group) over
// a table of 2^log_s slots whose keys are all empty and counts zero; leaves
// it so.  `list` holds up to 2^(log_s - 1) slot indices, *nlist is zero.
template <typename I, typename V, int W, typename L>
__device__ __forceinline__ void topk_hash_row(int64_t i, uint32_t* keys, uint32_t* cnts, int log_s, L* list,
                                              int* nlist, const I* __restrict__ arp, const I* __restrict__ aci,
                                              const I* __restrict__ trp, const I* __restrict__ tci, int k,
                                              HashWarpSmem* ws, int wg, int lane, uint64_t* tkey, I* tcol,
                                              int64_t* kept, int* err) {
  HashWarpSmem& me = ws[wg];
  // ---- counts
  const int64_t a0 = arp[i], nj = (int64_t)arp[i + 1] - a0;
  bool full = false;
  for (int64_t q0 = (int64_t)wg * 32; q0 < nj; q0 += W * 32) {
    const int64_t q = q0 + lane;
    int64_t st = 0;
    int32_t len = 0;
    if (q < nj) {
      const int64_t c = aci[a0 + q];
      st = trp[c];
      len = (int32_t)((int64_t)trp[c + 1] - st);
    }
    int32_t incl = len;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int32_t u = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += u;
    }
    me.st[lane] = st;
    me.off[lane + 1] = incl;
    if (lane == 0) me.off[0] = 0;
    __syncwarp();
    const int32_t total = me.off[32];
    for (int32_t t0 = lane; t0 < total; t0 += 128) {
      uint32_t jj[4];
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        const int32_t t = t0 + 32 * u;
        jj[u] = kEmptySlot;
        if (t < total) {
          int m = 0;  // the column of product t: last m with off[m] <= t
#pragma unroll
          for (int step = 16; step > 0; step >>= 1)
            if (me.off[m + step] <= t) m += step;
          jj[u] = (uint32_t)tci[me.st[m] + (t - me.off[m])];
        }
      }
#pragma unroll
      for (int u = 0; u < 4; ++u)
        if (jj[u] != kEmptySlot && (int64_t)jj[u] != i) {
          const int64_t h = slot_add(keys, cnts, jj[u], log_s);
          if (h < 0) full = true;
          else if (h >= kFreshSlot) list[atomicAdd(nlist, 1)] = (L)(h - kFreshSlot);
        }
    }
    __syncwarp();
  }
  if (full) atomicOr(err, 2);
  group_sync<W>();
  // ---- selection over the occupied slots
  const int d = *nlist;
  WarpTop top(me.bkey, me.bcol, k, lane);
  const int64_t li = nj;
  for (int q0 = wg * 32; q0 < d; q0 += W * 32) {
    const int q = q0 + lane;
    uint64_t key = kDiagKey;
    int64_t col = INT64_MAX;
    if (q < d) {
      const uint32_t h = (uint32_t)list[q];
      const uint32_t j = keys[h];
      const V inter = (V)cnts[h];
      const int64_t u = li + ((int64_t)arp[j + 1] - (int64_t)arp[j]) - (int64_t)inter;
      key = desc_key(u == 0 ? V(0) : V(1) * inter / (V)u);
      col = (int64_t)j;
    }
    top.offer(key, col, q < d);
  }
  top.flush();
  if constexpr (W > 1) {
    if (wg > 0) {  // the buffer is empty after flush: it carries this warp's best 32
      me.bkey[lane] = top.bk;
      me.bcol[lane] = top.bc;
    }
  }
  group_sync<W>();  // every slot has been read
  // ---- clear the used slots for the next row
  for (int q = wg * 32 + lane; q < d; q += W * 32) {
    const uint32_t h = (uint32_t)list[q];
    keys[h] = kEmptySlot;
    cnts[h] = 0;
  }
  if (wg == 0) {
    if constexpr (W > 1) {
      for (int w = 1; w < W; ++w) {
        const uint64_t ck = ws[w].bkey[lane];
        const int64_t cc = ws[w].bcol[lane];
        if (__any_sync(0xffffffffu, rank_less(ck, cc, top.tk, top.tc))) top.merge_sorted(ck, cc);
      }
    }
    if (lane < k) {
      tkey[i * k + lane] = top.bk;
      tcol[i * k + lane] = (I)(top.bc == INT64_MAX ? 0 : top.bc);
    }
    if (lane == 0) kept[i] = d < k ? d : k;
  }
  group_sync<W>();  // slots cleared and the warps' lists read
  if (wg == 0 && lane == 0) *nlist = 0;
  group_sync<W>();
}

// Rows whose tables fit in shared memory: RPB groups of W warps per block,
// each taking rows in turn over its own table of 2^LOG_S slots and its list.
template <typename I, typename V, int W, int RPB, int LOG_S>
__global__ void __launch_bounds__(W * RPB * 32)
    topk_hash_kernel(const int32_t* __restrict__ rows, int64_t nrows, const I* __restrict__ arp,
                     const I* __restrict__ aci, const I* __restrict__ trp, const I* __restrict__ tci, int k,
                     uint64_t* __restrict__ tkey, I* __restrict__ tcol, int64_t* __restrict__ kept,
                     int* __restrict__ err) {
  constexpr uint32_t S = 1u << LOG_S;
  extern __shared__ __align__(16) uint32_t hash_smem[];  // per group: keys[S], counts[S], list[S / 2] (16-bit)
  __shared__ HashWarpSmem ws[W * RPB];
  __shared__ int s_n[RPB];
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5, g = wib / W, wg = wib % W;
  uint32_t* keys = hash_smem + (size_t)g * (2 * S + S / 4);
  uint32_t* cnts = keys + S;
  uint16_t* list = reinterpret_cast<uint16_t*>(cnts + S);
  for (uint32_t q = wg * 32 + lane; q < S; q += W * 32) {
    keys[q] = kEmptySlot;
    cnts[q] = 0;
  }
  if (wg == 0 && lane == 0) s_n[g] = 0;
  group_sync<W>();
  // rows b = blockIdx.x * RPB + g + m * gridDim.x * RPB; a group whose rows
  // run out leaves (RPB > 1 only with W == 1: no block-wide barrier follows)
  for (int64_t b = blockIdx.x * (int64_t)RPB + g; b < nrows; b += (int64_t)gridDim.x * RPB)
    topk_hash_row<I, V, W, uint16_t>(rows[b], keys, cnts, LOG_S, list, s_n + g, arp, aci, trp, tci, k, ws + g * W,
                                     wg, lane, tkey, tcol, kept, err);
}

// The longest rows: one block of W warps per row at a time, over the first
// 2^ceil(log2(2P)) slots of a table of gslots slots and a list, in the
// block's region of global memory (keys[gslots], counts[gslots],
// list[gslots / 2]), cleared here once.
template <typename I, typename V, int W>
__global__ void __launch_bounds__(W * 32)
    topk_hash_global_kernel(const int32_t* __restrict__ rows, int64_t nrows, const int64_t* __restrict__ prods,
                            const I* __restrict__ arp, const I* __restrict__ aci, const I* __restrict__ trp,
                            const I* __restrict__ tci, int k, uint32_t* __restrict__ gtab, int64_t gslots,
                            uint64_t* __restrict__ tkey, I* __restrict__ tcol, int64_t* __restrict__ kept,
                            int* __restrict__ err) {
  __shared__ HashWarpSmem ws[W];
  __shared__ int s_n;
  const int lane = threadIdx.x & 31, wg = threadIdx.x >> 5;
  uint32_t* keys = gtab + (size_t)blockIdx.x * (2 * (size_t)gslots + (size_t)gslots / 2);
  uint32_t* cnts = keys + gslots;
  for (int64_t q = threadIdx.x; q < gslots; q += W * 32) {
    keys[q] = kEmptySlot;
    cnts[q] = 0;
  }
  if (threadIdx.x == 0) s_n = 0;
  __syncthreads();
  for (int64_t b = blockIdx.x; b < nrows; b += gridDim.x) {
    const int64_t i = rows[b];
    int log_s = 1;
    while (((int64_t)1 << log_s) < 2 * prods[i]) ++log_s;
    topk_hash_row<I, V, W, uint32_t>(i, keys, cnts, log_s, cnts + gslots, &s_n, arp, aci, trp, tci, k, ws, wg, lane,
                                     tkey, tcol, kept, err);
  }
}

// Products per row (sum over its columns c of the transpose's row length) and
// the row's bin; rows without entries keep nothing and take no bin.
template <typename I>
__global__ void topk_bin_kernel(const I* __restrict__ arp, const I* __restrict__ aci, const I* __restrict__ trp,
                                int64_t n, int64_t* __restrict__ prods, int32_t* __restrict__ lists,
                                unsigned long long* __restrict__ counts, unsigned long long* __restrict__ maxp) {
  const int64_t i = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (i >= n) return;
  int64_t p = 0;
  for (int64_t e = (int64_t)arp[i] + lane; e < (int64_t)arp[i + 1]; e += 32) {
    const int64_t c = aci[e];
    p += (int64_t)trp[c + 1] - (int64_t)trp[c];
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) p += __shfl_xor_sync(0xffffffffu, p, o);
  if (lane != 0 || p == 0) return;
  prods[i] = p;
  int bin = 0;
  while (bin < kHashBins - 1 && p > hash_bin_max(bin)) ++bin;
  const unsigned long long pos = atomicAdd(counts + bin, 1ULL);
  lists[(int64_t)bin * n + (int64_t)pos] = (int32_t)i;
  if (bin == kHashBins - 1) atomicMax(maxp, (unsigned long long)p);
}

// Transpose of the pattern with rows in any order: column counts, a scan, and
// a scatter by per-column cursors.
template <typename I>
__global__ void pattern_count_kernel(const I* __restrict__ ci, int64_t nnz, unsigned long long* __restrict__ cnt) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < nnz; e += stride)
    atomicAdd(cnt + (int64_t)ci[e], 1ULL);
}

template <typename I>
__global__ void pattern_scatter_kernel(const I* __restrict__ arp, const I* __restrict__ aci, int64_t n,
                                       unsigned long long* __restrict__ cursor, I* __restrict__ tci) {
  const int64_t i = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (i >= n) return;
  for (int64_t e = (int64_t)arp[i] + lane; e < (int64_t)arp[i + 1]; e += 32)
    tci[atomicAdd(cursor + (int64_t)aci[e], 1ULL)] = (I)i;
}

template <typename I>
__global__ void scan_to_index_kernel(const unsigned long long* __restrict__ a, int64_t m, I* __restrict__ b) {
  const int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (q < m) b[q] = (I)a[q];
}

template <typename I, typename V>
__global__ void topk_write_strided_kernel(const uint64_t* __restrict__ tkey, const I* __restrict__ tcol, int k,
                                          const int64_t* __restrict__ orp, int64_t n, I* __restrict__ out_rp,
                                          I* __restrict__ oci, V* __restrict__ ov) {
  const int64_t i = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (i > n) return;
  if (lane == 0) out_rp[i] = (I)orp[i];
  if (i == n) return;
  const int64_t o = orp[i], m = orp[i + 1] - orp[i];
  if (lane < m) {
    oci[o + lane] = tcol[i * k + lane];
    ov[o + lane] = from_key(tkey[i * k + lane], V(0));
  }
}

Matrix* new_csr(Context* ctx, const Matrix* like, int64_t rows, int64_t cols, int64_t nnz) {
  Matrix* C = new spops_matrix_s();
  C->ctx = ctx;
  C->format = SPOPS_FMT_CSR;
  C->itype = like->itype;
  C->vtype = like->vtype;
  C->rows = rows;
  C->cols = cols;
  C->nnz = nnz;
  return C;
}

// The fused top-k (k <= 32).  *done = false (nothing written) when a row has
// more than 2^29 products: the general path below then runs.
template <typename I, typename V>
spops_status_t topk_fused_t(Context* ctx, Matrix* A, int k, Matrix** out, bool* done) {
  *done = false;
  cudaStream_t st = ctx->stream;
  const int64_t n = A->rows, nnz = A->nnz, nc = A->cols;
  ArenaScope scope(ctx);  // this call's temporaries come from the arena
  PoolBuf cur(ctx), trp(ctx), tci(ctx), prods(ctx), lists(ctx), bins(ctx), skey(ctx), scol(ctx), kept(ctx),
      orp(ctx), tmp(ctx), gtab(ctx);
  // 1. the pattern's transpose, rows in any order
  SPOPS_TRY(cur.alloc((size_t)(nc + 1) * 8));
  SPOPS_TRY(trp.alloc((size_t)(nc + 1) * sizeof(I)));
  SPOPS_TRY(tci.alloc((size_t)std::max<int64_t>(nnz, 1) * sizeof(I)));
  SPOPS_CUDA(cudaMemsetAsync(cur.p, 0, (size_t)(nc + 1) * 8, st));
  if (nnz > 0) {
    pattern_count_kernel<I><<<std::min<unsigned>(grid_for(nnz), 8192u), 256, 0, st>>>(
        A->col.as<I>(), nnz, cur.as<unsigned long long>());
    SPOPS_LAUNCH_CHECK();
  }
  size_t sb = 0;
  SPOPS_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, sb, cur.as<unsigned long long>(), cur.as<unsigned long long>(),
                                           nc + 1, st));
  SPOPS_TRY(tmp.alloc(sb + 256));
  SPOPS_CUDA(cub::DeviceScan::ExclusiveSum(tmp.p, sb, cur.as<unsigned long long>(), cur.as<unsigned long long>(),
                                           nc + 1, st));
  scan_to_index_kernel<I><<<grid_for(nc + 1), 256, 0, st>>>(cur.as<unsigned long long>(), nc + 1, trp.as<I>());
  SPOPS_LAUNCH_CHECK();
  if (n > 0) {
    pattern_scatter_kernel<I><<<grid_for(n * 32), 256, 0, st>>>(A->row.as<I>(), A->col.as<I>(), n,
                                                                cur.as<unsigned long long>(), tci.as<I>());
    SPOPS_LAUNCH_CHECK();
  }
  // 2. products per row and bins
  SPOPS_TRY(prods.alloc((size_t)std::max<int64_t>(n, 1) * 8));
  SPOPS_TRY(lists.alloc((size_t)kHashBins * std::max<int64_t>(n, 1) * 4));
  SPOPS_TRY(bins.alloc((size_t)(kHashBins + 1) * 8));
  SPOPS_CUDA(cudaMemsetAsync(bins.p, 0, (size_t)(kHashBins + 1) * 8, st));
  if (n > 0) {
    topk_bin_kernel<I><<<grid_for(n * 32), 256, 0, st>>>(A->row.as<I>(), A->col.as<I>(), trp.as<I>(), n,
                                                         prods.as<int64_t>(), lists.as<int32_t>(),
                                                         bins.as<unsigned long long>(),
                                                         bins.as<unsigned long long>() + kHashBins);
    SPOPS_LAUNCH_CHECK();
  }
  unsigned long long hb[kHashBins + 1];
  SPOPS_CUDA(cudaMemcpyAsync(hb, bins.p, sizeof(hb), cudaMemcpyDeviceToHost, st));
  SPOPS_CUDA(cudaStreamSynchronize(st));
  const int64_t maxp = (int64_t)hb[kHashBins];
  if (maxp > ((int64_t)1 << 29)) return SPOPS_OK;
  // 3. the best k of every row
  const size_t nk = (size_t)std::max<int64_t>(n * k, 1);
  SPOPS_TRY(skey.alloc(nk * 8));
  SPOPS_TRY(scol.alloc(nk * sizeof(I)));
  SPOPS_TRY(kept.alloc((size_t)(n + 1) * 8));
  SPOPS_TRY(orp.alloc((size_t)(n + 1) * 8));
  SPOPS_CUDA(cudaMemsetAsync(kept.p, 0, (size_t)(n + 1) * 8, st));
  SPOPS_TRY(ctx->ensure_errword());
  int* err = ctx->errword.as<int>();
  const int32_t* L = lists.as<int32_t>();
  auto launch = [&](auto kern, int bin, int warps, int rpb, int log_s) -> spops_status_t {
    const int64_t cnt = (int64_t)hb[bin];
    if (cnt == 0 || k == 0) return SPOPS_OK;  // k = 0 keeps nothing
    const size_t S = (size_t)1 << log_s;
    const size_t smem = (size_t)rpb * (2 * S + S / 4) * 4;  // keys, counts, 16-bit list
    SPOPS_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    int bps = 0;
    SPOPS_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps, kern, warps * rpb * 32, smem));
    const int64_t grid = std::max<int64_t>(
        1, std::min<int64_t>((cnt + rpb - 1) / rpb, (int64_t)ctx->num_sms * std::max(bps, 1)));
    kern<<<(unsigned)grid, warps * rpb * 32, smem, st>>>(
        L + (int64_t)bin * n, cnt, A->row.as<I>(), A->col.as<I>(), trp.as<I>(), tci.as<I>(), k, skey.as<uint64_t>(),
        scol.as<I>(), kept.as<int64_t>(), err);
    SPOPS_LAUNCH_CHECK();
    return SPOPS_OK;
  };
  SPOPS_TRY(launch(topk_hash_kernel<I, V, 1, 4, 8>, 0, 1, 4, 8));
  SPOPS_TRY(launch(topk_hash_kernel<I, V, 1, 4, 10>, 1, 1, 4, 10));
  SPOPS_TRY(launch(topk_hash_kernel<I, V, 4, 1, 12>, 2, 4, 1, 12));
  SPOPS_TRY(launch(topk_hash_kernel<I, V, 8, 1, 14>, 3, 8, 1, 14));
  if (hb[kHashBins - 1] > 0 && k > 0) {
    int log_s = 1;
    while (((int64_t)1 << log_s) < 2 * maxp) ++log_s;
    const int64_t gslots = (int64_t)1 << log_s;
    const int64_t per_block = (2 * gslots + gslots / 2) * 4;
    int64_t grid = std::min<int64_t>((int64_t)hb[kHashBins - 1], 2 * (int64_t)ctx->num_sms);
    grid = std::max<int64_t>(1, std::min<int64_t>(grid, ((int64_t)1 << 29) / per_block));
    SPOPS_TRY(gtab.alloc((size_t)(grid * per_block)));
    topk_hash_global_kernel<I, V, 8><<<(unsigned)grid, 256, 0, st>>>(
        L + (int64_t)(kHashBins - 1) * n, (int64_t)hb[kHashBins - 1], prods.as<int64_t>(), A->row.as<I>(),
        A->col.as<I>(), trp.as<I>(), tci.as<I>(), k, gtab.as<uint32_t>(), gslots, skey.as<uint64_t>(), scol.as<I>(),
        kept.as<int64_t>(), err);
    SPOPS_LAUNCH_CHECK();
  }
  // 4. row offsets of the result and the rows
  SPOPS_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, sb, kept.as<int64_t>(), orp.as<int64_t>(), n + 1, st));
  SPOPS_TRY(tmp.alloc(sb + 256));
  SPOPS_CUDA(cub::DeviceScan::ExclusiveSum(tmp.p, sb, kept.as<int64_t>(), orp.as<int64_t>(), n + 1, st));
  int64_t onnz = 0;
  SPOPS_CUDA(cudaMemcpyAsync(&onnz, orp.as<int64_t>() + n, 8, cudaMemcpyDeviceToHost, st));
  SPOPS_CUDA(cudaStreamSynchronize(st));
  Matrix* C = new_csr(ctx, A, n, n, onnz);
  spops_status_t s = C->row.alloc_cached(ctx, (size_t)(n + 1) * sizeof(I));
  if (s == SPOPS_OK) s = C->col.alloc_cached(ctx, (size_t)std::max<int64_t>(onnz, 1) * sizeof(I));
  if (s == SPOPS_OK) s = C->val.alloc_cached(ctx, (size_t)std::max<int64_t>(onnz, 1) * sizeof(V));
  if (s == SPOPS_OK) {
    topk_write_strided_kernel<I, V><<<grid_for((n + 1) * 32), 256, 0, st>>>(
        skey.as<uint64_t>(), scol.as<I>(), k, orp.as<int64_t>(), n, C->row.as<I>(), C->col.as<I>(), C->val.as<V>());
    if (cudaGetLastError() != cudaSuccess) s = fail(SPOPS_ERR_CUDA, "top-k write launch failed");
  }
  if (s == SPOPS_OK && cudaStreamSynchronize(st) != cudaSuccess) s = fail(SPOPS_ERR_CUDA, "top-k: stream error");
  if (s != SPOPS_OK) {
    C->release_all();
    delete static_cast<spops_matrix_s*>(C);
    return s;
  }
  *out = C;
  *done = true;
  return SPOPS_OK;
}

template <typename I, typename V>
spops_status_t topk_t(Context* ctx, Matrix* A, int64_t top_k, Matrix** out) {
  if (top_k <= 32) {
    bool done = false;
    SPOPS_TRY((topk_fused_t<I, V>(ctx, A, (int)top_k, out, &done)));
    if (done) return SPOPS_OK;
  }
  cudaStream_t st = ctx->stream;
  const int64_t n = A->rows, nnz = A->nnz;
  // 1. binary pattern (A's arrays, values 1) and its transpose
  Matrix* Ab = new_csr(ctx, A, n, A->cols, nnz);
  struct Guard {
    Matrix* m;
    ~Guard() {
      m->release_all();
      delete static_cast<spops_matrix_s*>(m);
    }
  } gb{Ab};
  Ab->row.borrow(A->row.p, A->row.bytes);
  Ab->col.borrow(A->col.p, A->col.bytes);
  SPOPS_TRY(Ab->val.alloc_cached(ctx, (size_t)std::max<int64_t>(nnz, 1) * sizeof(V)));
  if (nnz > 0) {
    fill_kernel<V><<<grid_for(nnz), 256, 0, st>>>(Ab->val.as<V>(), nnz, V(1));
    SPOPS_LAUNCH_CHECK();
  }
  Matrix* At = nullptr;
  SPOPS_TRY(csr_transpose_view(ctx, Ab, &At));
  // 2. intersection counts, one cluster per row, every structural entry kept
  Matrix* Cn = nullptr;
  SPOPS_TRY(rowwise_spgemm(ctx, Ab, At, true, &Cn, nullptr));
  Guard gc{Cn};
  const int64_t cnnz = Cn->nnz;
  // 3. keys and the best k per row by a per-row stable sort
  ArenaScope scope(ctx);  // this call's temporaries come from the arena
  PoolBuf key(ctx), skey(ctx), col(ctx), scol(ctx), diag(ctx), kept(ctx), orp(ctx), tmp(ctx);
  const size_t c1 = (size_t)std::max<int64_t>(cnnz, 1);
  SPOPS_TRY(key.alloc(c1 * 8));
  SPOPS_TRY(skey.alloc(c1 * 8));
  SPOPS_TRY(col.alloc(c1 * sizeof(I)));
  SPOPS_TRY(scol.alloc(c1 * sizeof(I)));
  SPOPS_TRY(diag.alloc((size_t)std::max<int64_t>(n, 1) * 8));
  SPOPS_TRY(kept.alloc((size_t)(n + 1) * 8));
  SPOPS_TRY(orp.alloc((size_t)(n + 1) * 8));
  if (n > 0) {
    jaccard_key_kernel<I, V><<<grid_for(n * 32), 256, 0, st>>>(Cn->row.as<I>(), Cn->col.as<I>(), Cn->val.as<V>(),
                                                               A->row.as<I>(), n, key.as<uint64_t>(), col.as<I>(),
                                                               diag.as<int64_t>());
    SPOPS_LAUNCH_CHECK();
  }
  if (cnnz > 0) {
    size_t tb = 0;
    SPOPS_CUDA(cub::DeviceSegmentedSort::StableSortPairs(nullptr, tb, key.as<uint64_t>(), skey.as<uint64_t>(),
                                                         col.as<I>(), scol.as<I>(), cnnz, n, Cn->row.as<I>(),
                                                         Cn->row.as<I>() + 1, st));
    SPOPS_TRY(tmp.alloc(tb + 256));
    SPOPS_CUDA(cub::DeviceSegmentedSort::StableSortPairs(tmp.p, tb, key.as<uint64_t>(), skey.as<uint64_t>(),
                                                         col.as<I>(), scol.as<I>(), cnnz, n, Cn->row.as<I>(),
                                                         Cn->row.as<I>() + 1, st));
  }
  kept_kernel<I><<<grid_for(n + 1), 256, 0, st>>>(Cn->row.as<I>(), diag.as<int64_t>(), n, top_k, kept.as<int64_t>());
  SPOPS_LAUNCH_CHECK();
  size_t sb = 0;
  SPOPS_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, sb, kept.as<int64_t>(), orp.as<int64_t>(), n + 1, st));
  SPOPS_TRY(tmp.alloc(sb + 256));
  SPOPS_CUDA(cub::DeviceScan::ExclusiveSum(tmp.p, sb, kept.as<int64_t>(), orp.as<int64_t>(), n + 1, st));
  int64_t onnz = 0;
  SPOPS_CUDA(cudaMemcpyAsync(&onnz, orp.as<int64_t>() + n, 8, cudaMemcpyDeviceToHost, st));
  SPOPS_CUDA(cudaStreamSynchronize(st));
  Matrix* C = new_csr(ctx, A, n, n, onnz);
  spops_status_t s = C->row.alloc((size_t)(n + 1) * sizeof(I));
  if (s == SPOPS_OK) s = C->col.alloc((size_t)std::max<int64_t>(onnz, 1) * sizeof(I));
  if (s == SPOPS_OK) s = C->val.alloc((size_t)std::max<int64_t>(onnz, 1) * sizeof(V));
  if (s == SPOPS_OK) {
    topk_write_kernel<I, V><<<grid_for((n + 1) * 32), 256, 0, st>>>(
        Cn->row.as<I>(), skey.as<uint64_t>(), scol.as<I>(), orp.as<int64_t>(), n, C->row.as<I>(), C->col.as<I>(),
        C->val.as<V>());
    if (cudaGetLastError() != cudaSuccess) s = fail(SPOPS_ERR_CUDA, "top-k write launch failed");
  }
  if (s == SPOPS_OK && cudaStreamSynchronize(st) != cudaSuccess) s = fail(SPOPS_ERR_CUDA, "top-k: stream error");
  if (s != SPOPS_OK) {
    C->release_all();
    delete static_cast<spops_matrix_s*>(C);
    return s;
  }
  *out = C;
  return SPOPS_OK;
}

}  // namespace

spops_status_t rowwise_spgemm(Context* ctx, Matrix* A, Matrix* B, bool sort_output, Matrix** C, SpgemmStats* st) {
  std::vector<int64_t> perm((size_t)A->rows), offs((size_t)A->rows + 1);
  std::iota(perm.begin(), perm.end(), (int64_t)0);
  std::iota(offs.begin(), offs.end(), (int64_t)0);
  SpgemmStats local;
  return cluster_spgemm(ctx, A, B, perm.data(), offs.data(), A->rows, sort_output, 0.0, C, st ? st : &local, true);
}

spops_status_t topk_spgemm(Context* ctx, Matrix* A, int64_t top_k, Matrix** C) {
  if (A->format != SPOPS_FMT_CSR) return fail(SPOPS_ERR_INVALID, "top-k SpGEMM needs a CSR matrix");
  if (top_k < 0) return fail(SPOPS_ERR_INVALID, "top-k SpGEMM: top_k < 0");
  if (A->cols > INT32_MAX || A->rows > INT32_MAX)
    return fail(SPOPS_ERR_UNSUPPORTED, "top-k SpGEMM: more than 2^31 rows or columns");
  if (!A->plan.ready) SPOPS_TRY(csr_analyse(ctx, A));
  const bool i32 = A->itype == SPOPS_INDEX_I32, f64 = A->vtype == SPOPS_VALUE_F64;
  if (i32 && f64) return topk_t<int32_t, double>(ctx, A, top_k, C);
  if (i32) return topk_t<int32_t, float>(ctx, A, top_k, C);
  if (f64) return topk_t<int64_t, double>(ctx, A, top_k, C);
  return topk_t<int64_t, float>(ctx, A, top_k, C);
}

}  // namespace spops

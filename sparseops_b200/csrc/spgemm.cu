// Locality-enhanced cluster-wise SpGEMM C = A*B on the device.
//
// Replaces the kernel-3 ("mixed accumulator") path of LeSpGEMM_VLength
// (reference src/spgemm.cpp:544-680, src/spgemm_Vlength_mixed.cpp) together
// with the conversions around it in the reference's driver
// (test/test_spgemm_hc_lsh.cpp:230-300): csr_reorder_rows
// (include/sparse_conversion.h:1878), csr_to_vlength_cluster (1640),
// vlength_cluster2csr (1777) and the inverse reorder.
//
// Pipeline (rows of A grouped by the clustering's permutation / offsets):
//   1. clusters   entries of the reordered rows keyed by (cluster, column),
//                 one stable radix sort, unique keys -> each cluster's column
//                 list ASCENDING, values [columns x csz] column-major by row
//                 in the cluster (the reference's CSR_VlengthCluster layout;
//                 it orders a cluster's columns by hash-map iteration instead).
//   2. flops      per cluster sum of nnz(B row) over its columns; clusters
//                 binned by the size of their accumulator.
//   3. symbolic   per cluster (one thread block) a hash set of B columns in
//                 shared memory (global memory for the largest bin): number
//                 of distinct output columns nz, and min/max column.
//   4. classify   dense iff B_access + (max-min+1)*csz*8 <= L2 budget and
//                 nz/(max-min+1) >= 0.15 (src/spgemm_Vlength_mixed.cpp:267-319);
//                 only used for the reference's drop rule below.
//   5. numeric    per cluster: the hash set again, its keys sorted (bitonic,
//                 in shared memory) into the output column list, each key's
//                 position stored beside it; then for every cluster column j
//                 in ascending order and every entry b_jc of B's row j, the
//                 csz products a_j[l]*b_jc are added to acc[pos(c)][l].  Within
//                 one j the columns c are distinct, so no two threads touch the
//                 same slot, and j advances behind a barrier: the summation
//                 order is fixed (deterministic).  A column whose csz values
//                 are all below 1e-12 in magnitude is zeroed when the cluster
//                 is dense or output is sorted -- the reference drops it there
//                 (store_dense_to_output, sort_and_store_table2mat_vlcluster).
//   6. to CSR     entries with value != 0 (vlength_cluster2csr drops exact
//                 zeros), rows back in original order, columns ascending.
#include <cub/cub.cuh>

#include <algorithm>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "spops_internal.h"
#include "spgemm_sort.cuh"

namespace spops {
namespace {

inline unsigned grid_for(int64_t work, int threads = 256) {
  int64_t g = (work + threads - 1) / threads;
  return (unsigned)(g < 1 ? 1 : g);
}

inline int64_t pow2_at_least(int64_t v) {
  int64_t p = 1;
  while (p < v) p <<= 1;
  return p;
}

__device__ __forceinline__ uint32_t hslot(int32_t key, uint32_t mask) {
  return ((uint32_t)key * 2654435761u) & mask;
}

// insert key; returns true if it was not there
__device__ __forceinline__ bool hash_insert(int32_t* tab, uint32_t mask, int32_t key) {
  uint32_t h = hslot(key, mask);
  for (uint32_t probe = 0; probe <= mask; ++probe) {
    const int32_t old = atomicCAS(tab + h, -1, key);
    if (old == -1) return true;
    if (old == key) return false;
    h = (h + 1) & mask;
  }
  return false;  // unreachable: tables hold at least twice the keys
}

__device__ __forceinline__ uint32_t hash_find(const int32_t* tab, uint32_t mask, int32_t key) {
  uint32_t h = hslot(key, mask);
  for (uint32_t probe = 0; probe <= mask; ++probe) {
    if (tab[h] == key) return h;
    h = (h + 1) & mask;
  }
  return 0;  // unreachable: every looked-up key was inserted
}

// ----------------------------------------------------------- reorder + clusters
// bits that hold every value below m (at least 1)
inline int key_bits(int64_t m) {
  int b = 1;
  while (b < 62 && (int64_t(1) << b) < m) ++b;
  return b;
}

template <typename I, typename V>
__global__ void cluster_keys_kernel(const I* __restrict__ rp, const I* __restrict__ ci, const int64_t* __restrict__ perm,
                                    const int64_t* __restrict__ row_cluster, int64_t n, const int64_t* __restrict__ rpr,
                                    int shift, uint64_t* __restrict__ keys, int64_t* __restrict__ src) {
  // warp per reordered row: entries of original row perm[r] in order; key =
  // cluster << shift | column (shift: the bits of A's column count)
  const int64_t r = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (r >= n) return;
  const int64_t orow = perm[r];
  const int64_t s = rp[orow], e = rp[orow + 1], o = rpr[r];
  const uint64_t c = (uint64_t)row_cluster[r];
  for (int64_t k = lane; k < e - s; k += 32) {
    keys[o + k] = (c << shift) | (uint64_t)(uint32_t)ci[s + k];
    src[o + k] = s + k;  // entry of A
  }
}

template <typename I>
__global__ void reordered_len_kernel(const I* __restrict__ rp, const int64_t* __restrict__ perm, int64_t n,
                                     int64_t* __restrict__ len) {
  const int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (r < n) len[r] = (int64_t)rp[perm[r] + 1] - (int64_t)rp[perm[r]];
}

__global__ void row_cluster_kernel(const int64_t* __restrict__ offsets, int64_t ncl, int64_t* __restrict__ row_cluster) {
  const int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (c >= ncl) return;
  for (int64_t r = offsets[c]; r < offsets[c + 1]; ++r) row_cluster[r] = c;
}

__global__ void key_flag_kernel(const uint64_t* __restrict__ keys, int64_t m, int64_t* __restrict__ flag) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i < m) flag[i] = (i == 0 || keys[i] != keys[i - 1]) ? 1 : 0;
}

// per unique key: its cluster's column count, and the column itself
__global__ void cluster_cols_kernel(const uint64_t* __restrict__ keys, const int64_t* __restrict__ flag,
                                    const int64_t* __restrict__ uidx, int64_t m, int shift, int32_t* __restrict__ colids,
                                    unsigned long long* __restrict__ ncols) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= m || !flag[i]) return;
  const int64_t u = uidx[i] - 1;
  colids[u] = (int32_t)(keys[i] & ((1ULL << shift) - 1ULL));
  atomicAdd(ncols + (keys[i] >> shift), 1ULL);
}

template <typename I, typename V>
__global__ void cluster_vals_kernel(const uint64_t* __restrict__ keys, const int64_t* __restrict__ src,
                                    const int64_t* __restrict__ uidx, int64_t m, int shift, const V* __restrict__ av,
                                    const I* __restrict__ rp, const int64_t* __restrict__ perm,
                                    const int64_t* __restrict__ offsets, const int64_t* __restrict__ cptr,
                                    const int64_t* __restrict__ cptr_val, const int64_t* __restrict__ row_of_entry,
                                    V* __restrict__ cvals) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= m) return;
  const int64_t c = (int64_t)(keys[i] >> shift);
  const int64_t u = uidx[i] - 1;
  const int64_t l = row_of_entry[src[i]] - offsets[c];  // row within the cluster
  const int64_t csz = offsets[c + 1] - offsets[c];
  cvals[cptr_val[c] + (u - cptr[c]) * csz + l] = av[src[i]];
}

// reordered position of each entry's row: entry e of original row perm[r] -> r
template <typename I>
__global__ void entry_row_kernel(const I* __restrict__ rp, const int64_t* __restrict__ perm, int64_t n,
                                 int64_t* __restrict__ row_of_entry) {
  const int64_t r = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (r >= n) return;
  const int64_t orow = perm[r];
  for (int64_t k = (int64_t)rp[orow] + lane; k < (int64_t)rp[orow + 1]; k += 32) row_of_entry[k] = r;
}

// ------------------------------------------------------------ flops
template <typename I>
__global__ void cluster_flops_kernel(const int64_t* __restrict__ cptr, const int32_t* __restrict__ colids, int64_t ncl,
                                     const I* __restrict__ brp, int64_t* __restrict__ flops) {
  const int64_t c = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (c >= ncl) return;
  int64_t f = 0;
  for (int64_t j = cptr[c] + lane; j < cptr[c + 1]; j += 32) f += (int64_t)brp[colids[j] + 1] - (int64_t)brp[colids[j]];
  for (int o = 16; o > 0; o >>= 1) f += __shfl_down_sync(0xffffffffu, f, o);
  if (lane == 0) flops[c] = f;
}

// get_spgemm_flop (src/spgemm.cpp:24-42): 2 x sum over A's entries of nnz(B row)
template <typename I>
__global__ void product_count_kernel(const I* __restrict__ aci, int64_t nnz, const I* __restrict__ brp, int64_t brows,
                                     unsigned long long* __restrict__ out) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  unsigned long long s = 0;
  for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < nnz; k += stride) {
    const int64_t c = aci[k];
    if (c < brows) s += (unsigned long long)((int64_t)brp[c + 1] - (int64_t)brp[c]);
  }
  for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) atomicAdd(out, s);
}

// Flat sweep of a cluster's products by a whole block: the cluster's columns
// are taken kSweepCols at a time, their B row lengths scanned in shared
// memory, and every (column, B entry) product of the chunk handed to one
// thread (its column found by binary search), so all B loads of the chunk
// are issued at once whatever the row lengths.  fn(jj, k) gets the column's
// index in the cluster and the B entry.
constexpr int kSweepCols = 256;

struct SweepSmem {
  int64_t off[kSweepCols + 1];  // products before each column of the chunk
  int64_t start[kSweepCols];    // B row start of each column
};

template <typename I, typename F>
__device__ __forceinline__ void block_sweep(const int64_t* __restrict__ cptr, const int32_t* __restrict__ colids,
                                            int64_t c, const I* __restrict__ brp, SweepSmem& sw, F fn) {
  const int64_t j0 = cptr[c], nj = cptr[c + 1] - j0;
  for (int64_t jb = 0; jb < nj; jb += kSweepCols) {
    const int cnt = (int)(nj - jb < kSweepCols ? nj - jb : kSweepCols);
    __syncthreads();  // the previous chunk's readers are done
    if (threadIdx.x == 0) sw.off[0] = 0;
    for (int t = threadIdx.x; t < cnt; t += blockDim.x) {
      const int64_t r = colids[j0 + jb + t];
      sw.start[t] = brp[r];
      sw.off[t + 1] = (int64_t)brp[r + 1] - (int64_t)brp[r];
    }
    __syncthreads();
    if (threadIdx.x < 32) {  // inclusive scan of the lengths by warp 0
      const int lane = threadIdx.x;
      int64_t carry = 0;
      for (int t0 = 0; t0 < cnt; t0 += 32) {
        const int t = t0 + lane;
        int64_t v = t < cnt ? sw.off[t + 1] : 0;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
          const int64_t u = __shfl_up_sync(0xffffffffu, v, o);
          if (lane >= o) v += u;
        }
        if (t < cnt) sw.off[t + 1] = carry + v;
        carry += __shfl_sync(0xffffffffu, v, 31);
      }
    }
    __syncthreads();
    const int64_t total = sw.off[cnt];
    for (int64_t q = threadIdx.x; q < total; q += blockDim.x) {
      int lo = 0, hi = cnt;  // last t with off[t] <= q
      while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (sw.off[mid] <= q) lo = mid; else hi = mid;
      }
      fn(jb + lo, sw.start[lo] + (q - sw.off[lo]));
    }
  }
  __syncthreads();
}

// ------------------------------------------------------------ symbolic
// Block per cluster; table of tsize slots in shared memory, or at
// gtab + goff[b] in global memory when gtab != nullptr.
template <typename I>
__global__ void symbolic_kernel(const int64_t* __restrict__ list, int64_t nlist, const int64_t* __restrict__ tsizes,
                                const int64_t* __restrict__ cptr, const int32_t* __restrict__ colids,
                                const I* __restrict__ brp, const I* __restrict__ bci, int32_t* __restrict__ gtab,
                                const int64_t* __restrict__ goff, int64_t* __restrict__ nz, int64_t* __restrict__ cmin,
                                int64_t* __restrict__ cmax) {
  extern __shared__ __align__(16) unsigned char sm[];
  const int64_t b = blockIdx.x;
  if (b >= nlist) return;
  const int64_t c = list[b];
  const int64_t tsize = tsizes[b];
  int32_t* tab = gtab ? gtab + goff[b] : reinterpret_cast<int32_t*>(sm);
  const uint32_t mask = (uint32_t)(tsize - 1);
  __shared__ unsigned long long s_cnt;
  __shared__ int s_min, s_max;
  if (threadIdx.x == 0) {
    s_cnt = 0;
    s_min = INT32_MAX;
    s_max = -1;
  }
  for (int64_t t = threadIdx.x; t < tsize; t += blockDim.x) tab[t] = -1;
  __shared__ SweepSmem sw;
  unsigned long long cnt = 0;
  int mn = INT32_MAX, mx = -1;
  block_sweep(cptr, colids, c, brp, sw, [&](int64_t, int64_t k) {
    const int32_t key = (int32_t)bci[k];
    if (hash_insert(tab, mask, key)) {
      ++cnt;
      mn = key < mn ? key : mn;
      mx = key > mx ? key : mx;
    }
  });
  atomicAdd(&s_cnt, cnt);
  atomicMin(&s_min, mn);
  atomicMax(&s_max, mx);
  __syncthreads();
  if (threadIdx.x == 0) {
    nz[c] = (int64_t)s_cnt;
    cmin[c] = s_cnt ? s_min : 0;
    cmax[c] = s_cnt ? s_max : 0;
  }
}

// ------------------------------------------------------------ numeric
constexpr int kWideCols = 128;  // A columns per chunk of the wide warp kernel's sweep

struct NumSlot {   // per-cluster arena layout (elements)
  int64_t tsize;   // hash slots
  int64_t lsize;   // sort list length (power of two >= nz)
};

// ------------------------------------------------- warp-per-cluster phases
// Clusters with at most 32 distinct A columns and small tables run one warp
// each, several per block, with the table in the warp's slice of shared
// memory.  All (column j, B entry k) products of the cluster are visited in
// one flat, lane-parallel sweep: lane j holds B row j's start and the
// exclusive prefix of the row lengths, and product t finds its j by a 5-step
// shuffle search -- so every B entry load of the cluster is issued at once
// instead of one B row at a time.
struct WarpRows {
  int64_t start;  // B row start of this lane's column (lane < nj)
  int64_t off;    // products before it
  int64_t total;  // products of the cluster
};

template <typename I>
__device__ __forceinline__ WarpRows warp_rows(const int64_t* __restrict__ cptr, const int32_t* __restrict__ colids,
                                              int64_t c, const I* __restrict__ brp, int lane) {
  const int64_t j0 = cptr[c], nj = cptr[c + 1] - j0;
  int64_t st = 0, len = 0;
  if (lane < nj) {
    const int64_t r = colids[j0 + lane];
    st = brp[r];
    len = (int64_t)brp[r + 1] - st;
  }
  int64_t inc = len;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int64_t u = __shfl_up_sync(0xffffffffu, inc, o);
    if (lane >= o) inc += u;
  }
  return WarpRows{st, inc - len, __shfl_sync(0xffffffffu, inc, 31)};
}

// the column j (0..nj-1) holding flat product t: the largest j with off_j <= t
__device__ __forceinline__ int warp_find_row(const WarpRows& w, int64_t nj, int64_t t) {
  int lo = 0;
#pragma unroll
  for (int step = 16; step > 0; step >>= 1) {
    const int cand = lo + step;
    const int64_t oc = __shfl_sync(0xffffffffu, w.off, cand & 31);
    if (cand < nj && oc <= t) lo = cand;
  }
  return lo;
}

template <typename I>
__global__ void symbolic_warp_kernel(const int64_t* __restrict__ list, int64_t nlist, const int64_t* __restrict__ tsizes,
                                     int64_t warp_tab, const int64_t* __restrict__ cptr,
                                     const int32_t* __restrict__ colids, const I* __restrict__ brp,
                                     const I* __restrict__ bci, int64_t* __restrict__ nz, int64_t* __restrict__ cmin,
                                     int64_t* __restrict__ cmax) {
  extern __shared__ __align__(16) unsigned char sm[];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int64_t b = blockIdx.x * (int64_t)(blockDim.x >> 5) + w;
  if (b >= nlist) return;
  const int64_t c = list[b];
  const int64_t tsize = tsizes[b];
  int32_t* tab = reinterpret_cast<int32_t*>(sm) + (int64_t)w * warp_tab;
  const uint32_t mask = (uint32_t)(tsize - 1);
  for (int64_t t = lane; t < tsize; t += 32) tab[t] = -1;
  __syncwarp();
  const WarpRows wr = warp_rows(cptr, colids, c, brp, lane);
  const int64_t nj = cptr[c + 1] - cptr[c];
  unsigned long long cnt = 0;
  int mn = INT32_MAX, mx = -1;
  for (int64_t base = 0; base < wr.total; base += 32) {
    const int64_t t = base + lane;
    const int j = warp_find_row(wr, nj, t);
    const int64_t st = __shfl_sync(0xffffffffu, wr.start, j), of = __shfl_sync(0xffffffffu, wr.off, j);
    if (t < wr.total) {
      const int32_t key = (int32_t)bci[st + (t - of)];
      if (hash_insert(tab, mask, key)) {
        ++cnt;
        mn = key < mn ? key : mn;
        mx = key > mx ? key : mx;
      }
    }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    cnt += __shfl_down_sync(0xffffffffu, cnt, o);
    mn = min(mn, __shfl_down_sync(0xffffffffu, mn, o));
    mx = max(mx, __shfl_down_sync(0xffffffffu, mx, o));
  }
  if (lane == 0) {
    nz[c] = (int64_t)cnt;
    cmin[c] = cnt ? mn : 0;
    cmax[c] = cnt ? mx : 0;
  }
}

// Numeric phase, one warp per cluster.  Warp arena (bytes at w * warp_bytes):
// tab (int32, tsize) | pos (int32, tsize) | keys (int32, nz) | acc (V, nz*csz).
// Columns are ranked by counting (rank = number of smaller columns), which
// gives the ascending output order and each column's accumulator row.  The
// products are accumulated in flat (j, k) order, 32 at a time; products of one
// sweep that hit the same column are first summed in lane order (= ascending
// j) and added by the lowest lane, so the per-column summation order depends
// only on the matrices.
// The keys of a hash table (slots != -1) compacted into keys[0..n), padded
// with INT32_MAX to lsize (a power of two), and sorted ascending by one warp
// with a bitonic network.
__device__ __forceinline__ void warp_sort_keys(const int32_t* __restrict__ tab, int64_t tsize, int32_t* keys,
                                               int64_t lsize, int lane) {
  int64_t n = 0;
  for (int64_t t0 = 0; t0 < tsize; t0 += 32) {
    const int32_t v = t0 + lane < tsize ? tab[t0 + lane] : -1;
    const unsigned m = __ballot_sync(0xffffffffu, v != -1);
    if (v != -1) keys[n + __popc(m & ((1u << lane) - 1u))] = v;
    n += __popc(m);
  }
  for (int64_t t = n + lane; t < lsize; t += 32) keys[t] = INT32_MAX;
  __syncwarp();
  // one compare-exchange pair per lane and step: pair q of stage (kk, jj) is
  // (i, i + jj) with i = q with a zero bit inserted at jj
  const int64_t half = lsize >> 1;
  for (int64_t kk = 2; kk <= lsize; kk <<= 1) {
    for (int64_t jj = kk >> 1; jj > 0; jj >>= 1) {
      for (int64_t q = lane; q < half; q += 32) {
        const int64_t i = ((q & ~(jj - 1)) << 1) | (q & (jj - 1));
        const int64_t ixj = i + jj;
        const bool up = (i & kk) == 0;
        const int32_t a = keys[i], d = keys[ixj];
        if ((a > d) == up) {
          keys[i] = d;
          keys[ixj] = a;
        }
      }
      __syncwarp();
    }
  }
}

template <typename I, typename V>
__global__ void numeric_warp_kernel(const int64_t* __restrict__ list, int64_t nlist, const NumSlot* __restrict__ slots,
                                    int64_t warp_bytes, const int64_t* __restrict__ cptr,
                                    const int64_t* __restrict__ cptr_val, const int32_t* __restrict__ colids,
                                    const V* __restrict__ avals, const int64_t* __restrict__ offsets,
                                    const I* __restrict__ brp, const I* __restrict__ bci, const V* __restrict__ bv,
                                    const int64_t* __restrict__ nz, const int64_t* __restrict__ soff,
                                    const int64_t* __restrict__ soff_val, const unsigned char* __restrict__ drop_small,
                                    int32_t* __restrict__ ccol, V* __restrict__ cval) {
  extern __shared__ __align__(16) unsigned char sm[];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int64_t b = blockIdx.x * (int64_t)(blockDim.x >> 5) + w;
  if (b >= nlist) return;
  const int64_t c = list[b];
  const NumSlot S = slots[b];
  const int64_t nzc = nz[c];
  const int64_t csz = offsets[c + 1] - offsets[c];
  unsigned char* base = sm + (int64_t)w * warp_bytes;
  int32_t* tab = reinterpret_cast<int32_t*>(base);
  int32_t* pos = tab + S.tsize;
  int32_t* keys = pos + S.tsize;
  V* acc = reinterpret_cast<V*>(base + ((4 * (2 * S.tsize + S.lsize) + 15) & ~15LL));
  const uint32_t mask = (uint32_t)(S.tsize - 1);
  for (int64_t t = lane; t < S.tsize; t += 32) tab[t] = -1;
  for (int64_t t = lane; t < nzc * csz; t += 32) acc[t] = V(0);
  __syncwarp();
  const WarpRows wr = warp_rows(cptr, colids, c, brp, lane);
  const int64_t j0 = cptr[c], nj = cptr[c + 1] - j0;
  // 1. distinct columns
  for (int64_t b0 = 0; b0 < wr.total; b0 += 32) {
    const int64_t t = b0 + lane;
    const int j = warp_find_row(wr, nj, t);
    const int64_t st = __shfl_sync(0xffffffffu, wr.start, j), of = __shfl_sync(0xffffffffu, wr.off, j);
    if (t < wr.total) hash_insert(tab, mask, (int32_t)bci[st + (t - of)]);
  }
  __syncwarp();
  // 2. compact (slot order), pad to lsize, 3. bitonic sort; positions and
  //    the output column list in ascending order
  warp_sort_keys(tab, S.tsize, keys, S.lsize, lane);
  const int64_t co = soff[c], cvo = soff_val[c];
  for (int64_t p = lane; p < nzc; p += 32) {
    pos[hash_find(tab, mask, keys[p])] = (int32_t)p;
    ccol[co + p] = keys[p];
  }
  __syncwarp();
  // 4. accumulate in flat (j, k) order
  const int64_t vbase = cptr_val[c];
  for (int64_t b0 = 0; b0 < wr.total; b0 += 32) {
    const int64_t t = b0 + lane;
    const int j = warp_find_row(wr, nj, t);
    const int64_t st = __shfl_sync(0xffffffffu, wr.start, j), of = __shfl_sync(0xffffffffu, wr.off, j);
    const bool valid = t < wr.total;
    int32_t p = -1 - lane;  // distinct for idle lanes
    V bval = V(0);
    if (valid) {
      const int64_t k = st + (t - of);
      p = pos[hash_find(tab, mask, (int32_t)bci[k])];
      bval = bv[k];
    }
    const unsigned grp = __match_any_sync(0xffffffffu, p);
    const int leader = __ffs(grp) - 1;
    for (int64_t l = 0; l < csz; ++l) {
      const V v = valid ? avals[vbase + (int64_t)j * csz + l] * bval : V(0);
      V sum = v;
      if (grp != (1u << lane)) {  // several products of this sweep hit the column: sum in lane order
        sum = V(0);
        for (unsigned m = grp; m; m &= m - 1) sum += __shfl_sync(grp, v, __ffs(m) - 1);
      }
      if (valid && lane == leader) acc[p * csz + l] += sum;
    }
    __syncwarp();
  }
  // 5. drop rule and output (values in rank order, rows of the cluster interleaved)
  const bool drop = drop_small[c] != 0;
  for (int64_t p = lane; p < nzc; p += 32) {
    bool small = drop;
    if (drop)
      for (int64_t l = 0; l < csz; ++l)
        if (fabs((double)acc[p * csz + l]) >= 1e-12) {
          small = false;
          break;
        }
    for (int64_t l = 0; l < csz; ++l) cval[cvo + p * csz + l] = small ? V(0) : acc[p * csz + l];
  }
}


// Numeric phase, one warp per cluster with any number of A columns (the
// clusters beyond numeric_warp_kernel's 32 columns / 512 outputs whose arena
// fits the warp's slice of shared memory).  Warp arena (bytes at w * bytes):
// tab (int32, tsize) | pos (int32, tsize) | keys (int32, lsize) | offsets
// (int64, kWideCols + 1) | starts (int64, kWideCols) | acc (V, nz*csz).  The
// products are swept in flat (j, k) order kWideCols columns at a time, 32 per
// step (a lane finds its column by binary search in the chunk's offsets); the
// output columns are sorted by a bitonic network; products of one step that
// hit the same column are summed in lane order and added by the lowest lane,
// so the summation order depends only on the matrices.
template <typename I, typename V>
__global__ void numeric_warp_wide_kernel(const int64_t* __restrict__ list, int64_t nlist,
                                         const NumSlot* __restrict__ slots, int64_t warp_bytes,
                                         const int64_t* __restrict__ cptr, const int64_t* __restrict__ cptr_val,
                                         const int32_t* __restrict__ colids, const V* __restrict__ avals,
                                         const int64_t* __restrict__ offsets, const I* __restrict__ brp,
                                         const I* __restrict__ bci, const V* __restrict__ bv,
                                         const int64_t* __restrict__ nz, const int64_t* __restrict__ soff,
                                         const int64_t* __restrict__ soff_val,
                                         const unsigned char* __restrict__ drop_small, int32_t* __restrict__ ccol,
                                         V* __restrict__ cval) {
  extern __shared__ __align__(16) unsigned char sm[];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int64_t b = blockIdx.x * (int64_t)(blockDim.x >> 5) + w;
  if (b >= nlist) return;
  const int64_t c = list[b];
  const NumSlot S = slots[b];
  const int64_t nzc = nz[c];
  const int64_t csz = offsets[c + 1] - offsets[c];
  unsigned char* base = sm + (int64_t)w * warp_bytes;
  int32_t* tab = reinterpret_cast<int32_t*>(base);
  int32_t* pos = tab + S.tsize;
  int32_t* keys = pos + S.tsize;
  int64_t* coff = reinterpret_cast<int64_t*>(base + ((4 * (2 * S.tsize + S.lsize) + 15) & ~15LL));
  int64_t* cstart = coff + kWideCols + 1;
  V* acc = reinterpret_cast<V*>(cstart + kWideCols);
  const uint32_t mask = (uint32_t)(S.tsize - 1);
  for (int64_t t = lane; t < S.tsize; t += 32) tab[t] = -1;
  for (int64_t t = lane; t < nzc * csz; t += 32) acc[t] = V(0);
  const int64_t j0 = cptr[c], nj = cptr[c + 1] - j0;
  // fn(jj, k, valid) for every product in flat order, 32 per call, all lanes
  auto sweep = [&](auto fn) {
    for (int64_t jb = 0; jb < nj; jb += kWideCols) {
      const int cnt = (int)(nj - jb < kWideCols ? nj - jb : kWideCols);
      __syncwarp();
      int64_t carry = 0;
      for (int t0 = 0; t0 < cnt; t0 += 32) {
        const int t = t0 + lane;
        int64_t len = 0;
        if (t < cnt) {
          const int64_t r = colids[j0 + jb + t];
          cstart[t] = brp[r];
          len = (int64_t)brp[r + 1] - (int64_t)brp[r];
        }
        int64_t inc = len;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
          const int64_t u = __shfl_up_sync(0xffffffffu, inc, o);
          if (lane >= o) inc += u;
        }
        if (t < cnt) coff[t + 1] = carry + inc;
        carry += __shfl_sync(0xffffffffu, inc, 31);
      }
      if (lane == 0) coff[0] = 0;
      __syncwarp();
      const int64_t total = coff[cnt];
      for (int64_t q0 = 0; q0 < total; q0 += 32) {
        const int64_t q = q0 + lane;
        int lo = 0;
        int64_t k = 0;
        if (q < total) {
          int hi = cnt;
          while (hi - lo > 1) {
            const int mid = (lo + hi) >> 1;
            if (coff[mid] <= q) lo = mid; else hi = mid;
          }
          k = cstart[lo] + (q - coff[lo]);
        }
        fn(jb + lo, k, q < total);
      }
    }
    __syncwarp();
  };
  // 1. distinct columns
  sweep([&](int64_t, int64_t k, bool valid) {
    if (valid) hash_insert(tab, mask, (int32_t)bci[k]);
  });
  // 2. compact (slot order), pad to lsize, bitonic sort ascending
  warp_sort_keys(tab, S.tsize, keys, S.lsize, lane);
  // 3. position of every column; the output column list
  const int64_t co = soff[c], cvo = soff_val[c];
  for (int64_t p = lane; p < nzc; p += 32) {
    pos[hash_find(tab, mask, keys[p])] = (int32_t)p;
    ccol[co + p] = keys[p];
  }
  __syncwarp();
  // 4. accumulate in flat (j, k) order
  const int64_t vbase = cptr_val[c];
  sweep([&](int64_t jj, int64_t k, bool valid) {
    int32_t p = -1 - lane;  // distinct for idle lanes
    V bval = V(0);
    if (valid) {
      p = pos[hash_find(tab, mask, (int32_t)bci[k])];
      bval = bv[k];
    }
    const unsigned grp = __match_any_sync(0xffffffffu, p);
    const int leader = __ffs(grp) - 1;
    for (int64_t l = 0; l < csz; ++l) {
      const V v = valid ? avals[vbase + jj * csz + l] * bval : V(0);
      V sum = v;
      if (grp != (1u << lane)) {
        sum = V(0);
        for (unsigned m = grp; m; m &= m - 1) sum += __shfl_sync(grp, v, __ffs(m) - 1);
      }
      if (valid && lane == leader) acc[p * csz + l] += sum;
    }
    __syncwarp();
  });
  // 5. drop rule and output
  const bool drop = drop_small[c] != 0;
  for (int64_t p = lane; p < nzc; p += 32) {
    bool small = drop;
    if (drop)
      for (int64_t l = 0; l < csz; ++l)
        if (fabs((double)acc[p * csz + l]) >= 1e-12) {
          small = false;
          break;
        }
    for (int64_t l = 0; l < csz; ++l) cval[cvo + p * csz + l] = small ? V(0) : acc[p * csz + l];
  }
}

template <typename I, typename V>
__global__ void numeric_kernel(const int64_t* __restrict__ list, int64_t nlist, const NumSlot* __restrict__ slots,
                               const int64_t* __restrict__ cptr, const int64_t* __restrict__ cptr_val,
                               const int32_t* __restrict__ colids, const V* __restrict__ avals,
                               const int64_t* __restrict__ offsets, const I* __restrict__ brp,
                               const I* __restrict__ bci, const V* __restrict__ bv, const int64_t* __restrict__ nz,
                               const int64_t* __restrict__ soff, const int64_t* __restrict__ soff_val,
                               const unsigned char* __restrict__ drop_small, unsigned char* __restrict__ garena,
                               const int64_t* __restrict__ goff, int32_t* __restrict__ ccol, V* __restrict__ cval) {
  extern __shared__ __align__(16) unsigned char sm[];
  const int64_t b = blockIdx.x;
  if (b >= nlist) return;
  const int64_t c = list[b];
  const NumSlot S = slots[b];
  const int64_t nzc = nz[c];
  const int64_t csz = offsets[c + 1] - offsets[c];
  unsigned char* base = garena ? garena + goff[b] : sm;
  // arena: acc (V, nz*csz) | tab (int32, tsize) | pos (int32, tsize) | list (int32, lsize)
  V* acc = reinterpret_cast<V*>(base);
  int32_t* tab = reinterpret_cast<int32_t*>(base + ((nzc * csz * (int64_t)sizeof(V) + 15) & ~15LL));
  int32_t* pos = tab + S.tsize;
  int32_t* keys = pos + S.tsize;
  const uint32_t mask = (uint32_t)(S.tsize - 1);
  __shared__ int s_n;
  if (threadIdx.x == 0) s_n = 0;
  __shared__ SweepSmem sw;
  for (int64_t t = threadIdx.x; t < S.tsize; t += blockDim.x) tab[t] = -1;
  for (int64_t t = threadIdx.x; t < nzc * csz; t += blockDim.x) acc[t] = V(0);
  // 1. distinct columns
  block_sweep(cptr, colids, c, brp, sw, [&](int64_t, int64_t k) { hash_insert(tab, mask, (int32_t)bci[k]); });
  // 2. compact and sort them ascending
  for (int64_t t = threadIdx.x; t < S.tsize; t += blockDim.x)
    if (tab[t] != -1) keys[atomicAdd(&s_n, 1)] = tab[t];
  __syncthreads();
  for (int64_t t = s_n + threadIdx.x; t < S.lsize; t += blockDim.x) keys[t] = INT32_MAX;
  __syncthreads();
  for (int64_t kk = 2; kk <= S.lsize; kk <<= 1) {
    for (int64_t jj = kk >> 1; jj > 0; jj >>= 1) {
      for (int64_t i = threadIdx.x; i < S.lsize; i += blockDim.x) {
        const int64_t ixj = i ^ jj;
        if (ixj > i) {
          const bool up = (i & kk) == 0;
          const int32_t a = keys[i], d = keys[ixj];
          if ((a > d) == up) {
            keys[i] = d;
            keys[ixj] = a;
          }
        }
      }
      __syncthreads();
    }
  }
  // 3. position of every column
  for (int64_t p = threadIdx.x; p < nzc; p += blockDim.x) pos[hash_find(tab, mask, keys[p])] = (int32_t)p;
  __syncthreads();
  // 4. accumulate: columns j of the cluster in ascending order; within one j
  //    the (entry, row) items touch distinct slots
  const int64_t vbase = cptr_val[c];
  for (int64_t j = cptr[c]; j < cptr[c + 1]; ++j) {
    const int64_t r = colids[j];
    const int64_t k0 = brp[r], len = (int64_t)brp[r + 1] - k0;
    const V* aj = avals + vbase + (j - cptr[c]) * csz;
    for (int64_t t = threadIdx.x; t < len * csz; t += blockDim.x) {
      const int64_t k = k0 + t / csz, l = t % csz;
      const V a = aj[l];
      if (a != V(0)) {  // distinct slots within one j unless B repeats a column in a row
        const int32_t p = pos[hash_find(tab, mask, (int32_t)bci[k])];
        atomicAdd(acc + p * csz + l, a * bv[k]);
      }
    }
    __syncthreads();
  }
  // 5. drop rule and output
  const bool drop = drop_small[c] != 0;
  const int64_t co = soff[c], cvo = soff_val[c];
  for (int64_t p = threadIdx.x; p < nzc; p += blockDim.x) {
    ccol[co + p] = keys[p];
    bool small = drop;
    if (drop)
      for (int64_t l = 0; l < csz; ++l)
        if (fabs((double)acc[p * csz + l]) >= 1e-12) { small = false; break; }
    for (int64_t l = 0; l < csz; ++l) cval[cvo + p * csz + l] = small ? V(0) : acc[p * csz + l];
  }
}

__global__ void classify_kernel(const int64_t* __restrict__ cptr, const int64_t* __restrict__ offsets,
                                const int64_t* __restrict__ nz, const int64_t* __restrict__ cmin,
                                const int64_t* __restrict__ cmax, int64_t ncl, double b_rowdense, double budget,
                                bool sort_output, size_t vbytes, size_t ibytes,
                                const unsigned char* __restrict__ settled, unsigned char* __restrict__ drop,
                                unsigned long long* __restrict__ ndense) {
  const int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (c >= ncl || settled[c]) return;  // the sort path classified it
  bool dense = false;
  if (nz[c] > 0) {
    const int64_t range = cmax[c] - cmin[c] + 1;
    const double density = (double)nz[c] / (double)range;
    const size_t b_access = (size_t)((double)(cptr[c + 1] - cptr[c]) * b_rowdense * (double)(ibytes + vbytes));
    const size_t dense_bytes = (size_t)range * (size_t)(offsets[c + 1] - offsets[c]) * vbytes;
    dense = (double)(b_access + dense_bytes) <= budget && density >= 0.15;
  }
  if (dense) atomicAdd(ndense, 1ULL);
  drop[c] = (dense || sort_output) ? 1 : 0;
}

// ------------------------------------------------------------ to CSR
template <typename V>
__global__ void row_count_kernel(const int64_t* __restrict__ soff_val, const int64_t* __restrict__ nz,
                                 const int64_t* __restrict__ offsets, const int64_t* __restrict__ perm, int64_t ncl,
                                 const V* __restrict__ cval, bool keep_zeros, int64_t* __restrict__ rowcnt) {
  // warp per cluster, lanes over its rows (csz <= 32 common) and columns
  const int64_t c = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (c >= ncl) return;
  const int64_t csz = offsets[c + 1] - offsets[c];
  const int64_t ncol = nz[c];
  for (int64_t l = 0; l < csz; ++l) {
    int64_t cnt = 0;
    for (int64_t p = lane; p < ncol; p += 32) cnt += (keep_zeros || cval[soff_val[c] + p * csz + l] != V(0)) ? 1 : 0;
    for (int o = 16; o > 0; o >>= 1) cnt += __shfl_down_sync(0xffffffffu, cnt, o);
    if (lane == 0) rowcnt[perm[offsets[c] + l]] = cnt;
  }
}

template <typename I, typename V>
__global__ void row_write_kernel(const int64_t* __restrict__ soff, const int64_t* __restrict__ soff_val,
                                 const int64_t* __restrict__ nz, const int64_t* __restrict__ offsets,
                                 const int64_t* __restrict__ perm, int64_t ncl, const int32_t* __restrict__ ccol,
                                 const V* __restrict__ cval, bool keep_zeros, const int64_t* __restrict__ crp,
                                 I* __restrict__ oci, V* __restrict__ ov) {
  const int64_t c = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (c >= ncl) return;
  const int64_t csz = offsets[c + 1] - offsets[c];
  const int64_t ncol = nz[c];
  for (int64_t l = 0; l < csz; ++l) {
    int64_t o = crp[perm[offsets[c] + l]];
    for (int64_t p0 = 0; p0 < ncol; p0 += 32) {
      const int64_t p = p0 + lane;
      const V v = p < ncol ? cval[soff_val[c] + p * csz + l] : V(0);
      const bool keep = p < ncol && (keep_zeros || v != V(0));
      const unsigned m = __ballot_sync(0xffffffffu, keep);
      if (keep) {
        const int64_t at = o + __popc(m & ((1u << lane) - 1));
        oci[at] = (I)ccol[soff[c] + p];
        ov[at] = v;
      }
      o += __popc(m);
    }
  }
}

// ------------------------------------------------------------ binning
// Clusters are grouped by the kernel shape that serves them: a key per
// cluster (0..kBins-1, kNoBin to skip), one stable radix sort of (key,
// cluster) so each bin lists its clusters in ascending order, and the bin
// boundaries found by binary search in the sorted keys.  Only the
// boundaries come back to the host.
constexpr uint32_t kNoBin = 15;

__device__ __forceinline__ int64_t pow2_ceil(int64_t v) {
  return v <= 1 ? 1 : (int64_t)1 << (64 - __clzll((unsigned long long)(v - 1)));
}

__global__ void weight_kernel(const int64_t* __restrict__ cnt, const int64_t* __restrict__ offsets, int64_t ncl,
                              int64_t* __restrict__ weighted) {
  const int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (c < ncl) weighted[c] = cnt[c] * (offsets[c + 1] - offsets[c]);
}

// symbolic: table >= 2 * min(flops, cols) slots; 0 warp, 1 / 2 block in
// shared memory (smem0 / smem1 bytes), 3 block in global memory
__global__ void sym_bin_kernel(const int64_t* __restrict__ flops, const int64_t* __restrict__ cnt, int64_t ncl,
                               int64_t bcols, int64_t warp_tab, int64_t smem0, int64_t smem1,
                               const unsigned char* __restrict__ settled, uint32_t* __restrict__ key,
                               int64_t* __restrict__ ids, int64_t* __restrict__ tsz) {
  const int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (c >= ncl) return;
  if (settled[c]) {  // the sort path counts its own columns
    key[c] = kNoBin;
    ids[c] = c;
    tsz[c] = 0;
    return;
  }
  const int64_t f = flops[c] < bcols ? flops[c] : bcols;
  const int64_t ts = pow2_ceil(2 * f > 2 ? 2 * f : 2);
  uint32_t b;
  if (cnt[c] <= 32 && ts <= warp_tab) b = 0;
  else if (ts * 4 <= smem0) b = 1;
  else if (ts * 4 <= smem1) b = 2;
  else b = 3;
  key[c] = b;
  ids[c] = c;
  tsz[c] = ts;
}

// numeric: 0 / 1 warp arenas of wbytes[0] / [1] (at most 32 A columns and 512
// output columns); 2 / 3 / 4 wide-warp arenas of wbytes[2] / [3] / [4]; 5 / 6
// block arenas in wbytes[5] / [6] of shared memory; 7 block arena in global
// memory
struct NumBinLimits {
  int64_t wbytes[7];
};

__global__ void num_bin_kernel(const int64_t* __restrict__ nz, const int64_t* __restrict__ cnt,
                               const int64_t* __restrict__ offsets, int64_t ncl, int64_t vsize, NumBinLimits lim,
                               const unsigned char* __restrict__ settled, uint32_t* __restrict__ key,
                               int64_t* __restrict__ ids) {
  const int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (c >= ncl) return;
  ids[c] = c;
  const int64_t z = nz[c];
  if (z == 0 || settled[c]) {
    key[c] = kNoBin;
    return;
  }
  const int64_t csz = offsets[c + 1] - offsets[c];
  const int64_t tsize = pow2_ceil(2 * z > 2 ? 2 * z : 2), lsize = pow2_ceil(z);
  const int64_t accb = z * csz * vsize;
  if (cnt[c] <= 32 && z <= 512) {
    const int64_t wb = ((4 * (2 * tsize + lsize) + 15) & ~15LL) + accb;
    if (wb <= lim.wbytes[0]) { key[c] = 0; return; }
    if (wb <= lim.wbytes[1]) { key[c] = 1; return; }
  }
  const int64_t wide = ((4 * (2 * tsize + lsize) + 15) & ~15LL) + 8 * (2 * kWideCols + 1) + accb;
  for (uint32_t b = 2; b <= 4; ++b)
    if (wide <= lim.wbytes[b]) { key[c] = b; return; }
  const int64_t bytes = ((accb + 15) & ~15LL) + 4 * (2 * tsize + lsize);
  key[c] = bytes <= lim.wbytes[5] ? 5 : (bytes <= lim.wbytes[6] ? 6 : 7);
}

// sort path (spgemm_sort.cuh): bin q (R = 2^q keys per lane, q = 0..6)
// for a cluster with at most 32 * 2^q products and kSortCols columns whose
// output columns fit the key beside the product index; settled[c] = 1 then.
// bins 0-4: one warp, 2^q keys per lane (sort_accum_kernel); bins 5-8: 2^(q-4)
// warps of 16 keys per lane (sort_accum_multi_kernel); bin q holds P <= 32 << q
constexpr int kSortBins = 9;
constexpr int kSortOneWarpBins = 5;

__global__ void sort_bin_kernel(const int64_t* __restrict__ flops, const int64_t* __restrict__ cptr, int64_t ncl,
                                int64_t bcols, unsigned char* __restrict__ settled, uint32_t* __restrict__ key,
                                int64_t* __restrict__ ids) {
  const int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (c >= ncl) return;
  ids[c] = c;
  const int64_t P = flops[c], nj = cptr[c + 1] - cptr[c];
  uint32_t b = kNoBin;
  for (int q = 0; q < kSortBins; ++q) {
    if (P <= (32LL << q)) {
      const int tbits = 5 + q;
      const int64_t max_cols = q < kSortOneWarpBins ? kSortCols : kMultiCols;
      if (nj <= max_cols && bcols <= (1LL << (32 - tbits)) - 1) b = (uint32_t)q;
      break;
    }
  }
  key[c] = b;
  settled[c] = b != kNoBin ? 1 : 0;
}

// room in each cluster's output slab: its product count on the sort path (at
// most 32 * 2^8, and never below its distinct columns whatever B holds), the
// symbolic count otherwise; values: that times the cluster size
__global__ void slab_cap_kernel(const int64_t* __restrict__ flops, const int64_t* __restrict__ nz,
                                const unsigned char* __restrict__ settled, const int64_t* __restrict__ offsets,
                                int64_t ncl, int64_t* __restrict__ cap, int64_t* __restrict__ capv) {
  const int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (c > ncl) return;
  if (c == ncl) {  // the scans' last slot
    cap[c] = 0;
    capv[c] = 0;
    return;
  }
  const int64_t m = settled[c] ? flops[c] : nz[c];
  cap[c] = m;
  capv[c] = m * (offsets[c + 1] - offsets[c]);
}

__global__ void bin_bounds_kernel(const uint32_t* __restrict__ skey, int64_t ncl, int nb, int64_t* __restrict__ start) {
  const int b = threadIdx.x;
  if (b > nb) return;
  int64_t lo = 0, hi = ncl;  // first position with key >= b
  while (lo < hi) {
    const int64_t mid = (lo + hi) >> 1;
    if (skey[mid] < (uint32_t)b) lo = mid + 1; else hi = mid;
  }
  start[b] = lo;
}

// per listed cluster: symbolic table size (and its global-arena size)
__global__ void sym_list_kernel(const int64_t* __restrict__ sids, const int64_t* __restrict__ tsz, int64_t m,
                                int64_t* __restrict__ ltsz) {
  const int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (p < m) ltsz[p] = tsz[sids[p]];
}

// per listed cluster: numeric slots and arena bytes (256-aligned)
__global__ void num_list_kernel(const int64_t* __restrict__ sids, const int64_t* __restrict__ nz,
                                const int64_t* __restrict__ offsets, int64_t m, int64_t vsize,
                                NumSlot* __restrict__ slots, int64_t* __restrict__ gbytes) {
  const int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (p >= m) return;
  const int64_t c = sids[p], z = nz[c];
  const int64_t csz = offsets[c + 1] - offsets[c];
  NumSlot S;
  S.tsize = pow2_ceil(2 * z > 2 ? 2 * z : 2);
  S.lsize = pow2_ceil(z > 1 ? z : 1);
  slots[p] = S;
  const int64_t bytes = ((z * csz * vsize + 15) & ~15LL) + 4 * (2 * S.tsize + S.lsize);
  gbytes[p] = (bytes + 255) & ~255LL;
}

__global__ void to_i32_kernel(const int64_t* __restrict__ a, int64_t m, int32_t* __restrict__ b) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i < m) b[i] = (int32_t)a[i];
}

template <typename T>
spops_status_t d2h(cudaStream_t st, std::vector<T>& h, const void* d, size_t n) {
  h.resize(n);
  if (n) {
    SPOPS_CUDA(cudaMemcpyAsync(h.data(), d, n * sizeof(T), cudaMemcpyDeviceToHost, st));
    SPOPS_CUDA(cudaStreamSynchronize(st));
  }
  return SPOPS_OK;
}

template <typename T>
spops_status_t h2d(cudaStream_t st, PoolBuf& d, const std::vector<T>& h) {
  SPOPS_TRY(d.alloc(std::max<size_t>(h.size(), 1) * sizeof(T)));
  if (!h.empty()) SPOPS_CUDA(cudaMemcpyAsync(d.p, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice, st));
  return SPOPS_OK;
}

struct Timer {
  std::chrono::steady_clock::time_point t = std::chrono::steady_clock::now();
  double lap(cudaStream_t st) {
    cudaStreamSynchronize(st);
    const auto n = std::chrono::steady_clock::now();
    const double ms = std::chrono::duration<double, std::milli>(n - t).count();
    t = n;
    return ms;
  }
};

// rowwise: the row-wise kernels' output rules (every structural entry kept,
// exact zeros included; no small-value drop) instead of kernel 3's.
// ---- clustered (VLength) form
template <typename T, typename U>
__global__ void cast_kernel(const T* __restrict__ a, int64_t m, U* __restrict__ b) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i < m) b[i] = (U)a[i];
}

__global__ void iota_kernel(int64_t* __restrict__ a, int64_t m) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i < m) a[i] = i;
}

// Columns of C's clusters that stay in the clustered form: every column,
// except in clusters under the drop rule (dense and sorted paths), where a
// column whose values all came out as exactly 0 was dropped.  One warp per
// cluster; kcnt[c] = kept columns.
template <typename V>
__global__ void cl_keep_count_kernel(const int64_t* __restrict__ soff_val, const int64_t* __restrict__ nz,
                                     const int64_t* __restrict__ offs, int64_t ncl, const V* __restrict__ cval,
                                     const unsigned char* __restrict__ drop, int64_t* __restrict__ kcnt,
                                     int64_t* __restrict__ kval) {
  const int64_t c = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (c >= ncl) return;
  const int64_t csz = offs[c + 1] - offs[c], np = nz[c], v0 = soff_val[c];
  const bool dr = drop[c] != 0;
  int64_t kept = 0;
  for (int64_t p = lane; p < np; p += 32) {
    bool keep = !dr;
    for (int64_t l = 0; l < csz && !keep; ++l) keep = cval[v0 + p * csz + l] != V(0);
    kept += keep;
  }
  for (int o = 16; o; o >>= 1) kept += __shfl_xor_sync(0xffffffffu, kept, o);
  if (lane == 0) {
    kcnt[c] = kept;
    kval[c] = kept * csz;
  }
}

template <typename I, typename V>
__global__ void cl_compact_kernel(const int64_t* __restrict__ soff, const int64_t* __restrict__ soff_val,
                                  const int64_t* __restrict__ nz, const int64_t* __restrict__ offs, int64_t ncl,
                                  const int32_t* __restrict__ ccol,
                                  const V* __restrict__ cval, const unsigned char* __restrict__ drop,
                                  const int64_t* __restrict__ nrp, const int64_t* __restrict__ nrpv,
                                  I* __restrict__ colids, V* __restrict__ vals) {
  const int64_t c = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (c >= ncl) return;
  const int64_t csz = offs[c + 1] - offs[c], p0 = soff[c], np = nz[c], v0 = soff_val[c];
  const bool dr = drop[c] != 0;
  int64_t out = 0;  // kept columns before this batch
  for (int64_t b = 0; b < np; b += 32) {
    const int64_t p = b + lane;
    bool keep = false;
    if (p < np) {
      keep = !dr;
      for (int64_t l = 0; l < csz && !keep; ++l) keep = cval[v0 + p * csz + l] != V(0);
    }
    const unsigned m = __ballot_sync(0xffffffffu, keep);
    if (keep) {
      const int64_t q = out + __popc(m & ((1u << lane) - 1u));
      colids[nrp[c] + q] = (I)ccol[p0 + p];
      for (int64_t l = 0; l < csz; ++l) vals[nrpv[c] + q * csz + l] = cval[v0 + p * csz + l];
    }
    out += __popc(m);
  }
}

// Clustered form back to CSR rows in cluster order (vlength_cluster2csr):
// row off[c] + l holds, in the cluster's column order, the columns whose
// value for row l is not exactly 0.  One thread per (cluster, row).
template <typename I, typename V>
__global__ void vlc_row_count_kernel(const I* __restrict__ rp, const I* __restrict__ rpv,
                                     const int64_t* __restrict__ off, int64_t ncl, const int64_t* __restrict__ rowcl,
                                     int64_t n, const V* __restrict__ val, int64_t* __restrict__ cnt) {
  const int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (r >= n) return;
  const int64_t c = rowcl[r], l = r - off[c], csz = off[c + 1] - off[c];
  const int64_t p0 = (int64_t)rp[c], np = (int64_t)rp[c + 1] - p0, v0 = (int64_t)rpv[c];
  int64_t k = 0;
  for (int64_t p = 0; p < np; ++p) k += val[v0 + p * csz + l] != V(0);
  cnt[r] = k;
}

template <typename I, typename V>
__global__ void vlc_row_write_kernel(const I* __restrict__ rp, const I* __restrict__ rpv, const I* __restrict__ colids,
                                     const int64_t* __restrict__ off, const int64_t* __restrict__ rowcl, int64_t n,
                                     const V* __restrict__ val, const int64_t* __restrict__ crp, I* __restrict__ ci,
                                     V* __restrict__ cv) {
  const int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (r >= n) return;
  const int64_t c = rowcl[r], l = r - off[c], csz = off[c + 1] - off[c];
  const int64_t p0 = (int64_t)rp[c], np = (int64_t)rp[c + 1] - p0, v0 = (int64_t)rpv[c];
  int64_t o = crp[r];
  for (int64_t p = 0; p < np; ++p) {
    const V v = val[v0 + p * csz + l];
    if (v != V(0)) {
      ci[o] = colids[p0 + p];
      cv[o] = v;
      ++o;
    }
  }
}

// A clustered-form handle's arrays from int64 / int32 device arrays.
template <typename I, typename V>
spops_status_t make_vlcluster(Context* ctx, int64_t rows, int64_t cols, int64_t ncl, const int64_t* offs_d,
                              const int64_t* rptr, const int32_t* colids, int64_t nnzc, const int64_t* rptr_val,
                              const V* vals, int64_t nnzv, spops_index_t itype, Matrix** out) {
  cudaStream_t st = ctx->stream;
  Matrix* M = new spops_matrix_s();
  M->ctx = ctx;
  M->format = SPOPS_FMT_VLCLUSTER;
  M->itype = itype;
  M->vtype = sizeof(V) == 8 ? SPOPS_VALUE_F64 : SPOPS_VALUE_F32;
  M->rows = rows;
  M->cols = cols;
  M->nnz = nnzc;
  M->clusters = ncl;
  M->cl_nnzv = nnzv;
  spops_status_t s = M->row.alloc((size_t)(ncl + 1) * sizeof(I));
  if (s == SPOPS_OK) s = M->cl_rpv.alloc((size_t)(ncl + 1) * sizeof(I));
  if (s == SPOPS_OK) s = M->col.alloc((size_t)std::max<int64_t>(nnzc, 1) * sizeof(I));
  if (s == SPOPS_OK) s = M->val.alloc((size_t)std::max<int64_t>(nnzv, 1) * sizeof(V));
  if (s == SPOPS_OK) {
    cast_kernel<int64_t, I><<<grid_for(ncl + 1), 256, 0, st>>>(rptr, ncl + 1, M->row.as<I>());
    cast_kernel<int64_t, I><<<grid_for(ncl + 1), 256, 0, st>>>(rptr_val, ncl + 1, M->cl_rpv.as<I>());
    if (nnzc > 0) cast_kernel<int32_t, I><<<grid_for(nnzc), 256, 0, st>>>(colids, nnzc, M->col.as<I>());
    if (nnzv > 0)
      if (cudaMemcpyAsync(M->val.p, vals, (size_t)nnzv * sizeof(V), cudaMemcpyDeviceToDevice, st) != cudaSuccess)
        s = fail(SPOPS_ERR_CUDA, "clustered form: copy failed");
    if (cudaGetLastError() != cudaSuccess) s = fail(SPOPS_ERR_CUDA, "clustered form: launch failed");
  }
  std::vector<int64_t> off_h((size_t)ncl + 1);
  if (s == SPOPS_OK &&
      cudaMemcpyAsync(off_h.data(), offs_d, (size_t)(ncl + 1) * 8, cudaMemcpyDeviceToHost, st) != cudaSuccess)
    s = fail(SPOPS_ERR_CUDA, "clustered form: copy failed");
  if (s == SPOPS_OK && cudaStreamSynchronize(st) != cudaSuccess) s = fail(SPOPS_ERR_CUDA, "clustered form: stream");
  if (s == SPOPS_OK) s = vlcluster_finish(ctx, M, off_h.data());
  if (s != SPOPS_OK) {
    M->release_all();
    delete static_cast<spops_matrix_s*>(M);
    return s;
  }
  *out = M;
  return SPOPS_OK;
}

template <typename I, typename V>
spops_status_t spgemm_t(Context* ctx, Matrix* A, Matrix* B, const int64_t* perm_h, const int64_t* offs_h, int64_t ncl,
                        bool sort_output, double l2_budget, bool rowwise, Matrix** out, SpgemmStats* stats,
                        bool cluster_out) {
  cudaStream_t st = ctx->stream;
  const int64_t n = A->rows, nnz = A->nnz;
  Timer tm;
  Trace tr("spgemm");
  // --- permutation, offsets, per-row cluster
  ArenaScope scope(ctx);  // this call's temporaries come from the arena
  PoolBuf perm(ctx), offs(ctx), rowcl(ctx), rlen(ctx), rpr(ctx), keys(ctx), skeys(ctx), src(ctx), ssrc(ctx), flag(ctx), uidx(ctx), colids(ctx), ncols_u(ctx), cptr(ctx), cptr_val(ctx), avals(ctx), row_of_entry(ctx), tmp(ctx);
  SPOPS_TRY(perm.alloc((size_t)std::max<int64_t>(n, 1) * 8));
  SPOPS_TRY(offs.alloc((size_t)(ncl + 1) * 8));
  // host or device arrays (the device clustering hands over device ones)
  SPOPS_CUDA(cudaMemcpyAsync(perm.p, perm_h, (size_t)n * 8, cudaMemcpyDefault, st));
  SPOPS_CUDA(cudaMemcpyAsync(offs.p, offs_h, (size_t)(ncl + 1) * 8, cudaMemcpyDefault, st));
  const size_t nn = (size_t)std::max<int64_t>(n, 1), nz1 = (size_t)std::max<int64_t>(nnz, 1);
  SPOPS_TRY(rowcl.alloc(nn * 8));
  SPOPS_TRY(rlen.alloc(nn * 8));
  SPOPS_TRY(rpr.alloc((nn + 1) * 8));
  if (ncl > 0) row_cluster_kernel<<<grid_for(ncl), 256, 0, st>>>(offs.as<int64_t>(), ncl, rowcl.as<int64_t>());
  if (n > 0) reordered_len_kernel<I><<<grid_for(n), 256, 0, st>>>(A->row.as<I>(), perm.as<int64_t>(), n, rlen.as<int64_t>());
  SPOPS_LAUNCH_CHECK();
  size_t cb = 0;
  SPOPS_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, cb, rlen.as<int64_t>(), rpr.as<int64_t>(), (int64_t)nn, st));
  SPOPS_TRY(tmp.alloc(cb + 256));
  SPOPS_CUDA(cub::DeviceScan::ExclusiveSum(tmp.p, cb, rlen.as<int64_t>(), rpr.as<int64_t>(), (int64_t)n, st));
  tr.mark(st, "setup + reordered row scan");
  // --- cluster keys, sort, unique
  SPOPS_TRY(keys.alloc(nz1 * 8));
  SPOPS_TRY(skeys.alloc(nz1 * 8));
  SPOPS_TRY(src.alloc(nz1 * 8));
  SPOPS_TRY(ssrc.alloc(nz1 * 8));
  SPOPS_TRY(flag.alloc(nz1 * 8));
  SPOPS_TRY(uidx.alloc(nz1 * 8));
  SPOPS_TRY(row_of_entry.alloc(nz1 * 8));
  tr.mark(st, "alloc key arrays");
  if (tr.on && ctx->pool) {  // the pool's reserved and used bytes, for the trace
    unsigned long long rsv = 0, used = 0;
    cudaMemPoolGetAttribute(ctx->pool, cudaMemPoolAttrReservedMemCurrent, &rsv);
    cudaMemPoolGetAttribute(ctx->pool, cudaMemPoolAttrUsedMemCurrent, &used);
    std::fprintf(stderr, "[spgemm] pool reserved %.1f MB, used %.1f MB\n", rsv / 1e6, used / 1e6);
  }
  // key = cluster << kshift | column: sort only the bits in use
  const int kshift = key_bits(A->cols), kend = std::min(64, kshift + key_bits(ncl));
  if (n > 0) {
    cluster_keys_kernel<I, V><<<grid_for(n * 32), 256, 0, st>>>(A->row.as<I>(), A->col.as<I>(), perm.as<int64_t>(),
                                                                rowcl.as<int64_t>(), n, rpr.as<int64_t>(), kshift,
                                                                keys.as<uint64_t>(), src.as<int64_t>());
    entry_row_kernel<I><<<grid_for(n * 32), 256, 0, st>>>(A->row.as<I>(), perm.as<int64_t>(), n,
                                                          row_of_entry.as<int64_t>());
    SPOPS_LAUNCH_CHECK();
  }
  int64_t nnzc = 0;
  SPOPS_TRY(ncols_u.alloc((size_t)(ncl + 1) * 8));
  SPOPS_CUDA(cudaMemsetAsync(ncols_u.p, 0, (size_t)(ncl + 1) * 8, st));
  if (nnz > 0) {
    size_t c1 = 0, c2 = 0;
    SPOPS_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, c1, keys.as<uint64_t>(), skeys.as<uint64_t>(), src.as<int64_t>(),
                                               ssrc.as<int64_t>(), nnz, 0, kend, st));
    SPOPS_CUDA(cub::DeviceScan::InclusiveSum(nullptr, c2, flag.as<int64_t>(), uidx.as<int64_t>(), nnz, st));
    SPOPS_TRY(tmp.alloc(std::max(c1, c2) + 256));
    SPOPS_CUDA(cub::DeviceRadixSort::SortPairs(tmp.p, c1, keys.as<uint64_t>(), skeys.as<uint64_t>(), src.as<int64_t>(),
                                               ssrc.as<int64_t>(), nnz, 0, kend, st));
    key_flag_kernel<<<grid_for(nnz), 256, 0, st>>>(skeys.as<uint64_t>(), nnz, flag.as<int64_t>());
    SPOPS_LAUNCH_CHECK();
    SPOPS_CUDA(cub::DeviceScan::InclusiveSum(tmp.p, c2, flag.as<int64_t>(), uidx.as<int64_t>(), nnz, st));
    SPOPS_CUDA(cudaMemcpyAsync(&nnzc, uidx.as<int64_t>() + nnz - 1, 8, cudaMemcpyDeviceToHost, st));
    SPOPS_CUDA(cudaStreamSynchronize(st));
  }
  tr.mark(st, "keys + sort + unique");
  SPOPS_TRY(colids.alloc((size_t)std::max<int64_t>(nnzc, 1) * 4));
  if (nnz > 0) {
    cluster_cols_kernel<<<grid_for(nnz), 256, 0, st>>>(skeys.as<uint64_t>(), flag.as<int64_t>(), uidx.as<int64_t>(),
                                                       nnz, kshift, colids.as<int32_t>(),
                                                       reinterpret_cast<unsigned long long*>(ncols_u.p));
    SPOPS_LAUNCH_CHECK();
  }
  // cluster column pointers: exclusive scans of the column counts, plain and
  // weighted by the cluster size (ncols_u[ncl] and cw[ncl] are zero)
  PoolBuf cw(ctx), tot(ctx);
  SPOPS_TRY(cptr.alloc((size_t)(ncl + 1) * 8));
  SPOPS_TRY(cptr_val.alloc((size_t)(ncl + 1) * 8));
  SPOPS_TRY(cw.alloc((size_t)(ncl + 1) * 8));
  SPOPS_TRY(tot.alloc(64));
  SPOPS_CUDA(cudaMemsetAsync(cw.p, 0, (size_t)(ncl + 1) * 8, st));
  const int64_t* cnt_d = reinterpret_cast<const int64_t*>(ncols_u.p);
  if (ncl > 0) {
    weight_kernel<<<grid_for(ncl), 256, 0, st>>>(cnt_d, offs.as<int64_t>(), ncl, cw.as<int64_t>());
    SPOPS_LAUNCH_CHECK();
  }
  {
    size_t c1 = 0, c2 = 0;
    SPOPS_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, c1, cnt_d, cptr.as<int64_t>(), ncl + 1, st));
    SPOPS_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, c2, cw.as<int64_t>(), cptr_val.as<int64_t>(), ncl + 1, st));
    SPOPS_TRY(tmp.alloc(std::max(c1, c2) + 256));
    SPOPS_CUDA(cub::DeviceScan::ExclusiveSum(tmp.p, c1, cnt_d, cptr.as<int64_t>(), ncl + 1, st));
    SPOPS_CUDA(cub::DeviceScan::ExclusiveSum(tmp.p, c2, cw.as<int64_t>(), cptr_val.as<int64_t>(), ncl + 1, st));
  }
  int64_t nnzv = 0;
  SPOPS_CUDA(cudaMemcpyAsync(&nnzv, cptr_val.as<int64_t>() + ncl, 8, cudaMemcpyDeviceToHost, st));
  SPOPS_CUDA(cudaStreamSynchronize(st));
  tr.mark(st, "cluster pointers");
  SPOPS_TRY(avals.alloc((size_t)std::max<int64_t>(nnzv, 1) * sizeof(V)));
  SPOPS_CUDA(cudaMemsetAsync(avals.p, 0, avals.bytes, st));
  if (nnz > 0) {
    cluster_vals_kernel<I, V><<<grid_for(nnz), 256, 0, st>>>(
        skeys.as<uint64_t>(), ssrc.as<int64_t>(), uidx.as<int64_t>(), nnz, kshift, A->val.as<V>(), A->row.as<I>(),
        perm.as<int64_t>(), offs.as<int64_t>(), cptr.as<int64_t>(), cptr_val.as<int64_t>(),
        row_of_entry.as<int64_t>(), avals.as<V>());
    SPOPS_LAUNCH_CHECK();
  }
  keys.release(); skeys.release(); src.release(); ssrc.release(); flag.release(); uidx.release();
  row_of_entry.release(); rlen.release(); rpr.release(); rowcl.release();
  if (stats) stats->cluster_ms = tm.lap(st);
  tr.mark(st, "cluster values + frees");

  // --- flops per cluster
  PoolBuf flops(ctx), nzd(ctx), cmin(ctx), cmax(ctx);
  SPOPS_TRY(flops.alloc((size_t)std::max<int64_t>(ncl, 1) * 8));
  SPOPS_TRY(nzd.alloc((size_t)(ncl + 1) * 8));
  SPOPS_TRY(cmin.alloc((size_t)std::max<int64_t>(ncl, 1) * 8));
  SPOPS_TRY(cmax.alloc((size_t)std::max<int64_t>(ncl, 1) * 8));
  SPOPS_CUDA(cudaMemsetAsync(nzd.p, 0, (size_t)(ncl + 1) * 8, st));
  if (ncl > 0) {
    cluster_flops_kernel<I><<<grid_for(ncl * 32), 256, 0, st>>>(cptr.as<int64_t>(), colids.as<int32_t>(), ncl,
                                                                B->row.as<I>(), flops.as<int64_t>());
    SPOPS_LAUNCH_CHECK();
  }
  int64_t total_products = 0;
  {
    SPOPS_CUDA(cudaMemsetAsync(tot.p, 0, 8, st));
    if (nnz > 0) {
      product_count_kernel<I><<<std::min<unsigned>(grid_for(nnz), 4096u), 256, 0, st>>>(
          A->col.as<I>(), nnz, B->row.as<I>(), B->rows, reinterpret_cast<unsigned long long*>(tot.p));
      SPOPS_LAUNCH_CHECK();
    }
    SPOPS_CUDA(cudaMemcpyAsync(&total_products, tot.p, 8, cudaMemcpyDeviceToHost, st));
  }
  // the hash-table kernels want the largest shared-memory split of each SM
  SPOPS_CUDA(cudaFuncSetAttribute(numeric_warp_kernel<I, V>, cudaFuncAttributePreferredSharedMemoryCarveout, 100));
  SPOPS_CUDA(cudaFuncSetAttribute(numeric_warp_wide_kernel<I, V>, cudaFuncAttributePreferredSharedMemoryCarveout, 100));
  SPOPS_CUDA(cudaFuncSetAttribute(numeric_kernel<I, V>, cudaFuncAttributePreferredSharedMemoryCarveout, 100));
  SPOPS_CUDA(cudaFuncSetAttribute(symbolic_warp_kernel<I>, cudaFuncAttributePreferredSharedMemoryCarveout, 100));
  SPOPS_CUDA(cudaFuncSetAttribute(symbolic_kernel<I>, cudaFuncAttributePreferredSharedMemoryCarveout, 100));
  // sort (bin key, cluster) pairs; bounds of the nb bins to the host
  PoolBuf bkey(ctx), bkey_s(ctx), bid(ctx), bid_s(ctx), bstart(ctx);
  const size_t ncl1 = (size_t)std::max<int64_t>(ncl, 1);
  SPOPS_TRY(bkey.alloc(ncl1 * 4));
  SPOPS_TRY(bkey_s.alloc(ncl1 * 4));
  SPOPS_TRY(bid.alloc(ncl1 * 8));
  SPOPS_TRY(bid_s.alloc(ncl1 * 8));
  SPOPS_TRY(bstart.alloc(64 * 8));
  auto sort_bins = [&](int nb, std::vector<int64_t>& start) -> spops_status_t {
    start.assign((size_t)nb + 1, 0);
    if (ncl == 0) return SPOPS_OK;
    size_t cb2 = 0;
    SPOPS_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, cb2, bkey.as<uint32_t>(), bkey_s.as<uint32_t>(),
                                               bid.as<int64_t>(), bid_s.as<int64_t>(), ncl, 0, 4, st));
    SPOPS_TRY(tmp.alloc(cb2 + 256));
    SPOPS_CUDA(cub::DeviceRadixSort::SortPairs(tmp.p, cb2, bkey.as<uint32_t>(), bkey_s.as<uint32_t>(),
                                               bid.as<int64_t>(), bid_s.as<int64_t>(), ncl, 0, 4, st));
    bin_bounds_kernel<<<1, 32, 0, st>>>(bkey_s.as<uint32_t>(), ncl, nb, bstart.as<int64_t>());
    SPOPS_LAUNCH_CHECK();
    SPOPS_CUDA(cudaMemcpyAsync(start.data(), bstart.p, ((size_t)nb + 1) * 8, cudaMemcpyDeviceToHost, st));
    SPOPS_CUDA(cudaStreamSynchronize(st));
    return SPOPS_OK;
  };
  // exclusive scan of sizes[from, to) into offs_out[from, to); returns the total
  auto seg_scan = [&](int64_t* sizes, int64_t* offs_out, int64_t from, int64_t to, int64_t* total) -> spops_status_t {
    *total = 0;
    if (to <= from) return SPOPS_OK;
    size_t cb2 = 0;
    SPOPS_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, cb2, sizes + from, offs_out + from, to - from, st));
    SPOPS_TRY(tmp.alloc(cb2 + 256));
    SPOPS_CUDA(cub::DeviceScan::ExclusiveSum(tmp.p, cb2, sizes + from, offs_out + from, to - from, st));
    int64_t last[2] = {0, 0};
    SPOPS_CUDA(cudaMemcpyAsync(&last[0], offs_out + to - 1, 8, cudaMemcpyDeviceToHost, st));
    SPOPS_CUDA(cudaMemcpyAsync(&last[1], sizes + to - 1, 8, cudaMemcpyDeviceToHost, st));
    SPOPS_CUDA(cudaStreamSynchronize(st));
    *total = last[0] + last[1];
    return SPOPS_OK;
  };
  tr.mark(st, "flops per cluster");

  // --- sort path: which clusters the one-warp sort-accumulate kernels take
  // (their list kept apart: the bin buffers are reused below)
  const int64_t bcols = B->cols;
  PoolBuf settled(ctx), slist(ctx);
  SPOPS_TRY(settled.alloc(ncl1));
  SPOPS_CUDA(cudaMemsetAsync(settled.p, 0, ncl1, st));
  std::vector<int64_t> tstart((size_t)kSortBins + 1, 0);
  if (ncl > 0) {
    sort_bin_kernel<<<grid_for(ncl), 256, 0, st>>>(flops.as<int64_t>(), cptr.as<int64_t>(), ncl, bcols,
                                                  settled.as<unsigned char>(), bkey.as<uint32_t>(),
                                                  bid.as<int64_t>());
    SPOPS_LAUNCH_CHECK();
    SPOPS_TRY(sort_bins(kSortBins, tstart));
  }
  const int64_t nsorted = tstart[kSortBins];
  SPOPS_TRY(slist.alloc((size_t)std::max<int64_t>(nsorted, 1) * 8));
  if (nsorted > 0)
    SPOPS_CUDA(cudaMemcpyAsync(slist.p, bid_s.p, (size_t)nsorted * 8, cudaMemcpyDeviceToDevice, st));
  tr.mark(st, "sort-path bins");

  // --- symbolic for the other clusters: 0 warp per cluster (<= 32 A
  // columns, table <= kSymWarpTab), 1 / 2 block with the table in 16 KB /
  // 128 KB of shared memory, 3 global
  constexpr int kSymWarps = 8;
  constexpr int64_t kSymWarpTab = 2048;
  const int sym_threads[4] = {32 * kSymWarps, 32, 256, 256};
  const size_t sym_smem[4] = {(size_t)kSymWarps * kSymWarpTab * 4, 16 << 10, 128 << 10, 0};
  PoolBuf tszc(ctx), ltsz(ctx), sgoff(ctx), gtab(ctx);
  SPOPS_TRY(tszc.alloc(ncl1 * 8));
  SPOPS_TRY(ltsz.alloc(ncl1 * 8));
  SPOPS_TRY(sgoff.alloc(ncl1 * 8));
  std::vector<int64_t> sstart(5, 0);
  if (ncl > nsorted) {
    sym_bin_kernel<<<grid_for(ncl), 256, 0, st>>>(flops.as<int64_t>(), cnt_d, ncl, bcols, kSymWarpTab,
                                                 (int64_t)sym_smem[1], (int64_t)sym_smem[2],
                                                 settled.as<unsigned char>(), bkey.as<uint32_t>(), bid.as<int64_t>(),
                                                 tszc.as<int64_t>());
    SPOPS_LAUNCH_CHECK();
    SPOPS_TRY(sort_bins(4, sstart));
    sym_list_kernel<<<grid_for(ncl), 256, 0, st>>>(bid_s.as<int64_t>(), tszc.as<int64_t>(), ncl, ltsz.as<int64_t>());
    SPOPS_LAUNCH_CHECK();
  }
  int64_t gsym = 0;
  SPOPS_TRY(seg_scan(ltsz.as<int64_t>(), sgoff.as<int64_t>(), sstart[3], sstart[4], &gsym));
  if (gsym) SPOPS_TRY(gtab.alloc((size_t)gsym * 4));
  tr.mark(st, "symbolic bins");
  for (int w = 0; w < 4; ++w) {
    const int64_t m = sstart[w + 1] - sstart[w];
    if (m <= 0) continue;
    const int64_t* dl = bid_s.as<int64_t>() + sstart[w];
    const int64_t* dt = ltsz.as<int64_t>() + sstart[w];
    if (w == 0) {
      SPOPS_CUDA(cudaFuncSetAttribute(symbolic_warp_kernel<I>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)sym_smem[0]));
      symbolic_warp_kernel<I><<<(unsigned)((m + kSymWarps - 1) / kSymWarps), sym_threads[0], sym_smem[0], st>>>(
          dl, m, dt, kSymWarpTab, cptr.as<int64_t>(), colids.as<int32_t>(), B->row.as<I>(), B->col.as<I>(),
          nzd.as<int64_t>(), cmin.as<int64_t>(), cmax.as<int64_t>());
    } else {
      const bool global = w == 3;
      if (sym_smem[w] > 48 * 1024)
        SPOPS_CUDA(cudaFuncSetAttribute(symbolic_kernel<I>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        (int)sym_smem[w]));
      symbolic_kernel<I><<<(unsigned)m, sym_threads[w], sym_smem[w], st>>>(
          dl, m, dt, cptr.as<int64_t>(), colids.as<int32_t>(), B->row.as<I>(), B->col.as<I>(),
          global ? gtab.as<int32_t>() : nullptr, global ? sgoff.as<int64_t>() + sstart[3] : nullptr,
          nzd.as<int64_t>(), cmin.as<int64_t>(), cmax.as<int64_t>());
    }
    SPOPS_LAUNCH_CHECK();
  }
  gtab.release();
  // output slabs: per cluster room for its columns (exact for the hash
  // path, its product count for the sort path) and values
  PoolBuf soff(ctx), soff_val(ctx), ccol(ctx), cval(ctx);
  SPOPS_TRY(soff.alloc((size_t)(ncl + 1) * 8));
  SPOPS_TRY(soff_val.alloc((size_t)(ncl + 1) * 8));
  PoolBuf capc(ctx), capv(ctx);
  SPOPS_TRY(capc.alloc((size_t)(ncl + 1) * 8));
  SPOPS_TRY(capv.alloc((size_t)(ncl + 1) * 8));
  slab_cap_kernel<<<grid_for(ncl + 1), 256, 0, st>>>(flops.as<int64_t>(), nzd.as<int64_t>(),
                                                     settled.as<unsigned char>(), offs.as<int64_t>(), ncl,
                                                     capc.as<int64_t>(), capv.as<int64_t>());
  SPOPS_LAUNCH_CHECK();
  int64_t slab_cols = 0, slab_vals = 0;
  {
    size_t c1 = 0, c2 = 0;
    SPOPS_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, c1, capc.as<int64_t>(), soff.as<int64_t>(), ncl + 1, st));
    SPOPS_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, c2, capv.as<int64_t>(), soff_val.as<int64_t>(), ncl + 1, st));
    SPOPS_TRY(tmp.alloc(std::max(c1, c2) + 256));
    SPOPS_CUDA(cub::DeviceScan::ExclusiveSum(tmp.p, c1, capc.as<int64_t>(), soff.as<int64_t>(), ncl + 1, st));
    SPOPS_CUDA(cub::DeviceScan::ExclusiveSum(tmp.p, c2, capv.as<int64_t>(), soff_val.as<int64_t>(), ncl + 1, st));
    SPOPS_CUDA(cudaMemcpyAsync(&slab_cols, soff.as<int64_t>() + ncl, 8, cudaMemcpyDeviceToHost, st));
    SPOPS_CUDA(cudaMemcpyAsync(&slab_vals, soff_val.as<int64_t>() + ncl, 8, cudaMemcpyDeviceToHost, st));
    SPOPS_CUDA(cudaStreamSynchronize(st));
  }
  capc.release();
  capv.release();
  SPOPS_TRY(ccol.alloc((size_t)std::max<int64_t>(slab_cols, 1) * 4));
  SPOPS_TRY(cval.alloc((size_t)std::max<int64_t>(slab_vals, 1) * sizeof(V)));
  if (stats) stats->symbolic_ms = tm.lap(st);
  tr.mark(st, "symbolic kernels + slab offsets");

  // --- sort path: columns, classification and values in one pass
  PoolBuf drop(ctx), ndense(ctx);
  SPOPS_TRY(drop.alloc(ncl1));
  SPOPS_TRY(ndense.alloc(8));
  SPOPS_CUDA(cudaMemsetAsync(ndense.p, 0, 8, st));
  if (rowwise) SPOPS_CUDA(cudaMemsetAsync(drop.p, 0, ncl1, st));
  const double b_rowdense = (double)B->nnz / (double)std::max<int64_t>(B->rows, 1);
  for (int q = 0; q < kSortBins; ++q) {
    const int64_t m = tstart[q + 1] - tstart[q];
    if (m <= 0) continue;
    const unsigned grid = (unsigned)((m + kSortWarps - 1) / kSortWarps);
    const int64_t* dl = slist.as<int64_t>() + tstart[q];
    const int tbits = 5 + q;
#define SPOPS_SORT_LAUNCH(RR)                                                                                    \
  /* static + dynamic shared memory can pass 48 KB: raise the limit */                                         \
  SPOPS_CUDA(cudaFuncSetAttribute(sort_accum_kernel<I, V, RR>, cudaFuncAttributeMaxDynamicSharedMemorySize,       \
                                  (int)sort_accum_smem<V, RR>()));                                                \
  sort_accum_kernel<I, V, RR><<<grid, 32 * kSortWarps, sort_accum_smem<V, RR>(), st>>>(                         \
      dl, m, cptr.as<int64_t>(), cptr_val.as<int64_t>(), colids.as<int32_t>(), avals.as<V>(), offs.as<int64_t>(), \
      B->row.as<I>(), B->col.as<I>(), B->val.as<V>(), tbits, b_rowdense, l2_budget, sort_output, rowwise,        \
      soff.as<int64_t>(), soff_val.as<int64_t>(), nzd.as<int64_t>(), cmin.as<int64_t>(), cmax.as<int64_t>(),      \
      drop.as<unsigned char>(), reinterpret_cast<unsigned long long*>(ndense.p), ccol.as<int32_t>(), cval.as<V>())
#define SPOPS_MULTI_LAUNCH(WW)                                                                                    \
  SPOPS_CUDA(cudaFuncSetAttribute(sort_accum_multi_kernel<I, V, WW>, cudaFuncAttributeMaxDynamicSharedMemorySize, \
                                  (int)sort_multi_smem<V, WW>()));                                                \
  sort_accum_multi_kernel<I, V, WW><<<(unsigned)m, 32 * WW, sort_multi_smem<V, WW>(), st>>>(                     \
      dl, m, cptr.as<int64_t>(), cptr_val.as<int64_t>(), colids.as<int32_t>(), avals.as<V>(), offs.as<int64_t>(), \
      B->row.as<I>(), B->col.as<I>(), B->val.as<V>(), tbits, b_rowdense, l2_budget, sort_output, rowwise,        \
      soff.as<int64_t>(), soff_val.as<int64_t>(), nzd.as<int64_t>(), cmin.as<int64_t>(), cmax.as<int64_t>(),      \
      drop.as<unsigned char>(), reinterpret_cast<unsigned long long*>(ndense.p), ccol.as<int32_t>(), cval.as<V>())
    switch (q) {
      case 0: SPOPS_SORT_LAUNCH(1); break;
      case 1: SPOPS_SORT_LAUNCH(2); break;
      case 2: SPOPS_SORT_LAUNCH(4); break;
      case 3: SPOPS_SORT_LAUNCH(8); break;
      case 4: SPOPS_SORT_LAUNCH(16); break;
      case 5: SPOPS_MULTI_LAUNCH(2); break;
      case 6: SPOPS_MULTI_LAUNCH(4); break;
      case 7: SPOPS_MULTI_LAUNCH(8); break;
      default: SPOPS_MULTI_LAUNCH(16); break;
    }
#undef SPOPS_SORT_LAUNCH
#undef SPOPS_MULTI_LAUNCH
    SPOPS_LAUNCH_CHECK();
  }
  tr.mark(st, "sort-path kernels");

  // --- classify the other clusters (drop rule)
  if (!rowwise && ncl > nsorted) {
    classify_kernel<<<grid_for(ncl), 256, 0, st>>>(cptr.as<int64_t>(), offs.as<int64_t>(), nzd.as<int64_t>(),
                                                   cmin.as<int64_t>(), cmax.as<int64_t>(), ncl, b_rowdense, l2_budget,
                                                   sort_output, sizeof(V), sizeof(int64_t),
                                                   settled.as<unsigned char>(), drop.as<unsigned char>(),
                                                   reinterpret_cast<unsigned long long*>(ndense.p));
    SPOPS_LAUNCH_CHECK();
  }
  tr.mark(st, "classify");

  // --- numeric bins: 0 / 1 warp per cluster (8 KB arena, 8 warps / 16 KB, 4
  // warps), 2 / 3 / 4 wide warp per cluster (16 KB, 2 warps / 32 KB, 1 warp /
  // 56 KB, 1 warp: small blocks so that the SM's shared memory fills), 5 / 6
  // block with the arena in 96 / 200 KB of shared memory, 7 block with the
  // arena in global memory; clusters with nz == 0 and those the sort path
  // settled are skipped
  constexpr int kWarpBins = 5;
  const int64_t warp_bytes[kWarpBins] = {8 << 10, 16 << 10, 16 << 10, 32 << 10, 56 << 10};
  const int warp_count[kWarpBins] = {8, 4, 2, 1, 1};
  const int num_threads[3] = {128, 256, 256};
  const size_t num_smem[3] = {96 << 10, 200 << 10, 0};
  NumBinLimits lim{{warp_bytes[0], warp_bytes[1], warp_bytes[2], warp_bytes[3], warp_bytes[4], (int64_t)num_smem[0],
                    (int64_t)num_smem[1]}};
  PoolBuf nslots(ctx), ngb(ctx), ngoff(ctx), arena(ctx);
  SPOPS_TRY(nslots.alloc(ncl1 * sizeof(NumSlot)));
  SPOPS_TRY(ngb.alloc(ncl1 * 8));
  SPOPS_TRY(ngoff.alloc(ncl1 * 8));
  std::vector<int64_t> nstart(9, 0);
  if (ncl > nsorted) {
    num_bin_kernel<<<grid_for(ncl), 256, 0, st>>>(nzd.as<int64_t>(), cnt_d, offs.as<int64_t>(), ncl, (int64_t)sizeof(V),
                                                 lim, settled.as<unsigned char>(), bkey.as<uint32_t>(),
                                                 bid.as<int64_t>());
    SPOPS_LAUNCH_CHECK();
    SPOPS_TRY(sort_bins(8, nstart));
  }
  const int64_t nlisted = nstart[8];
  if (nlisted > 0) {
    num_list_kernel<<<grid_for(nlisted), 256, 0, st>>>(bid_s.as<int64_t>(), nzd.as<int64_t>(), offs.as<int64_t>(),
                                                      nlisted, (int64_t)sizeof(V), nslots.as<NumSlot>(),
                                                      ngb.as<int64_t>());
    SPOPS_LAUNCH_CHECK();
  }
  int64_t garena = 0;
  SPOPS_TRY(seg_scan(ngb.as<int64_t>(), ngoff.as<int64_t>(), nstart[7], nstart[8], &garena));
  if (garena) SPOPS_TRY(arena.alloc((size_t)garena));
  for (int w = 0; w < kWarpBins; ++w) {
    const int64_t m = nstart[w + 1] - nstart[w];
    if (m <= 0) continue;
    const size_t smem = (size_t)warp_count[w] * (size_t)warp_bytes[w];
    const unsigned grid = (unsigned)((m + warp_count[w] - 1) / warp_count[w]);
    if (w < 2) {
      SPOPS_CUDA(cudaFuncSetAttribute(numeric_warp_kernel<I, V>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)smem));
      numeric_warp_kernel<I, V><<<grid, 32 * warp_count[w], smem, st>>>(
          bid_s.as<int64_t>() + nstart[w], m, nslots.as<NumSlot>() + nstart[w], warp_bytes[w], cptr.as<int64_t>(),
          cptr_val.as<int64_t>(), colids.as<int32_t>(), avals.as<V>(), offs.as<int64_t>(), B->row.as<I>(),
          B->col.as<I>(), B->val.as<V>(), nzd.as<int64_t>(), soff.as<int64_t>(), soff_val.as<int64_t>(),
          drop.as<unsigned char>(), ccol.as<int32_t>(), cval.as<V>());
    } else {
      SPOPS_CUDA(cudaFuncSetAttribute(numeric_warp_wide_kernel<I, V>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)smem));
      numeric_warp_wide_kernel<I, V><<<grid, 32 * warp_count[w], smem, st>>>(
          bid_s.as<int64_t>() + nstart[w], m, nslots.as<NumSlot>() + nstart[w], warp_bytes[w], cptr.as<int64_t>(),
          cptr_val.as<int64_t>(), colids.as<int32_t>(), avals.as<V>(), offs.as<int64_t>(), B->row.as<I>(),
          B->col.as<I>(), B->val.as<V>(), nzd.as<int64_t>(), soff.as<int64_t>(), soff_val.as<int64_t>(),
          drop.as<unsigned char>(), ccol.as<int32_t>(), cval.as<V>());
    }
    SPOPS_LAUNCH_CHECK();
  }
  tr.mark(st, "numeric bins + warp kernels");
  for (int w = 0; w < 3; ++w) {
    const int64_t m = nstart[w + kWarpBins + 1] - nstart[w + kWarpBins];
    if (m <= 0) continue;
    const bool global = w == 2;
    if (num_smem[w] > 48 * 1024)
      SPOPS_CUDA(cudaFuncSetAttribute(numeric_kernel<I, V>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)num_smem[w]));
    numeric_kernel<I, V><<<(unsigned)m, num_threads[w], num_smem[w], st>>>(
        bid_s.as<int64_t>() + nstart[w + kWarpBins], m, nslots.as<NumSlot>() + nstart[w + kWarpBins], cptr.as<int64_t>(),
        cptr_val.as<int64_t>(), colids.as<int32_t>(), avals.as<V>(), offs.as<int64_t>(), B->row.as<I>(),
        B->col.as<I>(), B->val.as<V>(), nzd.as<int64_t>(), soff.as<int64_t>(), soff_val.as<int64_t>(),
        drop.as<unsigned char>(), global ? arena.as<unsigned char>() : nullptr,
        global ? ngoff.as<int64_t>() + nstart[7] : nullptr, ccol.as<int32_t>(), cval.as<V>());
    SPOPS_LAUNCH_CHECK();
  }
  int64_t hdense = 0, c_cols = 0;
  SPOPS_CUDA(cudaMemcpyAsync(&hdense, ndense.p, 8, cudaMemcpyDeviceToHost, st));
  if (ncl > 0) {  // distinct output columns over all clusters (statistics)
    size_t c1 = 0;
    SPOPS_CUDA(cub::DeviceReduce::Sum(nullptr, c1, nzd.as<int64_t>(), tot.as<int64_t>(), ncl, st));
    SPOPS_TRY(tmp.alloc(c1 + 256));
    SPOPS_CUDA(cub::DeviceReduce::Sum(tmp.p, c1, nzd.as<int64_t>(), tot.as<int64_t>(), ncl, st));
    SPOPS_CUDA(cudaMemcpyAsync(&c_cols, tot.p, 8, cudaMemcpyDeviceToHost, st));
  }
  SPOPS_CUDA(cudaStreamSynchronize(st));
  arena.release();
  if (stats) stats->numeric_ms = tm.lap(st);
  tr.mark(st, "numeric block kernels");

  if (cluster_out) {  // --- C in the clustered form of A's clusters
    PoolBuf kcnt(ctx), kval(ctx), nrp(ctx), nrpv(ctx), kcol(ctx), kv(ctx);
    SPOPS_TRY(kcnt.alloc((size_t)(ncl + 1) * 8));
    SPOPS_TRY(kval.alloc((size_t)(ncl + 1) * 8));
    SPOPS_TRY(nrp.alloc((size_t)(ncl + 1) * 8));
    SPOPS_TRY(nrpv.alloc((size_t)(ncl + 1) * 8));
    SPOPS_CUDA(cudaMemsetAsync(kcnt.p, 0, (size_t)(ncl + 1) * 8, st));
    SPOPS_CUDA(cudaMemsetAsync(kval.p, 0, (size_t)(ncl + 1) * 8, st));
    if (ncl > 0) {
      cl_keep_count_kernel<V><<<grid_for(ncl * 32), 256, 0, st>>>(soff_val.as<int64_t>(), nzd.as<int64_t>(),
                                                                 offs.as<int64_t>(), ncl, cval.as<V>(),
                                                                 drop.as<unsigned char>(), kcnt.as<int64_t>(),
                                                                 kval.as<int64_t>());
      SPOPS_LAUNCH_CHECK();
    }
    size_t c1 = 0;
    SPOPS_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, c1, kcnt.as<int64_t>(), nrp.as<int64_t>(), ncl + 1, st));
    SPOPS_TRY(tmp.alloc(c1 + 256));
    SPOPS_CUDA(cub::DeviceScan::ExclusiveSum(tmp.p, c1, kcnt.as<int64_t>(), nrp.as<int64_t>(), ncl + 1, st));
    SPOPS_CUDA(cub::DeviceScan::ExclusiveSum(tmp.p, c1, kval.as<int64_t>(), nrpv.as<int64_t>(), ncl + 1, st));
    int64_t h2[2] = {0, 0};
    SPOPS_CUDA(cudaMemcpyAsync(h2, nrp.as<int64_t>() + ncl, 8, cudaMemcpyDeviceToHost, st));
    SPOPS_CUDA(cudaMemcpyAsync(h2 + 1, nrpv.as<int64_t>() + ncl, 8, cudaMemcpyDeviceToHost, st));
    SPOPS_CUDA(cudaStreamSynchronize(st));
    if (sizeof(I) == 4 && h2[1] > INT32_MAX)
      return fail(SPOPS_ERR_TOO_LARGE, "SpGEMM: %lld clustered values exceed int32 indices", (long long)h2[1]);
    SPOPS_TRY(kcol.alloc((size_t)std::max<int64_t>(h2[0], 1) * 4));
    SPOPS_TRY(kv.alloc((size_t)std::max<int64_t>(h2[1], 1) * sizeof(V)));
    if (ncl > 0) {
      cl_compact_kernel<int32_t, V><<<grid_for(ncl * 32), 256, 0, st>>>(
          soff.as<int64_t>(), soff_val.as<int64_t>(), nzd.as<int64_t>(), offs.as<int64_t>(), ncl, ccol.as<int32_t>(),
          cval.as<V>(),
          drop.as<unsigned char>(), nrp.as<int64_t>(), nrpv.as<int64_t>(), kcol.as<int32_t>(), kv.as<V>());
      SPOPS_LAUNCH_CHECK();
    }
    SPOPS_TRY((make_vlcluster<I, V>(ctx, n, B->cols, ncl, offs.as<int64_t>(), nrp.as<int64_t>(), kcol.as<int32_t>(),
                                    h2[0], nrpv.as<int64_t>(), kv.as<V>(), h2[1], A->itype, out)));
    if (stats) {
      stats->to_csr_ms = tm.lap(st);
      stats->flops = 2 * total_products;
      stats->clusters = ncl;
      stats->dense_clusters = hdense;
      stats->cluster_columns = nnzc;
      stats->c_cluster_columns = h2[0];
    }
    return SPOPS_OK;
  }

  // --- back to CSR, original row order
  PoolBuf rowcnt(ctx), crp(ctx);
  SPOPS_TRY(rowcnt.alloc((nn + 1) * 8));
  SPOPS_TRY(crp.alloc((nn + 1) * 8));
  SPOPS_CUDA(cudaMemsetAsync(rowcnt.p, 0, (nn + 1) * 8, st));
  if (ncl > 0) {
    row_count_kernel<V><<<grid_for(ncl * 32), 256, 0, st>>>(soff_val.as<int64_t>(), nzd.as<int64_t>(),
                                                            offs.as<int64_t>(), perm.as<int64_t>(), ncl, cval.as<V>(),
                                                            rowwise, rowcnt.as<int64_t>());
    SPOPS_LAUNCH_CHECK();
  }
  SPOPS_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, cb, rowcnt.as<int64_t>(), crp.as<int64_t>(), (int64_t)(n + 1), st));
  SPOPS_TRY(tmp.alloc(cb + 256));
  SPOPS_CUDA(cub::DeviceScan::ExclusiveSum(tmp.p, cb, rowcnt.as<int64_t>(), crp.as<int64_t>(), (int64_t)(n + 1), st));
  int64_t cnnz = 0;
  SPOPS_CUDA(cudaMemcpyAsync(&cnnz, crp.as<int64_t>() + n, 8, cudaMemcpyDeviceToHost, st));
  SPOPS_CUDA(cudaStreamSynchronize(st));
  tr.mark(st, "row counts + scan");
  if (sizeof(I) == 4 && cnnz > INT32_MAX)
    return fail(SPOPS_ERR_TOO_LARGE, "SpGEMM: %lld output entries exceed int32 indices", (long long)cnnz);
  Matrix* C = new spops_matrix_s();
  C->ctx = ctx;
  C->format = SPOPS_FMT_CSR;
  C->itype = A->itype;
  C->vtype = A->vtype;
  C->rows = n;
  C->cols = B->cols;
  C->nnz = cnnz;
  spops_status_t s = C->row.alloc_cached(ctx, (nn + 1) * sizeof(I));
  if (s == SPOPS_OK) s = C->col.alloc_cached(ctx, (size_t)std::max<int64_t>(cnnz, 1) * sizeof(I));
  if (s == SPOPS_OK) s = C->val.alloc_cached(ctx, (size_t)std::max<int64_t>(cnnz, 1) * sizeof(V));
  if (s != SPOPS_OK) {
    C->release_all();
    delete static_cast<spops_matrix_s*>(C);
    return s;
  }
  // row offsets in the index type
  tr.mark(st, "C alloc");
  if (sizeof(I) == 8) {
    SPOPS_CUDA(cudaMemcpyAsync(C->row.p, crp.p, (size_t)(n + 1) * 8, cudaMemcpyDeviceToDevice, st));
  } else {
    to_i32_kernel<<<grid_for(n + 1), 256, 0, st>>>(crp.as<int64_t>(), n + 1, C->row.as<int32_t>());
    SPOPS_LAUNCH_CHECK();
  }
  if (ncl > 0 && cnnz > 0) {
    row_write_kernel<I, V><<<grid_for(ncl * 32), 256, 0, st>>>(soff.as<int64_t>(), soff_val.as<int64_t>(),
                                                               nzd.as<int64_t>(), offs.as<int64_t>(),
                                                               perm.as<int64_t>(), ncl,
                                                               ccol.as<int32_t>(), cval.as<V>(), rowwise,
                                                               crp.as<int64_t>(), C->col.as<I>(), C->val.as<V>());
    SPOPS_LAUNCH_CHECK();
  }
  SPOPS_CUDA(cudaStreamSynchronize(st));
  tr.mark(st, "row offsets + row write");
  if (stats) {
    stats->to_csr_ms = tm.lap(st);
    stats->flops = 2 * total_products;
    stats->clusters = ncl;
    stats->dense_clusters = hdense;
    stats->cluster_columns = nnzc;
    stats->c_cluster_columns = c_cols;
  }
  *out = C;
  return SPOPS_OK;
}

}  // namespace

spops_status_t cluster_spgemm(Context* ctx, Matrix* A, Matrix* B, const int64_t* perm, const int64_t* offsets,
                              int64_t nclusters, bool sort_output, double l2_budget, Matrix** C, SpgemmStats* st,
                              bool rowwise, bool cluster_out, bool device_arrays) {
  if (A->format != SPOPS_FMT_CSR || B->format != SPOPS_FMT_CSR)
    return fail(SPOPS_ERR_INVALID, "SpGEMM needs CSR matrices");
  if (A->cols != B->rows) return fail(SPOPS_ERR_INVALID, "SpGEMM: A.cols (%lld) != B.rows (%lld)",
                                      (long long)A->cols, (long long)B->rows);
  if (A->itype != B->itype || A->vtype != B->vtype) return fail(SPOPS_ERR_INVALID, "SpGEMM: mixed types");
  if (B->cols > INT32_MAX || A->cols > INT32_MAX || nclusters > INT32_MAX)
    return fail(SPOPS_ERR_UNSUPPORTED, "SpGEMM: more than 2^31 columns or clusters");
  if (nclusters < 0) return fail(SPOPS_ERR_INVALID, "SpGEMM: negative cluster count");
  // a caller's host arrays are checked here; the device clustering's own
  // output (device_arrays) is a permutation with offsets from 0 to rows by
  // construction
  if (!device_arrays && (offsets[0] != 0 || offsets[nclusters] != A->rows))
    return fail(SPOPS_ERR_INVALID, "SpGEMM: offsets must run from 0 to rows");
  for (int64_t c = 0; !device_arrays && c < nclusters; ++c)
    if (offsets[c + 1] < offsets[c]) return fail(SPOPS_ERR_INVALID, "SpGEMM: offsets not monotone");
  if (!device_arrays) {
    std::vector<unsigned char> seen((size_t)A->rows, 0);
    for (int64_t r = 0; r < A->rows; ++r) {
      if (perm[r] < 0 || perm[r] >= A->rows || seen[perm[r]]) return fail(SPOPS_ERR_INVALID, "SpGEMM: bad permutation");
      seen[perm[r]] = 1;
    }
  }
  if (!A->plan.ready) SPOPS_TRY(csr_analyse(ctx, A));  // validates patterns
  if (!B->plan.ready) SPOPS_TRY(csr_analyse(ctx, B));
  const bool i32 = A->itype == SPOPS_INDEX_I32, f64 = A->vtype == SPOPS_VALUE_F64;
  if (i32 && f64) return spgemm_t<int32_t, double>(ctx, A, B, perm, offsets, nclusters, sort_output, l2_budget, rowwise, C, st,
                                            cluster_out);
  if (i32) return spgemm_t<int32_t, float>(ctx, A, B, perm, offsets, nclusters, sort_output, l2_budget, rowwise, C, st,
                                            cluster_out);
  if (f64) return spgemm_t<int64_t, double>(ctx, A, B, perm, offsets, nclusters, sort_output, l2_budget, rowwise, C, st,
                                            cluster_out);
  return spgemm_t<int64_t, float>(ctx, A, B, perm, offsets, nclusters, sort_output, l2_budget, rowwise, C, st,
                                            cluster_out);
}

namespace {

template <typename I, typename V>
spops_status_t vl_from_csr_t(Context* ctx, Matrix* A, const int64_t* offs_h, int64_t ncl, Matrix** out) {
  cudaStream_t st = ctx->stream;
  const int64_t n = A->rows, nnz = A->nnz;
  const size_t nn = (size_t)std::max<int64_t>(n, 1), nz1 = (size_t)std::max<int64_t>(nnz, 1);
  ArenaScope scope(ctx);  // this call's temporaries come from the arena
  PoolBuf perm(ctx), offs(ctx), rowcl(ctx), rlen(ctx), rpr(ctx), keys(ctx), skeys(ctx), src(ctx), ssrc(ctx),
      flag(ctx), uidx(ctx), colids(ctx), ncols_u(ctx), cptr(ctx), cptr_val(ctx), cw(ctx), avals(ctx), roe(ctx),
      tmp(ctx);
  SPOPS_TRY(perm.alloc(nn * 8));
  SPOPS_TRY(offs.alloc((size_t)(ncl + 1) * 8));
  SPOPS_TRY(rowcl.alloc(nn * 8));
  SPOPS_TRY(rlen.alloc(nn * 8));
  SPOPS_TRY(rpr.alloc((nn + 1) * 8));
  SPOPS_CUDA(cudaMemcpyAsync(offs.p, offs_h, (size_t)(ncl + 1) * 8, cudaMemcpyHostToDevice, st));
  if (n > 0) iota_kernel<<<grid_for(n), 256, 0, st>>>(perm.as<int64_t>(), n);
  if (ncl > 0) row_cluster_kernel<<<grid_for(ncl), 256, 0, st>>>(offs.as<int64_t>(), ncl, rowcl.as<int64_t>());
  if (n > 0) reordered_len_kernel<I><<<grid_for(n), 256, 0, st>>>(A->row.as<I>(), perm.as<int64_t>(), n, rlen.as<int64_t>());
  SPOPS_LAUNCH_CHECK();
  size_t cb = 0;
  SPOPS_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, cb, rlen.as<int64_t>(), rpr.as<int64_t>(), (int64_t)nn, st));
  SPOPS_TRY(tmp.alloc(cb + 256));
  if (n > 0) SPOPS_CUDA(cub::DeviceScan::ExclusiveSum(tmp.p, cb, rlen.as<int64_t>(), rpr.as<int64_t>(), n, st));
  SPOPS_TRY(keys.alloc(nz1 * 8));
  SPOPS_TRY(skeys.alloc(nz1 * 8));
  SPOPS_TRY(src.alloc(nz1 * 8));
  SPOPS_TRY(ssrc.alloc(nz1 * 8));
  SPOPS_TRY(flag.alloc(nz1 * 8));
  SPOPS_TRY(uidx.alloc(nz1 * 8));
  SPOPS_TRY(roe.alloc(nz1 * 8));
  // key = cluster << kshift | column: sort only the bits in use
  const int kshift = key_bits(A->cols), kend = std::min(64, kshift + key_bits(ncl));
  if (n > 0) {
    cluster_keys_kernel<I, V><<<grid_for(n * 32), 256, 0, st>>>(A->row.as<I>(), A->col.as<I>(), perm.as<int64_t>(),
                                                                rowcl.as<int64_t>(), n, rpr.as<int64_t>(), kshift,
                                                                keys.as<uint64_t>(), src.as<int64_t>());
    entry_row_kernel<I><<<grid_for(n * 32), 256, 0, st>>>(A->row.as<I>(), perm.as<int64_t>(), n, roe.as<int64_t>());
    SPOPS_LAUNCH_CHECK();
  }
  int64_t nnzc = 0;
  SPOPS_TRY(ncols_u.alloc((size_t)(ncl + 1) * 8));
  SPOPS_CUDA(cudaMemsetAsync(ncols_u.p, 0, (size_t)(ncl + 1) * 8, st));
  if (nnz > 0) {
    size_t c1 = 0, c2 = 0;
    SPOPS_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, c1, keys.as<uint64_t>(), skeys.as<uint64_t>(), src.as<int64_t>(),
                                               ssrc.as<int64_t>(), nnz, 0, kend, st));
    SPOPS_CUDA(cub::DeviceScan::InclusiveSum(nullptr, c2, flag.as<int64_t>(), uidx.as<int64_t>(), nnz, st));
    SPOPS_TRY(tmp.alloc(std::max(c1, c2) + 256));
    SPOPS_CUDA(cub::DeviceRadixSort::SortPairs(tmp.p, c1, keys.as<uint64_t>(), skeys.as<uint64_t>(), src.as<int64_t>(),
                                               ssrc.as<int64_t>(), nnz, 0, kend, st));
    key_flag_kernel<<<grid_for(nnz), 256, 0, st>>>(skeys.as<uint64_t>(), nnz, flag.as<int64_t>());
    SPOPS_LAUNCH_CHECK();
    SPOPS_CUDA(cub::DeviceScan::InclusiveSum(tmp.p, c2, flag.as<int64_t>(), uidx.as<int64_t>(), nnz, st));
    SPOPS_CUDA(cudaMemcpyAsync(&nnzc, uidx.as<int64_t>() + nnz - 1, 8, cudaMemcpyDeviceToHost, st));
    SPOPS_CUDA(cudaStreamSynchronize(st));
  }
  SPOPS_TRY(colids.alloc((size_t)std::max<int64_t>(nnzc, 1) * 4));
  if (nnz > 0) {
    cluster_cols_kernel<<<grid_for(nnz), 256, 0, st>>>(skeys.as<uint64_t>(), flag.as<int64_t>(), uidx.as<int64_t>(),
                                                       nnz, kshift, colids.as<int32_t>(),
                                                       reinterpret_cast<unsigned long long*>(ncols_u.p));
    SPOPS_LAUNCH_CHECK();
  }
  SPOPS_TRY(cptr.alloc((size_t)(ncl + 1) * 8));
  SPOPS_TRY(cptr_val.alloc((size_t)(ncl + 1) * 8));
  SPOPS_TRY(cw.alloc((size_t)(ncl + 1) * 8));
  SPOPS_CUDA(cudaMemsetAsync(cw.p, 0, (size_t)(ncl + 1) * 8, st));
  const int64_t* cnt_d = reinterpret_cast<const int64_t*>(ncols_u.p);
  if (ncl > 0) {
    weight_kernel<<<grid_for(ncl), 256, 0, st>>>(cnt_d, offs.as<int64_t>(), ncl, cw.as<int64_t>());
    SPOPS_LAUNCH_CHECK();
  }
  {
    size_t c1 = 0, c2 = 0;
    SPOPS_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, c1, cnt_d, cptr.as<int64_t>(), ncl + 1, st));
    SPOPS_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, c2, cw.as<int64_t>(), cptr_val.as<int64_t>(), ncl + 1, st));
    SPOPS_TRY(tmp.alloc(std::max(c1, c2) + 256));
    SPOPS_CUDA(cub::DeviceScan::ExclusiveSum(tmp.p, c1, cnt_d, cptr.as<int64_t>(), ncl + 1, st));
    SPOPS_CUDA(cub::DeviceScan::ExclusiveSum(tmp.p, c2, cw.as<int64_t>(), cptr_val.as<int64_t>(), ncl + 1, st));
  }
  int64_t nnzv = 0;
  SPOPS_CUDA(cudaMemcpyAsync(&nnzv, cptr_val.as<int64_t>() + ncl, 8, cudaMemcpyDeviceToHost, st));
  SPOPS_CUDA(cudaStreamSynchronize(st));
  if (sizeof(I) == 4 && nnzv > INT32_MAX)
    return fail(SPOPS_ERR_TOO_LARGE, "csr_to_vlength_cluster: %lld values exceed int32 indices", (long long)nnzv);
  SPOPS_TRY(avals.alloc((size_t)std::max<int64_t>(nnzv, 1) * sizeof(V)));
  SPOPS_CUDA(cudaMemsetAsync(avals.p, 0, avals.bytes, st));
  if (nnz > 0) {
    cluster_vals_kernel<I, V><<<grid_for(nnz), 256, 0, st>>>(
        skeys.as<uint64_t>(), ssrc.as<int64_t>(), uidx.as<int64_t>(), nnz, kshift, A->val.as<V>(), A->row.as<I>(),
        perm.as<int64_t>(), offs.as<int64_t>(), cptr.as<int64_t>(), cptr_val.as<int64_t>(), roe.as<int64_t>(),
        avals.as<V>());
    SPOPS_LAUNCH_CHECK();
  }
  return make_vlcluster<I, V>(ctx, n, A->cols, ncl, offs.as<int64_t>(), cptr.as<int64_t>(), colids.as<int32_t>(),
                              nnzc, cptr_val.as<int64_t>(), avals.as<V>(), nnzv, A->itype, out);
}

template <typename I, typename V>
spops_status_t vl_to_csr_t(Context* ctx, Matrix* M, Matrix** out) {
  cudaStream_t st = ctx->stream;
  const int64_t n = M->rows, ncl = M->clusters;
  const size_t nn = (size_t)std::max<int64_t>(n, 1);
  ArenaScope scope(ctx);  // this call's temporaries come from the arena
  PoolBuf rowcl(ctx), cnt(ctx), crp(ctx), tmp(ctx);
  SPOPS_TRY(rowcl.alloc(nn * 8));
  SPOPS_TRY(cnt.alloc((nn + 1) * 8));
  SPOPS_TRY(crp.alloc((nn + 1) * 8));
  SPOPS_CUDA(cudaMemsetAsync(cnt.p, 0, (nn + 1) * 8, st));
  if (ncl > 0) row_cluster_kernel<<<grid_for(ncl), 256, 0, st>>>(M->cl_off.as<int64_t>(), ncl, rowcl.as<int64_t>());
  if (n > 0)
    vlc_row_count_kernel<I, V><<<grid_for(n), 256, 0, st>>>(M->row.as<I>(), M->cl_rpv.as<I>(), M->cl_off.as<int64_t>(),
                                                            ncl, rowcl.as<int64_t>(), n, M->val.as<V>(),
                                                            cnt.as<int64_t>());
  SPOPS_LAUNCH_CHECK();
  size_t cb = 0;
  SPOPS_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, cb, cnt.as<int64_t>(), crp.as<int64_t>(), n + 1, st));
  SPOPS_TRY(tmp.alloc(cb + 256));
  SPOPS_CUDA(cub::DeviceScan::ExclusiveSum(tmp.p, cb, cnt.as<int64_t>(), crp.as<int64_t>(), n + 1, st));
  int64_t cnnz = 0;
  SPOPS_CUDA(cudaMemcpyAsync(&cnnz, crp.as<int64_t>() + n, 8, cudaMemcpyDeviceToHost, st));
  SPOPS_CUDA(cudaStreamSynchronize(st));
  Matrix* C = new spops_matrix_s();
  C->ctx = ctx;
  C->format = SPOPS_FMT_CSR;
  C->itype = M->itype;
  C->vtype = M->vtype;
  C->rows = n;
  C->cols = M->cols;
  C->nnz = cnnz;
  spops_status_t s = C->row.alloc_cached(ctx, (nn + 1) * sizeof(I));
  if (s == SPOPS_OK) s = C->col.alloc_cached(ctx, (size_t)std::max<int64_t>(cnnz, 1) * sizeof(I));
  if (s == SPOPS_OK) s = C->val.alloc_cached(ctx, (size_t)std::max<int64_t>(cnnz, 1) * sizeof(V));
  if (s == SPOPS_OK) {
    cast_kernel<int64_t, I><<<grid_for(n + 1), 256, 0, st>>>(crp.as<int64_t>(), n + 1, C->row.as<I>());
    if (n > 0 && cnnz > 0)
      vlc_row_write_kernel<I, V><<<grid_for(n), 256, 0, st>>>(M->row.as<I>(), M->cl_rpv.as<I>(), M->col.as<I>(),
                                                              M->cl_off.as<int64_t>(), rowcl.as<int64_t>(), n,
                                                              M->val.as<V>(), crp.as<int64_t>(), C->col.as<I>(),
                                                              C->val.as<V>());
    if (cudaGetLastError() != cudaSuccess || cudaStreamSynchronize(st) != cudaSuccess)
      s = fail(SPOPS_ERR_CUDA, "vlength_cluster2csr: launch failed");
  }
  if (s != SPOPS_OK) {
    C->release_all();
    delete static_cast<spops_matrix_s*>(C);
    return s;
  }
  *out = C;
  return SPOPS_OK;
}

}  // namespace

spops_status_t vlcluster_finish(Context* ctx, Matrix* M, const int64_t* off_h) {
  cudaStream_t st = ctx->stream;
  const int64_t ncl = M->clusters;
  int64_t mx = 256;  // as csr_to_vlength_cluster: starts at 256, raised by larger clusters
  std::vector<int64_t> sz((size_t)std::max<int64_t>(ncl, 1), 0);
  for (int64_t c = 0; c < ncl; ++c) {
    sz[(size_t)c] = off_h[c + 1] - off_h[c];
    mx = std::max(mx, sz[(size_t)c]);
  }
  M->cl_max_sz = mx;
  SPOPS_TRY(M->cl_off.alloc((size_t)(ncl + 1) * 8));
  SPOPS_TRY(M->cl_sz.alloc((size_t)std::max<int64_t>(ncl, 1) * M->isize()));
  SPOPS_CUDA(cudaMemcpyAsync(M->cl_off.p, off_h, (size_t)(ncl + 1) * 8, cudaMemcpyHostToDevice, st));
  if (M->itype == SPOPS_INDEX_I64) {
    SPOPS_CUDA(cudaMemcpyAsync(M->cl_sz.p, sz.data(), (size_t)ncl * 8, cudaMemcpyHostToDevice, st));
  } else {
    std::vector<int32_t> s32(sz.begin(), sz.end());
    SPOPS_CUDA(cudaMemcpyAsync(M->cl_sz.p, s32.data(), (size_t)ncl * 4, cudaMemcpyHostToDevice, st));
  }
  SPOPS_CUDA(cudaStreamSynchronize(st));
  return SPOPS_OK;
}

spops_status_t vlcluster_from_csr(Context* ctx, Matrix* A, const int64_t* offsets, int64_t nclusters, Matrix** out) {
  if (A->format != SPOPS_FMT_CSR) return fail(SPOPS_ERR_INVALID, "csr_to_vlength_cluster: needs a CSR matrix");
  if (nclusters < 0 || offsets[0] != 0 || offsets[nclusters] != A->rows)
    return fail(SPOPS_ERR_INVALID, "csr_to_vlength_cluster: offsets must run from 0 to rows");
  for (int64_t c = 0; c < nclusters; ++c)
    if (offsets[c + 1] < offsets[c]) return fail(SPOPS_ERR_INVALID, "csr_to_vlength_cluster: offsets not monotone");
  if (A->cols > INT32_MAX || nclusters > INT32_MAX)
    return fail(SPOPS_ERR_UNSUPPORTED, "csr_to_vlength_cluster: more than 2^31 columns or clusters");
  if (!A->plan.ready) SPOPS_TRY(csr_analyse(ctx, A));  // validates the pattern
  const bool i32 = A->itype == SPOPS_INDEX_I32, f64 = A->vtype == SPOPS_VALUE_F64;
  if (i32 && f64) return vl_from_csr_t<int32_t, double>(ctx, A, offsets, nclusters, out);
  if (i32) return vl_from_csr_t<int32_t, float>(ctx, A, offsets, nclusters, out);
  if (f64) return vl_from_csr_t<int64_t, double>(ctx, A, offsets, nclusters, out);
  return vl_from_csr_t<int64_t, float>(ctx, A, offsets, nclusters, out);
}

spops_status_t vlcluster_to_csr(Context* ctx, Matrix* M, Matrix** out) {
  if (M->format != SPOPS_FMT_VLCLUSTER) return fail(SPOPS_ERR_INVALID, "vlength_cluster2csr: needs a clustered matrix");
  const bool i32 = M->itype == SPOPS_INDEX_I32, f64 = M->vtype == SPOPS_VALUE_F64;
  if (i32 && f64) return vl_to_csr_t<int32_t, double>(ctx, M, out);
  if (i32) return vl_to_csr_t<int32_t, float>(ctx, M, out);
  if (f64) return vl_to_csr_t<int64_t, double>(ctx, M, out);
  return vl_to_csr_t<int64_t, float>(ctx, M, out);
}

}  // namespace spops

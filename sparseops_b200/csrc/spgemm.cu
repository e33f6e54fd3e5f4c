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
template <typename I, typename V>
__global__ void cluster_keys_kernel(const I* __restrict__ rp, const I* __restrict__ ci, const int64_t* __restrict__ perm,
                                    const int64_t* __restrict__ row_cluster, int64_t n, const int64_t* __restrict__ rpr,
                                    uint64_t* __restrict__ keys, int64_t* __restrict__ src) {
  // warp per reordered row: entries of original row perm[r] in order
  const int64_t r = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (r >= n) return;
  const int64_t orow = perm[r];
  const int64_t s = rp[orow], e = rp[orow + 1], o = rpr[r];
  const uint64_t c = (uint64_t)row_cluster[r];
  for (int64_t k = lane; k < e - s; k += 32) {
    keys[o + k] = (c << 32) | (uint64_t)(uint32_t)ci[s + k];
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
                                    const int64_t* __restrict__ uidx, int64_t m, int32_t* __restrict__ colids,
                                    unsigned long long* __restrict__ ncols) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= m || !flag[i]) return;
  const int64_t u = uidx[i] - 1;
  colids[u] = (int32_t)(keys[i] & 0xffffffffULL);
  atomicAdd(ncols + (keys[i] >> 32), 1ULL);
}

template <typename I, typename V>
__global__ void cluster_vals_kernel(const uint64_t* __restrict__ keys, const int64_t* __restrict__ src,
                                    const int64_t* __restrict__ uidx, int64_t m, const V* __restrict__ av,
                                    const I* __restrict__ rp, const int64_t* __restrict__ perm,
                                    const int64_t* __restrict__ offsets, const int64_t* __restrict__ cptr,
                                    const int64_t* __restrict__ cptr_val, const int64_t* __restrict__ row_of_entry,
                                    V* __restrict__ cvals) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= m) return;
  const int64_t c = (int64_t)(keys[i] >> 32);
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
  __syncthreads();
  unsigned long long cnt = 0;
  int mn = INT32_MAX, mx = -1;
  for (int64_t j = cptr[c] + threadIdx.x; j < cptr[c + 1]; j += blockDim.x) {
    const int64_t r = colids[j];
    for (int64_t k = brp[r]; k < brp[r + 1]; ++k) {
      const int32_t key = (int32_t)bci[k];
      if (hash_insert(tab, mask, key)) {
        ++cnt;
        mn = key < mn ? key : mn;
        mx = key > mx ? key : mx;
      }
    }
  }
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
template <typename I, typename V>
__global__ void numeric_warp_kernel(const int64_t* __restrict__ list, int64_t nlist, const NumSlot* __restrict__ slots,
                                    int64_t warp_bytes, const int64_t* __restrict__ cptr,
                                    const int64_t* __restrict__ cptr_val, const int32_t* __restrict__ colids,
                                    const V* __restrict__ avals, const int64_t* __restrict__ offsets,
                                    const I* __restrict__ brp, const I* __restrict__ bci, const V* __restrict__ bv,
                                    const int64_t* __restrict__ nz, const int64_t* __restrict__ ccptr,
                                    const int64_t* __restrict__ ccptr_val, const unsigned char* __restrict__ drop_small,
                                    int32_t* __restrict__ ccol, V* __restrict__ cval) {
  extern __shared__ __align__(16) unsigned char sm[];
  constexpr int kMaxPerLane = 16;  // nz <= 512
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
  V* acc = reinterpret_cast<V*>(base + ((4 * (2 * S.tsize + nzc) + 15) & ~15LL));
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
  // 2. compact (slot order)
  int64_t n = 0;
  for (int64_t t0 = 0; t0 < S.tsize; t0 += 32) {
    const int32_t v = t0 + lane < S.tsize ? tab[t0 + lane] : -1;
    const unsigned m = __ballot_sync(0xffffffffu, v != -1);
    if (v != -1) keys[n + __popc(m & ((1u << lane) - 1u))] = v;
    n += __popc(m);
  }
  __syncwarp();
  // 3. rank by counting; the output column list is written in rank order
  int32_t mine[kMaxPerLane];
  int rank[kMaxPerLane];
#pragma unroll
  for (int q = 0; q < kMaxPerLane; ++q) {
    const int64_t p = lane + 32 * q;
    mine[q] = p < nzc ? keys[p] : INT32_MAX;
    rank[q] = 0;
  }
  for (int64_t p = 0; p < nzc; ++p) {
    const int32_t kq = keys[p];
#pragma unroll
    for (int q = 0; q < kMaxPerLane; ++q) rank[q] += kq < mine[q] ? 1 : 0;
  }
  const int64_t co = ccptr[c], cvo = ccptr_val[c];
#pragma unroll
  for (int q = 0; q < kMaxPerLane; ++q) {
    const int64_t p = lane + 32 * q;
    if (p < nzc) {
      pos[hash_find(tab, mask, mine[q])] = rank[q];
      ccol[co + rank[q]] = mine[q];
    }
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


template <typename I, typename V>
__global__ void numeric_kernel(const int64_t* __restrict__ list, int64_t nlist, const NumSlot* __restrict__ slots,
                               const int64_t* __restrict__ cptr, const int64_t* __restrict__ cptr_val,
                               const int32_t* __restrict__ colids, const V* __restrict__ avals,
                               const int64_t* __restrict__ offsets, const I* __restrict__ brp,
                               const I* __restrict__ bci, const V* __restrict__ bv, const int64_t* __restrict__ nz,
                               const int64_t* __restrict__ ccptr, const int64_t* __restrict__ ccptr_val,
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
  for (int64_t t = threadIdx.x; t < S.tsize; t += blockDim.x) tab[t] = -1;
  for (int64_t t = threadIdx.x; t < nzc * csz; t += blockDim.x) acc[t] = V(0);
  __syncthreads();
  // 1. distinct columns
  for (int64_t j = cptr[c] + threadIdx.x; j < cptr[c + 1]; j += blockDim.x) {
    const int64_t r = colids[j];
    for (int64_t k = brp[r]; k < brp[r + 1]; ++k) hash_insert(tab, mask, (int32_t)bci[k]);
  }
  __syncthreads();
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
  const int64_t co = ccptr[c], cvo = ccptr_val[c];
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
                                bool sort_output, size_t vbytes, size_t ibytes, unsigned char* __restrict__ drop,
                                unsigned long long* __restrict__ ndense) {
  const int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (c >= ncl) return;
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
__global__ void row_count_kernel(const int64_t* __restrict__ ccptr, const int64_t* __restrict__ ccptr_val,
                                 const int64_t* __restrict__ offsets, const int64_t* __restrict__ perm, int64_t ncl,
                                 const V* __restrict__ cval, int64_t* __restrict__ rowcnt) {
  // warp per cluster, lanes over its rows (csz <= 32 common) and columns
  const int64_t c = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (c >= ncl) return;
  const int64_t csz = offsets[c + 1] - offsets[c];
  const int64_t ncol = ccptr[c + 1] - ccptr[c];
  for (int64_t l = 0; l < csz; ++l) {
    int64_t cnt = 0;
    for (int64_t p = lane; p < ncol; p += 32) cnt += cval[ccptr_val[c] + p * csz + l] != V(0) ? 1 : 0;
    for (int o = 16; o > 0; o >>= 1) cnt += __shfl_down_sync(0xffffffffu, cnt, o);
    if (lane == 0) rowcnt[perm[offsets[c] + l]] = cnt;
  }
}

template <typename I, typename V>
__global__ void row_write_kernel(const int64_t* __restrict__ ccptr, const int64_t* __restrict__ ccptr_val,
                                 const int64_t* __restrict__ offsets, const int64_t* __restrict__ perm, int64_t ncl,
                                 const int32_t* __restrict__ ccol, const V* __restrict__ cval,
                                 const int64_t* __restrict__ crp, I* __restrict__ oci, V* __restrict__ ov) {
  const int64_t c = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (c >= ncl) return;
  const int64_t csz = offsets[c + 1] - offsets[c];
  const int64_t ncol = ccptr[c + 1] - ccptr[c];
  for (int64_t l = 0; l < csz; ++l) {
    int64_t o = crp[perm[offsets[c] + l]];
    for (int64_t p0 = 0; p0 < ncol; p0 += 32) {
      const int64_t p = p0 + lane;
      const V v = p < ncol ? cval[ccptr_val[c] + p * csz + l] : V(0);
      const bool keep = p < ncol && v != V(0);
      const unsigned m = __ballot_sync(0xffffffffu, keep);
      if (keep) {
        const int64_t at = o + __popc(m & ((1u << lane) - 1));
        oci[at] = (I)ccol[ccptr[c] + p];
        ov[at] = v;
      }
      o += __popc(m);
    }
  }
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

// SPOPS_TRACE=1 in the environment: wall time of each step of the SpGEMM
// driver on stderr (the stream is synchronised at every mark).
struct Trace {
  bool on = false;
  std::chrono::steady_clock::time_point t = std::chrono::steady_clock::now();
  Trace() {
    const char* e = std::getenv("SPOPS_TRACE");
    on = e && e[0] == '1';
  }
  void mark(cudaStream_t st, const char* what) {
    if (!on) return;
    cudaStreamSynchronize(st);
    const auto n = std::chrono::steady_clock::now();
    std::fprintf(stderr, "[spgemm] %-28s %9.3f ms\n", what, std::chrono::duration<double, std::milli>(n - t).count());
    t = n;
  }
};

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

template <typename I, typename V>
spops_status_t spgemm_t(Context* ctx, Matrix* A, Matrix* B, const int64_t* perm_h, const int64_t* offs_h, int64_t ncl,
                        bool sort_output, double l2_budget, Matrix** out, SpgemmStats* stats) {
  cudaStream_t st = ctx->stream;
  const int64_t n = A->rows, nnz = A->nnz;
  Timer tm;
  Trace tr;
  // --- permutation, offsets, per-row cluster
  PoolBuf perm(ctx), offs(ctx), rowcl(ctx), rlen(ctx), rpr(ctx), keys(ctx), skeys(ctx), src(ctx), ssrc(ctx), flag(ctx), uidx(ctx), colids(ctx), ncols_u(ctx), cptr(ctx), cptr_val(ctx), avals(ctx), row_of_entry(ctx), tmp(ctx);
  SPOPS_TRY(perm.alloc((size_t)std::max<int64_t>(n, 1) * 8));
  SPOPS_TRY(offs.alloc((size_t)(ncl + 1) * 8));
  SPOPS_CUDA(cudaMemcpyAsync(perm.p, perm_h, (size_t)n * 8, cudaMemcpyHostToDevice, st));
  SPOPS_CUDA(cudaMemcpyAsync(offs.p, offs_h, (size_t)(ncl + 1) * 8, cudaMemcpyHostToDevice, st));
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
  if (n > 0) {
    cluster_keys_kernel<I, V><<<grid_for(n * 32), 256, 0, st>>>(A->row.as<I>(), A->col.as<I>(), perm.as<int64_t>(),
                                                                rowcl.as<int64_t>(), n, rpr.as<int64_t>(),
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
                                               ssrc.as<int64_t>(), nnz, 0, 64, st));
    SPOPS_CUDA(cub::DeviceScan::InclusiveSum(nullptr, c2, flag.as<int64_t>(), uidx.as<int64_t>(), nnz, st));
    SPOPS_TRY(tmp.alloc(std::max(c1, c2) + 256));
    SPOPS_CUDA(cub::DeviceRadixSort::SortPairs(tmp.p, c1, keys.as<uint64_t>(), skeys.as<uint64_t>(), src.as<int64_t>(),
                                               ssrc.as<int64_t>(), nnz, 0, 64, st));
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
                                                       nnz, colids.as<int32_t>(),
                                                       reinterpret_cast<unsigned long long*>(ncols_u.p));
    SPOPS_LAUNCH_CHECK();
  }
  // cluster pointers on the host (ncl values)
  std::vector<int64_t> hcnt, hoff(offs_h, offs_h + ncl + 1), hcptr(ncl + 1, 0), hcptr_val(ncl + 1, 0);
  SPOPS_TRY(d2h(st, hcnt, ncols_u.p, (size_t)ncl));
  for (int64_t c = 0; c < ncl; ++c) {
    const int64_t csz = hoff[c + 1] - hoff[c];
    hcptr[c + 1] = hcptr[c] + hcnt[c];
    hcptr_val[c + 1] = hcptr_val[c] + hcnt[c] * csz;
  }
  SPOPS_TRY(h2d(st, cptr, hcptr));
  SPOPS_TRY(h2d(st, cptr_val, hcptr_val));
  tr.mark(st, "cluster pointers (host)");
  const int64_t nnzv = hcptr_val[ncl];
  SPOPS_TRY(avals.alloc((size_t)std::max<int64_t>(nnzv, 1) * sizeof(V)));
  SPOPS_CUDA(cudaMemsetAsync(avals.p, 0, avals.bytes, st));
  if (nnz > 0) {
    cluster_vals_kernel<I, V><<<grid_for(nnz), 256, 0, st>>>(
        skeys.as<uint64_t>(), ssrc.as<int64_t>(), uidx.as<int64_t>(), nnz, A->val.as<V>(), A->row.as<I>(),
        perm.as<int64_t>(), offs.as<int64_t>(), cptr.as<int64_t>(), cptr_val.as<int64_t>(),
        row_of_entry.as<int64_t>(), avals.as<V>());
    SPOPS_LAUNCH_CHECK();
  }
  keys.release(); skeys.release(); src.release(); ssrc.release(); flag.release(); uidx.release();
  row_of_entry.release(); rlen.release(); rpr.release(); rowcl.release();
  if (stats) stats->cluster_ms = tm.lap(st);
  tr.mark(st, "cluster values + frees");

  // --- flops per cluster and symbolic bins
  PoolBuf flops(ctx), nzd(ctx), cmin(ctx), cmax(ctx);
  SPOPS_TRY(flops.alloc((size_t)std::max<int64_t>(ncl, 1) * 8));
  SPOPS_TRY(nzd.alloc((size_t)std::max<int64_t>(ncl, 1) * 8));
  SPOPS_TRY(cmin.alloc((size_t)std::max<int64_t>(ncl, 1) * 8));
  SPOPS_TRY(cmax.alloc((size_t)std::max<int64_t>(ncl, 1) * 8));
  if (ncl > 0) {
    cluster_flops_kernel<I><<<grid_for(ncl * 32), 256, 0, st>>>(cptr.as<int64_t>(), colids.as<int32_t>(), ncl,
                                                                B->row.as<I>(), flops.as<int64_t>());
    SPOPS_LAUNCH_CHECK();
  }
  std::vector<int64_t> hflops;
  SPOPS_TRY(d2h(st, hflops, flops.p, (size_t)ncl));
  tr.mark(st, "flops per cluster");
  int64_t total_products = 0;
  {
    PoolBuf pc(ctx);
    SPOPS_TRY(pc.alloc(8));
    SPOPS_CUDA(cudaMemsetAsync(pc.p, 0, 8, st));
    if (nnz > 0) {
      product_count_kernel<I><<<std::min<unsigned>(grid_for(nnz), 4096u), 256, 0, st>>>(
          A->col.as<I>(), nnz, B->row.as<I>(), B->rows, reinterpret_cast<unsigned long long*>(pc.p));
      SPOPS_LAUNCH_CHECK();
    }
    SPOPS_CUDA(cudaMemcpyAsync(&total_products, pc.p, 8, cudaMemcpyDeviceToHost, st));
    SPOPS_CUDA(cudaStreamSynchronize(st));
    pc.release();
  }
  const int64_t bcols = B->cols;
  // symbolic: table >= 2 * min(flops, cols) slots
  struct Bin {
    std::vector<int64_t> list, tsize, goff;
    int threads = 32;
    size_t smem = 0;
    bool global = false;
  };
  auto sym_tsize = [&](int64_t c) { return pow2_at_least(std::max<int64_t>(2 * std::min(hflops[c], bcols), 2)); };
  Bin sb[3];
  sb[0].threads = 32; sb[0].smem = 16 << 10;
  sb[1].threads = 256; sb[1].smem = 128 << 10;
  sb[2].threads = 256; sb[2].global = true;
  // warp-per-cluster bin: at most 32 distinct A columns, table of <= kSymWarpTab slots
  constexpr int kSymWarps = 8;
  constexpr int64_t kSymWarpTab = 2048;
  std::vector<int64_t> wlist, wtsize;
  int64_t gsym = 0;
  for (int64_t c = 0; c < ncl; ++c) {
    const int64_t ts = sym_tsize(c);
    if (hcnt[c] <= 32 && ts <= kSymWarpTab) {
      wlist.push_back(c);
      wtsize.push_back(ts);
      continue;
    }
    const int which = ts * 4 <= (int64_t)sb[0].smem ? 0 : (ts * 4 <= (int64_t)sb[1].smem ? 1 : 2);
    sb[which].list.push_back(c);
    sb[which].tsize.push_back(ts);
    if (which == 2) {
      sb[2].goff.push_back(gsym);
      gsym += ts;
    }
  }
  if (!wlist.empty()) {
    PoolBuf dl(ctx), dt(ctx);
    SPOPS_TRY(h2d(st, dl, wlist));
    SPOPS_TRY(h2d(st, dt, wtsize));
    const size_t smem = (size_t)kSymWarps * kSymWarpTab * 4;
    SPOPS_CUDA(cudaFuncSetAttribute(symbolic_warp_kernel<I>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    const int64_t blocks = ((int64_t)wlist.size() + kSymWarps - 1) / kSymWarps;
    symbolic_warp_kernel<I><<<(unsigned)blocks, 32 * kSymWarps, smem, st>>>(
        dl.as<int64_t>(), (int64_t)wlist.size(), dt.as<int64_t>(), kSymWarpTab, cptr.as<int64_t>(),
        colids.as<int32_t>(), B->row.as<I>(), B->col.as<I>(), nzd.as<int64_t>(), cmin.as<int64_t>(),
        cmax.as<int64_t>());
    SPOPS_LAUNCH_CHECK();
    SPOPS_CUDA(cudaStreamSynchronize(st));
  }
  PoolBuf gtab(ctx);
  if (gsym) SPOPS_TRY(gtab.alloc((size_t)gsym * 4));
  tr.mark(st, "symbolic bins + warp kernel");
  for (int w = 0; w < 3; ++w) {
    Bin& bn = sb[w];
    if (bn.list.empty()) continue;
    PoolBuf dl(ctx), dt(ctx), dg(ctx);
    SPOPS_TRY(h2d(st, dl, bn.list));
    SPOPS_TRY(h2d(st, dt, bn.tsize));
    if (bn.global) SPOPS_TRY(h2d(st, dg, bn.goff));
    const size_t smem = bn.global ? 0 : bn.smem;
    if (smem > 48 * 1024)
      SPOPS_CUDA(cudaFuncSetAttribute(symbolic_kernel<I>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    symbolic_kernel<I><<<(unsigned)bn.list.size(), bn.threads, smem, st>>>(
        dl.as<int64_t>(), (int64_t)bn.list.size(), dt.as<int64_t>(), cptr.as<int64_t>(), colids.as<int32_t>(),
        B->row.as<I>(), B->col.as<I>(), bn.global ? gtab.as<int32_t>() : nullptr,
        bn.global ? dg.as<int64_t>() : nullptr, nzd.as<int64_t>(), cmin.as<int64_t>(), cmax.as<int64_t>());
    SPOPS_LAUNCH_CHECK();
    SPOPS_CUDA(cudaStreamSynchronize(st));
    dl.release(); dt.release(); dg.release();
  }
  gtab.release();
  std::vector<int64_t> hnz;
  SPOPS_TRY(d2h(st, hnz, nzd.p, (size_t)ncl));
  std::vector<int64_t> hccptr(ncl + 1, 0), hccptr_val(ncl + 1, 0);
  for (int64_t c = 0; c < ncl; ++c) {
    const int64_t csz = hoff[c + 1] - hoff[c];
    hccptr[c + 1] = hccptr[c] + hnz[c];
    hccptr_val[c + 1] = hccptr_val[c] + hnz[c] * csz;
  }
  if (stats) stats->symbolic_ms = tm.lap(st);
  tr.mark(st, "symbolic block kernels + nz");

  // --- classify (drop rule)
  PoolBuf drop(ctx), ndense(ctx);
  SPOPS_TRY(drop.alloc((size_t)std::max<int64_t>(ncl, 1)));
  SPOPS_TRY(ndense.alloc(8));
  SPOPS_CUDA(cudaMemsetAsync(ndense.p, 0, 8, st));
  const double b_rowdense = (double)B->nnz / (double)std::max<int64_t>(B->rows, 1);
  if (ncl > 0) {
    classify_kernel<<<grid_for(ncl), 256, 0, st>>>(cptr.as<int64_t>(), offs.as<int64_t>(), nzd.as<int64_t>(),
                                                   cmin.as<int64_t>(), cmax.as<int64_t>(), ncl, b_rowdense, l2_budget,
                                                   sort_output, sizeof(V), sizeof(int64_t), drop.as<unsigned char>(),
                                                   reinterpret_cast<unsigned long long*>(ndense.p));
    SPOPS_LAUNCH_CHECK();
  }
  int64_t hdense = 0;
  SPOPS_CUDA(cudaMemcpyAsync(&hdense, ndense.p, 8, cudaMemcpyDeviceToHost, st));

  // --- numeric bins by arena size
  PoolBuf ccptr(ctx), ccptr_val(ctx), ccol(ctx), cval(ctx);
  SPOPS_TRY(h2d(st, ccptr, hccptr));
  SPOPS_TRY(h2d(st, ccptr_val, hccptr_val));
  SPOPS_TRY(ccol.alloc((size_t)std::max<int64_t>(hccptr[ncl], 1) * 4));
  SPOPS_TRY(cval.alloc((size_t)std::max<int64_t>(hccptr_val[ncl], 1) * sizeof(V)));
  tr.mark(st, "classify + cluster output alloc");
  struct NBin {
    std::vector<int64_t> list, goff;
    std::vector<NumSlot> slots;
    int threads;
    size_t smem;
    bool global;
  };
  NBin nb[4] = {{{}, {}, {}, 32, 24 << 10, false},
                {{}, {}, {}, 128, 96 << 10, false},
                {{}, {}, {}, 256, 200 << 10, false},
                {{}, {}, {}, 256, 0, true}};
  // warp-per-cluster bins (at most 32 distinct A columns, nz <= 512): arena bytes per warp, warps per block
  struct WBin {
    std::vector<int64_t> list;
    std::vector<NumSlot> slots;
    int64_t bytes;
    int warps;
  };
  WBin wb[2] = {{{}, {}, 8 << 10, 8}, {{}, {}, 16 << 10, 4}};
  int64_t garena = 0;
  for (int64_t c = 0; c < ncl; ++c) {
    if (hnz[c] == 0) continue;
    const int64_t csz = hoff[c + 1] - hoff[c];
    NumSlot S;
    S.tsize = pow2_at_least(std::max<int64_t>(2 * hnz[c], 2));
    S.lsize = pow2_at_least(std::max<int64_t>(hnz[c], 1));
    if (hcnt[c] <= 32 && hnz[c] <= 512) {
      const int64_t wbytes = ((4 * (2 * S.tsize + hnz[c]) + 15) & ~15LL) + hnz[c] * csz * (int64_t)sizeof(V);
      int w = -1;
      for (int t = 0; t < 2 && w < 0; ++t)
        if (wbytes <= wb[t].bytes) w = t;
      if (w >= 0) {
        wb[w].list.push_back(c);
        wb[w].slots.push_back(S);
        continue;
      }
    }
    const int64_t bytes = ((hnz[c] * csz * (int64_t)sizeof(V) + 15) & ~15LL) + 4 * (2 * S.tsize + S.lsize);
    int w = 3;
    for (int t = 0; t < 3; ++t)
      if (bytes <= (int64_t)nb[t].smem) { w = t; break; }
    nb[w].list.push_back(c);
    nb[w].slots.push_back(S);
    if (w == 3) {
      nb[3].goff.push_back(garena);
      garena += (bytes + 255) & ~255LL;
    }
  }
  for (int w = 0; w < 2; ++w) {
    WBin& bn = wb[w];
    if (bn.list.empty()) continue;
    PoolBuf dl(ctx), ds(ctx);
    SPOPS_TRY(h2d(st, dl, bn.list));
    SPOPS_TRY(h2d(st, ds, bn.slots));
    const size_t smem = (size_t)bn.warps * (size_t)bn.bytes;
    SPOPS_CUDA(cudaFuncSetAttribute(numeric_warp_kernel<I, V>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    const int64_t blocks = ((int64_t)bn.list.size() + bn.warps - 1) / bn.warps;
    numeric_warp_kernel<I, V><<<(unsigned)blocks, 32 * bn.warps, smem, st>>>(
        dl.as<int64_t>(), (int64_t)bn.list.size(), ds.as<NumSlot>(), bn.bytes, cptr.as<int64_t>(),
        cptr_val.as<int64_t>(), colids.as<int32_t>(), avals.as<V>(), offs.as<int64_t>(), B->row.as<I>(),
        B->col.as<I>(), B->val.as<V>(), nzd.as<int64_t>(), ccptr.as<int64_t>(), ccptr_val.as<int64_t>(),
        drop.as<unsigned char>(), ccol.as<int32_t>(), cval.as<V>());
    SPOPS_LAUNCH_CHECK();
    SPOPS_CUDA(cudaStreamSynchronize(st));
  }
  PoolBuf arena(ctx);
  if (garena) SPOPS_TRY(arena.alloc((size_t)garena));
  tr.mark(st, "numeric bins + warp kernels");
  for (int w = 0; w < 4; ++w) {
    NBin& bn = nb[w];
    if (bn.list.empty()) continue;
    PoolBuf dl(ctx), ds(ctx), dg(ctx);
    SPOPS_TRY(h2d(st, dl, bn.list));
    SPOPS_TRY(h2d(st, ds, bn.slots));
    if (bn.global) SPOPS_TRY(h2d(st, dg, bn.goff));
    if (bn.smem > 48 * 1024)
      SPOPS_CUDA(cudaFuncSetAttribute(numeric_kernel<I, V>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bn.smem));
    numeric_kernel<I, V><<<(unsigned)bn.list.size(), bn.threads, bn.smem, st>>>(
        dl.as<int64_t>(), (int64_t)bn.list.size(), ds.as<NumSlot>(), cptr.as<int64_t>(), cptr_val.as<int64_t>(),
        colids.as<int32_t>(), avals.as<V>(), offs.as<int64_t>(), B->row.as<I>(), B->col.as<I>(), B->val.as<V>(),
        nzd.as<int64_t>(), ccptr.as<int64_t>(), ccptr_val.as<int64_t>(), drop.as<unsigned char>(),
        bn.global ? arena.as<unsigned char>() : nullptr, bn.global ? dg.as<int64_t>() : nullptr,
        ccol.as<int32_t>(), cval.as<V>());
    SPOPS_LAUNCH_CHECK();
    SPOPS_CUDA(cudaStreamSynchronize(st));
    dl.release(); ds.release(); dg.release();
  }
  arena.release();
  if (stats) stats->numeric_ms = tm.lap(st);
  tr.mark(st, "numeric block kernels");

  // --- back to CSR, original row order
  PoolBuf rowcnt(ctx), crp(ctx);
  SPOPS_TRY(rowcnt.alloc((nn + 1) * 8));
  SPOPS_TRY(crp.alloc((nn + 1) * 8));
  SPOPS_CUDA(cudaMemsetAsync(rowcnt.p, 0, (nn + 1) * 8, st));
  if (ncl > 0) {
    row_count_kernel<V><<<grid_for(ncl * 32), 256, 0, st>>>(ccptr.as<int64_t>(), ccptr_val.as<int64_t>(),
                                                            offs.as<int64_t>(), perm.as<int64_t>(), ncl, cval.as<V>(),
                                                            rowcnt.as<int64_t>());
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
  spops_status_t s = C->row.alloc((nn + 1) * sizeof(I));
  if (s == SPOPS_OK) s = C->col.alloc((size_t)std::max<int64_t>(cnnz, 1) * sizeof(I));
  if (s == SPOPS_OK) s = C->val.alloc((size_t)std::max<int64_t>(cnnz, 1) * sizeof(V));
  if (s != SPOPS_OK) {
    C->release_all();
    delete static_cast<spops_matrix_s*>(C);
    return s;
  }
  // row offsets in the index type
  tr.mark(st, "C alloc");
  std::vector<int64_t> hcrp;
  SPOPS_TRY(d2h(st, hcrp, crp.p, (size_t)n + 1));
  if (sizeof(I) == 8) {
    SPOPS_CUDA(cudaMemcpyAsync(C->row.p, crp.p, (size_t)(n + 1) * 8, cudaMemcpyDeviceToDevice, st));
  } else {
    std::vector<int32_t> r32(hcrp.begin(), hcrp.end());
    SPOPS_CUDA(cudaMemcpyAsync(C->row.p, r32.data(), r32.size() * 4, cudaMemcpyHostToDevice, st));
    SPOPS_CUDA(cudaStreamSynchronize(st));
  }
  if (ncl > 0 && cnnz > 0) {
    row_write_kernel<I, V><<<grid_for(ncl * 32), 256, 0, st>>>(ccptr.as<int64_t>(), ccptr_val.as<int64_t>(),
                                                               offs.as<int64_t>(), perm.as<int64_t>(), ncl,
                                                               ccol.as<int32_t>(), cval.as<V>(), crp.as<int64_t>(),
                                                               C->col.as<I>(), C->val.as<V>());
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
    stats->c_cluster_columns = hccptr[ncl];
  }
  *out = C;
  return SPOPS_OK;
}

}  // namespace

spops_status_t cluster_spgemm(Context* ctx, Matrix* A, Matrix* B, const int64_t* perm, const int64_t* offsets,
                              int64_t nclusters, bool sort_output, double l2_budget, Matrix** C, SpgemmStats* st) {
  if (A->format != SPOPS_FMT_CSR || B->format != SPOPS_FMT_CSR)
    return fail(SPOPS_ERR_INVALID, "SpGEMM needs CSR matrices");
  if (A->cols != B->rows) return fail(SPOPS_ERR_INVALID, "SpGEMM: A.cols (%lld) != B.rows (%lld)",
                                      (long long)A->cols, (long long)B->rows);
  if (A->itype != B->itype || A->vtype != B->vtype) return fail(SPOPS_ERR_INVALID, "SpGEMM: mixed types");
  if (B->cols > INT32_MAX || A->cols > INT32_MAX || nclusters > INT32_MAX)
    return fail(SPOPS_ERR_UNSUPPORTED, "SpGEMM: more than 2^31 columns or clusters");
  if (nclusters < 0 || offsets[0] != 0 || offsets[nclusters] != A->rows)
    return fail(SPOPS_ERR_INVALID, "SpGEMM: offsets must run from 0 to rows");
  for (int64_t c = 0; c < nclusters; ++c)
    if (offsets[c + 1] < offsets[c]) return fail(SPOPS_ERR_INVALID, "SpGEMM: offsets not monotone");
  {
    std::vector<unsigned char> seen((size_t)A->rows, 0);
    for (int64_t r = 0; r < A->rows; ++r) {
      if (perm[r] < 0 || perm[r] >= A->rows || seen[perm[r]]) return fail(SPOPS_ERR_INVALID, "SpGEMM: bad permutation");
      seen[perm[r]] = 1;
    }
  }
  if (!A->plan.ready) SPOPS_TRY(csr_analyse(ctx, A));  // validates patterns
  if (!B->plan.ready) SPOPS_TRY(csr_analyse(ctx, B));
  const bool i32 = A->itype == SPOPS_INDEX_I32, f64 = A->vtype == SPOPS_VALUE_F64;
  if (i32 && f64) return spgemm_t<int32_t, double>(ctx, A, B, perm, offsets, nclusters, sort_output, l2_budget, C, st);
  if (i32) return spgemm_t<int32_t, float>(ctx, A, B, perm, offsets, nclusters, sort_output, l2_budget, C, st);
  if (f64) return spgemm_t<int64_t, double>(ctx, A, B, perm, offsets, nclusters, sort_output, l2_budget, C, st);
  return spgemm_t<int64_t, float>(ctx, A, B, perm, offsets, nclusters, sort_output, l2_budget, C, st);
}

}  // namespace spops

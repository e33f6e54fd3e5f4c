// Sort-accumulate numeric phase of the cluster-wise SpGEMM: one warp per
// cluster, no hash table, no separate symbolic pass.
//
// For a cluster whose products (pairs of a cluster column j and an entry k of
// B's row j) number P <= 32*R, every product t (flat (j, k) order: the
// cluster's columns in order, each B row in storage order) becomes one 32-bit
// key (output column << tbits | t), held R to a lane in registers.  One
// bitonic network over the 32*R keys (blocked: lane L holds sorted positions
// L*R .. L*R+R-1) sorts them by column and, within a column, by t.  A column's
// products are then adjacent, in flat order: their values are summed along
// the sorted sequence (in each lane in order, then across lanes by a
// segmented suffix scan), so the summation order depends only on the
// matrices.  The number of distinct columns, their min and max come from the
// same sorted keys, which settles the reference's dense/hash classification
// (src/spgemm_Vlength_mixed.cpp:267-319) and its drop rule for the cluster
// without a symbolic pass.
//
// Each product's B value (its A value too, for a one-row cluster: then the
// product itself) and its cluster column are parked in the warp's slice of
// dynamic shared memory at index t while the keys are built, so that after
// the sort a key's low bits find its operands with one shared-memory read.
//
// Output goes to the cluster's slab: ccol[soff[c] ..], cval[soff_val[c] ..]
// (room for P columns), columns ascending, values [column x csz] with the
// rows of the cluster interleaved -- the same layout the hash kernels write.
//
// Limits (the caller bins clusters accordingly): P <= 32*R (R <= 16), the cluster has
// at most kSortCols columns, and B's column count fits the key
// (cols <= 2^(32 - tbits) - 1, tbits = log2(32*R)).
#pragma once

#include <cstdint>

namespace spops {
namespace {

constexpr int kSortCols = 256;  // cluster columns staged per warp
constexpr int kSortWarps = 4;   // warps per block

// dynamic shared memory of sort_accum_kernel<I, V, R>: per warp 32R values
// and 32R one-byte cluster columns
template <typename V, int R>
constexpr size_t sort_accum_smem() {
  return (size_t)kSortWarps * 32 * R * (sizeof(V) + 1);
}

// Ascending bitonic sort of 32*R keys, blocked: element e = lane*R + s.
// Stages are instantiated by template recursion so that every partner slot
// index is a compile-time constant and the keys stay in registers.
template <int R, int KK, int JJ>
__device__ __forceinline__ void bitonic_stage(uint32_t (&k)[R], int lane) {
  constexpr int N = 32 * R;
  if constexpr (JJ >= R) {  // partner: lane ^ (JJ / R), same slot
    constexpr int lm = JJ / R;
    const bool lower = (lane & lm) == 0;
    const bool asc = (KK >= N) ? true : ((lane & (KK / R)) == 0);
    const bool keep_min = lower == asc;
#pragma unroll
    for (int s = 0; s < R; ++s) {
      const uint32_t o = __shfl_xor_sync(0xffffffffu, k[s], lm);
      k[s] = keep_min ? min(k[s], o) : max(k[s], o);
    }
  } else {  // partner: slot s ^ JJ of the same lane
    const bool lane_asc = (KK >= N) ? true : ((lane & (KK / R)) == 0);
#pragma unroll
    for (int s = 0; s < R; ++s) {
      const int p = s ^ JJ;
      if (p > s) {
        const bool asc = KK < R ? (s & KK) == 0 : lane_asc;
        const uint32_t a = k[s], b = k[p];
        const uint32_t lo = min(a, b), hi = max(a, b);
        k[s] = asc ? lo : hi;
        k[p] = asc ? hi : lo;
      }
    }
  }
  if constexpr (JJ > 1) bitonic_stage<R, KK, JJ / 2>(k, lane);
}

template <int R, int KK>
__device__ __forceinline__ void bitonic_pass(uint32_t (&k)[R], int lane) {
  bitonic_stage<R, KK, KK / 2>(k, lane);
  if constexpr (KK < 32 * R) bitonic_pass<R, KK * 2>(k, lane);
}

// One warp's bitonic sort of its 32*R keys, R <= 16 (larger sorts run on
// several warps, sort_accum_multi_kernel).
template <int R>
__device__ __forceinline__ void warp_bitonic_sort(uint32_t (&k)[R], int lane) {
  static_assert(R >= 1 && R <= 16 && (R & (R - 1)) == 0, "R: a power of two up to 16");
  bitonic_pass<R, 2>(k, lane);
}

template <typename I, typename V, int R>
__global__ void __launch_bounds__(32 * kSortWarps)
    sort_accum_kernel(const int64_t* __restrict__ list, int64_t nlist, const int64_t* __restrict__ cptr,
                      const int64_t* __restrict__ cptr_val, const int32_t* __restrict__ colids,
                      const V* __restrict__ avals, const int64_t* __restrict__ offsets, const I* __restrict__ brp,
                      const I* __restrict__ bci, const V* __restrict__ bv, int tbits, double b_rowdense,
                      double budget, bool sort_output, bool rowwise, const int64_t* __restrict__ soff,
                      const int64_t* __restrict__ soff_val, int64_t* __restrict__ nz, int64_t* __restrict__ cmin,
                      int64_t* __restrict__ cmax, unsigned char* __restrict__ drop_out,
                      unsigned long long* __restrict__ ndense, int32_t* __restrict__ ccol, V* __restrict__ cval) {
  __shared__ int32_t s_off[kSortWarps][kSortCols + 1];
  __shared__ int64_t s_start[kSortWarps][kSortCols];
  extern __shared__ __align__(16) unsigned char sort_dyn_smem[];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  V* pv = reinterpret_cast<V*>(sort_dyn_smem) + (size_t)w * 32 * R;  // per product: value or B value
  unsigned char* pj = sort_dyn_smem + (size_t)kSortWarps * 32 * R * sizeof(V) + (size_t)w * 32 * R;  // its column
  const int64_t b = blockIdx.x * (int64_t)kSortWarps + w;
  if (b >= nlist) return;
  const int64_t c = list[b];
  const int64_t csz = offsets[c + 1] - offsets[c];
  const int64_t j0 = cptr[c];
  const int nj = (int)(cptr[c + 1] - j0);
  int32_t* off = s_off[w];
  int64_t* start = s_start[w];
  // B row starts of the cluster's columns and the products before each
  int32_t carry = 0;
  for (int t0 = 0; t0 < nj; t0 += 32) {
    const int t = t0 + lane;
    int32_t len = 0;
    if (t < nj) {
      const int64_t r = colids[j0 + t];
      const int64_t st = brp[r];
      start[t] = st;
      len = (int32_t)((int64_t)brp[r + 1] - st);
    }
    int32_t inc = len;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int32_t u = __shfl_up_sync(0xffffffffu, inc, o);
      if (lane >= o) inc += u;
    }
    if (t < nj) off[t + 1] = carry + inc;
    carry += __shfl_sync(0xffffffffu, inc, 31);
  }
  if (lane == 0) off[0] = 0;
  __syncwarp();
  const int32_t P = off[nj];
  // keys: slot s of this lane holds product t = s*32 + lane before sorting
  constexpr uint32_t kNone = 0xffffffffu;
  const int64_t vbase = cptr_val[c];
  uint32_t key[R];
  {
    int j = 0;
#pragma unroll
    for (int s = 0; s < R; ++s) {
      const int32_t t = s * 32 + lane;
      key[s] = kNone;
      if (t < P) {
        while (off[j + 1] <= t) ++j;
        const int64_t k = start[j] + (t - off[j]);
        key[s] = ((uint32_t)bci[k] << tbits) | (uint32_t)t;
        const V b = bv[k];
        if (csz == 1) {
          pv[t] = avals[vbase + j] * b;
        } else {
          pv[t] = b;
          pj[t] = (unsigned char)j;
        }
      }
    }
  }
  __syncwarp();
  warp_bitonic_sort<R>(key, lane);
  const uint32_t tmask = (1u << tbits) - 1u;
  // column starts in this lane's sorted run; the distinct-column count
  const uint32_t prev_last = __shfl_up_sync(0xffffffffu, key[R - 1], 1);
  unsigned long long first = 0;  // bit s: sorted position lane*R + s starts a column
  int cnt = 0;
#pragma unroll
  for (int s = 0; s < R; ++s) {
    const uint32_t prev = s == 0 ? (lane == 0 ? kNone : prev_last) : key[s - 1];
    const bool f = key[s] != kNone && (s == 0 && lane == 0 ? true : (prev >> tbits) != (key[s] >> tbits));
    first |= (f ? 1ULL : 0ULL) << s;
    cnt += f ? 1 : 0;
  }
  int incl = cnt;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int u = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += u;
  }
  const int base = incl - cnt;  // rank of this lane's first column start
  const int64_t nzc = __shfl_sync(0xffffffffu, incl, 31);
  int64_t mx = -1;
#pragma unroll
  for (int s = 0; s < R; ++s)
    if (key[s] != kNone) mx = (int64_t)(key[s] >> tbits);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) mx = max(mx, __shfl_xor_sync(0xffffffffu, mx, o));
  const int64_t mn = (int64_t)(__shfl_sync(0xffffffffu, key[0], 0) >> tbits);
  // the reference's classification (the same arithmetic as classify_kernel)
  bool dense = false;
  if (nzc > 0) {
    const int64_t range = mx - mn + 1;
    const double density = (double)nzc / (double)range;
    const size_t b_access = (size_t)((double)nj * b_rowdense * (double)(sizeof(int64_t) + sizeof(V)));
    const size_t dense_bytes = (size_t)range * (size_t)csz * sizeof(V);
    dense = (double)(b_access + dense_bytes) <= budget && density >= 0.15;
  }
  const bool drop = !rowwise && (dense || sort_output);
  if (lane == 0) {
    nz[c] = nzc;
    cmin[c] = nzc ? mn : 0;
    cmax[c] = nzc ? mx : 0;
    drop_out[c] = drop ? 1 : 0;
    if (dense && !rowwise) atomicAdd(ndense, 1ULL);
  }
  const int64_t co = soff[c], cvo = soff_val[c];
  // output columns
  {
    int r = base;
#pragma unroll
    for (int s = 0; s < R; ++s)
      if (first >> s & 1ULL) ccol[co + r++] = (int32_t)(key[s] >> tbits);
  }
  // values, one row of the cluster at a time
  for (int64_t l = 0; l < csz; ++l) {
    V head = V(0), run = V(0);
    bool seen = false;
    int r = base - 1;
#pragma unroll
    for (int s = 0; s < R; ++s) {
      if (key[s] != kNone) {
        const int32_t t = (int32_t)(key[s] & tmask);
        const V v = csz == 1 ? pv[t] : avals[vbase + (int64_t)pj[t] * csz + l] * pv[t];
        if (first >> s & 1ULL) {
          if (seen) {
            const V o = (csz == 1 && drop && fabs((double)run) < 1e-12) ? V(0) : run;
            cval[cvo + (int64_t)r * csz + l] = o;
          }
          seen = true;
          run = v;
          ++r;
        } else if (seen) {
          run += v;
        } else {
          head += v;
        }
      }
    }
    // the sums of the lanes after this one that continue its last column:
    // S[L] = head[L] + (lane L starts a column ? 0 : S[L+1])
    V S = head;
    bool stop = seen;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const V ov = __shfl_down_sync(0xffffffffu, S, o);
      const bool os = __shfl_down_sync(0xffffffffu, stop ? 1 : 0, o) != 0;
      if (lane + o < 32 && !stop) {
        S += ov;
        stop = os;
      }
    }
    V next = __shfl_down_sync(0xffffffffu, S, 1);
    if (lane == 31) next = V(0);
    if (seen) {
      const V tot = run + next;
      const V o = (csz == 1 && drop && fabs((double)tot) < 1e-12) ? V(0) : tot;
      cval[cvo + (int64_t)r * csz + l] = o;
    }
  }
  if (csz > 1 && drop) {  // a column is zeroed when all its rows fall below 1e-12
    for (int r = base; r < base + cnt; ++r) {
      bool small = true;
      for (int64_t l = 0; l < csz; ++l)
        if (fabs((double)cval[cvo + (int64_t)r * csz + l]) >= 1e-12) {
          small = false;
          break;
        }
      if (small)
        for (int64_t l = 0; l < csz; ++l) cval[cvo + (int64_t)r * csz + l] = V(0);
    }
  }
}

// ---------------------------------------------------------------------------
// Clusters with 512 < P <= 512 W products: W warps of one block take one
// cluster, 16 keys per lane each (N = 512 W keys).  Each warp sorts its 512
// keys (ascending or descending by warp parity, as the bitonic network wants
// at that size), then the merge levels above 512 run their cross-warp stages
// through shared memory and their in-warp stages in registers.  The sorted
// sequence is blocked: warp w, lane L, slot s holds position
// w * 512 + L * 16 + s.  The per-column sums chain across lanes as in the
// one-warp kernel and across warps through shared memory, in a fixed order.
constexpr int kMultiR = 16;        // keys per lane in the multi-warp kernel
constexpr int kMultiCols = 1024;   // cluster columns it stages

// dynamic shared memory of sort_accum_multi_kernel<I, V, W>
template <typename V, int W>
constexpr size_t sort_multi_smem() {
  constexpr size_t N = (size_t)32 * kMultiR * W;
  return N * sizeof(V)                        // product operand per product
         + N * 4                              // key exchange between warps
         + N * 2                              // cluster column per product
         + (size_t)kMultiCols * 8             // B row starts of the columns
         + ((size_t)kMultiCols + 1) * 4       // products before each column
         + (size_t)W * 32;                    // per-warp scalars
}

// Bitonic merge of a bitonic sequence of one warp's 32R keys (blocked), in
// the direction asc: stages JJ = 16R .. 1.
template <int R, int JJ>
__device__ __forceinline__ void warp_merge_stage(uint32_t (&k)[R], int lane, bool asc) {
  if constexpr (JJ >= R) {  // partner: lane ^ (JJ / R), same slot
    constexpr int lm = JJ / R;
    const bool keep_min = ((lane & lm) == 0) == asc;
#pragma unroll
    for (int s = 0; s < R; ++s) {
      const uint32_t o = __shfl_xor_sync(0xffffffffu, k[s], lm);
      k[s] = keep_min ? min(k[s], o) : max(k[s], o);
    }
  } else {  // partner: slot s ^ JJ of the same lane
#pragma unroll
    for (int s = 0; s < R; ++s) {
      const int p = s ^ JJ;
      if (p > s) {
        const uint32_t a = k[s], b = k[p];
        const uint32_t lo = min(a, b), hi = max(a, b);
        k[s] = asc ? lo : hi;
        k[p] = asc ? hi : lo;
      }
    }
  }
  if constexpr (JJ > 1) warp_merge_stage<R, JJ / 2>(k, lane, asc);
}

template <typename I, typename V, int W>
__global__ void __launch_bounds__(32 * W)
    sort_accum_multi_kernel(const int64_t* __restrict__ list, int64_t nlist, const int64_t* __restrict__ cptr,
                            const int64_t* __restrict__ cptr_val, const int32_t* __restrict__ colids,
                            const V* __restrict__ avals, const int64_t* __restrict__ offsets,
                            const I* __restrict__ brp, const I* __restrict__ bci, const V* __restrict__ bv,
                            int tbits, double b_rowdense, double budget, bool sort_output, bool rowwise,
                            const int64_t* __restrict__ soff, const int64_t* __restrict__ soff_val,
                            int64_t* __restrict__ nz, int64_t* __restrict__ cmin, int64_t* __restrict__ cmax,
                            unsigned char* __restrict__ drop_out, unsigned long long* __restrict__ ndense,
                            int32_t* __restrict__ ccol, V* __restrict__ cval) {
  constexpr int R = kMultiR;
  constexpr int NW = 32 * R;  // keys per warp
  constexpr int N = NW * W;
  constexpr uint32_t kNone = 0xffffffffu;
  extern __shared__ __align__(16) unsigned char multi_smem[];
  V* pv = reinterpret_cast<V*>(multi_smem);
  uint32_t* xk = reinterpret_cast<uint32_t*>(pv + N);
  uint16_t* pj = reinterpret_cast<uint16_t*>(xk + N);
  int64_t* start = reinterpret_cast<int64_t*>(multi_smem + (size_t)N * (sizeof(V) + 4 + 2));
  int32_t* off = reinterpret_cast<int32_t*>(start + kMultiCols);
  // per-warp scalars: last key, column count, max column, chain value, chain stop
  uint32_t* w_last = reinterpret_cast<uint32_t*>(off + kMultiCols + 1);
  int32_t* w_cnt = reinterpret_cast<int32_t*>(w_last + W);
  int64_t* w_max = reinterpret_cast<int64_t*>(((uintptr_t)(w_cnt + W) + 7) & ~(uintptr_t)7);
  V* w_s0 = reinterpret_cast<V*>(w_max + W);
  int32_t* w_stop = reinterpret_cast<int32_t*>(w_s0 + W);
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  if (blockIdx.x >= nlist) return;
  const int64_t c = list[blockIdx.x];
  const int64_t csz = offsets[c + 1] - offsets[c];
  const int64_t j0 = cptr[c];
  const int nj = (int)(cptr[c + 1] - j0);
  // B row starts of the cluster's columns and the products before each (warp 0)
  if (w == 0) {
    int32_t carry = 0;
    for (int t0 = 0; t0 < nj; t0 += 32) {
      const int t = t0 + lane;
      int32_t len = 0;
      if (t < nj) {
        const int64_t r = colids[j0 + t];
        const int64_t st = brp[r];
        start[t] = st;
        len = (int32_t)((int64_t)brp[r + 1] - st);
      }
      int32_t inc = len;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const int32_t u = __shfl_up_sync(0xffffffffu, inc, o);
        if (lane >= o) inc += u;
      }
      if (t < nj) off[t + 1] = carry + inc;
      carry += __shfl_sync(0xffffffffu, inc, 31);
    }
    if (lane == 0) off[0] = 0;
  }
  __syncthreads();
  const int32_t P = off[nj];
  const int64_t vbase = cptr_val[c];
  // keys: warp w, slot s of lane L holds product t = (w * R + s) * 32 + L
  uint32_t key[R];
  {
    const int32_t tfirst = w * NW + lane;
    int lo = 0, hi = nj;  // the column holding product tfirst
    while (hi - lo > 1) {
      const int mid = (lo + hi) >> 1;
      if (off[mid] <= tfirst) lo = mid; else hi = mid;
    }
    int j = lo;
#pragma unroll
    for (int s = 0; s < R; ++s) {
      const int32_t t = (w * R + s) * 32 + lane;
      key[s] = kNone;
      if (t < P) {
        while (off[j + 1] <= t) ++j;
        const int64_t k = start[j] + (t - off[j]);
        key[s] = ((uint32_t)bci[k] << tbits) | (uint32_t)t;
        const V b = bv[k];
        if (csz == 1) {
          pv[t] = avals[vbase + j] * b;
        } else {
          pv[t] = b;
          pj[t] = (uint16_t)j;
        }
      }
    }
  }
  __syncthreads();  // operands parked
  // sort: warp w's 512 keys in the direction the network wants at size 512
  // (descending for odd w: sorting the complements ascending), then the
  // merge levels 1024 .. N
  {
    const bool desc = (w & 1) != 0;
    if (desc) {
#pragma unroll
      for (int s = 0; s < R; ++s) key[s] = ~key[s];
    }
    warp_bitonic_sort<R>(key, lane);
    if (desc) {
#pragma unroll
      for (int s = 0; s < R; ++s) key[s] = ~key[s];
    }
  }
#pragma unroll 1
  for (int kk = 2 * NW; kk <= N; kk <<= 1) {
    const bool asc = kk >= N ? true : ((w & (kk / NW)) == 0);
#pragma unroll 1
    for (int jj = kk >> 1; jj >= NW; jj >>= 1) {  // partner: warp w ^ (jj / NW), same lane and slot
      const int pw = w ^ (jj / NW);
      const bool keep_min = ((w & (jj / NW)) == 0) == asc;
#pragma unroll
      for (int s = 0; s < R; ++s) xk[w * NW + s * 32 + lane] = key[s];
      __syncthreads();
#pragma unroll
      for (int s = 0; s < R; ++s) {
        const uint32_t o = xk[pw * NW + s * 32 + lane];
        key[s] = keep_min ? min(key[s], o) : max(key[s], o);
      }
      __syncthreads();
    }
    warp_merge_stage<R, NW / 2>(key, lane, asc);
  }
  const uint32_t tmask = (1u << tbits) - 1u;
  // the key before this lane's first slot: the previous lane's last, or for
  // lane 0 the previous warp's last
  if (lane == 31) w_last[w] = key[R - 1];
  __syncthreads();
  uint32_t prev_last = __shfl_up_sync(0xffffffffu, key[R - 1], 1);
  if (lane == 0) prev_last = w > 0 ? w_last[w - 1] : kNone;
  const bool global_first = w == 0 && lane == 0;
  uint32_t first = 0;  // bit s: position (w, lane, s) starts a column
  int cnt = 0;
#pragma unroll
  for (int s = 0; s < R; ++s) {
    const uint32_t prev = s == 0 ? prev_last : key[s - 1];
    const bool f = key[s] != kNone && ((s == 0 && global_first) || (prev >> tbits) != (key[s] >> tbits));
    first |= (f ? 1u : 0u) << s;
    cnt += f ? 1 : 0;
  }
  int incl = cnt;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int u = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += u;
  }
  int64_t mx = -1;
#pragma unroll
  for (int s = 0; s < R; ++s)
    if (key[s] != kNone) mx = (int64_t)(key[s] >> tbits);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) mx = max(mx, __shfl_xor_sync(0xffffffffu, mx, o));
  if (lane == 31) w_cnt[w] = incl;
  if (lane == 0) w_max[w] = mx;
  __syncthreads();
  int wbase = 0, nzi = 0;
  for (int v = 0; v < W; ++v) {
    if (v < w) wbase += w_cnt[v];
    nzi += w_cnt[v];
    mx = max(mx, w_max[v]);
  }
  const int base = wbase + incl - cnt;  // rank of this lane's first column start
  const int64_t nzc = nzi;
  const int64_t mn = nzc ? (int64_t)(__shfl_sync(0xffffffffu, key[0], 0) >> tbits) : 0;  // valid in warp 0
  // the reference's classification (the same arithmetic as classify_kernel)
  bool dense = false;
  if (w == 0 && nzc > 0) {
    const int64_t range = mx - mn + 1;
    const double density = (double)nzc / (double)range;
    const size_t b_access = (size_t)((double)nj * b_rowdense * (double)(sizeof(int64_t) + sizeof(V)));
    const size_t dense_bytes = (size_t)range * (size_t)csz * sizeof(V);
    dense = (double)(b_access + dense_bytes) <= budget && density >= 0.15;
  }
  if (w == 0 && lane == 0) {
    nz[c] = nzc;
    cmin[c] = nzc ? mn : 0;
    cmax[c] = nzc ? mx : 0;
    drop_out[c] = (!rowwise && (dense || sort_output)) ? 1 : 0;
    if (dense && !rowwise) atomicAdd(ndense, 1ULL);
    w_stop[0] = dense ? 1 : 0;  // (reused below) the classification for the other warps
  }
  __syncthreads();
  dense = w_stop[0] != 0;
  const bool drop = !rowwise && (dense || sort_output);
  const int64_t co = soff[c], cvo = soff_val[c];
  {
    int r = base;
#pragma unroll
    for (int s = 0; s < R; ++s)
      if (first >> s & 1u) ccol[co + r++] = (int32_t)(key[s] >> tbits);
  }
  __syncthreads();  // w_stop is reused by the value chains
  // values, one row of the cluster at a time
  for (int64_t l = 0; l < csz; ++l) {
    V head = V(0), run = V(0);
    bool seen = false;
    int r = base - 1;
#pragma unroll
    for (int s = 0; s < R; ++s) {
      if (key[s] != kNone) {
        const int32_t t = (int32_t)(key[s] & tmask);
        const V v = csz == 1 ? pv[t] : avals[vbase + (int64_t)pj[t] * csz + l] * pv[t];
        if (first >> s & 1u) {
          if (seen) {
            const V o = (csz == 1 && drop && fabs((double)run) < 1e-12) ? V(0) : run;
            cval[cvo + (int64_t)r * csz + l] = o;
          }
          seen = true;
          run = v;
          ++r;
        } else if (seen) {
          run += v;
        } else {
          head += v;
        }
      }
    }
    // within the warp: S[L] = head[L] + (lane L starts a column ? 0 : S[L+1])
    V S = head;
    bool stop = seen;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const V ov = __shfl_down_sync(0xffffffffu, S, o);
      const bool os = __shfl_down_sync(0xffffffffu, stop ? 1 : 0, o) != 0;
      if (lane + o < 32 && !stop) {
        S += ov;
        stop = os;
      }
    }
    // across warps: X = what the lanes of this warp that reach its end
    // continue into (the following warps' heads up to the first warp with a
    // column start), added from the far end
    if (lane == 0) {
      w_s0[w] = S;
      w_stop[w] = stop ? 1 : 0;
    }
    __syncthreads();
    V X = V(0);
    if (w + 1 < W) {
      int m = w + 1;
      while (m + 1 < W && !w_stop[m]) ++m;
      X = w_s0[m];
      for (int v = m - 1; v > w; --v) X = w_s0[v] + X;
    }
    __syncthreads();  // w_s0 / w_stop are rewritten for the next row
    if (!stop) S += X;
    V next = __shfl_down_sync(0xffffffffu, S, 1);
    if (lane == 31) next = X;
    if (seen) {
      const V tot = run + next;
      const V o = (csz == 1 && drop && fabs((double)tot) < 1e-12) ? V(0) : tot;
      cval[cvo + (int64_t)r * csz + l] = o;
    }
  }
  if (csz > 1 && drop) {  // a column is zeroed when all its rows fall below 1e-12
    for (int r = base; r < base + cnt; ++r) {
      bool small = true;
      for (int64_t l = 0; l < csz; ++l)
        if (fabs((double)cval[cvo + (int64_t)r * csz + l]) >= 1e-12) {
          small = false;
          break;
        }
      if (small)
        for (int64_t l = 0; l < csz; ++l) cval[cvo + (int64_t)r * csz + l] = V(0);
    }
  }
}

}  // namespace
}  // namespace spops

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
//      the first top_k kept, the diagonal excluded: for top_k <= 32 a warp
//      per row selects them in registers, else one stable segmented radix
//      sort of a descending key with the columns in ascending order as
//      payload.  Rows of the result are in that order, as the reference's.
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

// Top-k (k <= 32) without sorting every entry: one warp per row of the
// intersection counts keeps the row's best 32 entries so far sorted across
// the lanes (lane l holds the l-th best).  Only entries that rank before the
// current k-th best are kept as candidates, compacted into a per-warp buffer
// in shared memory; each time 32 are there they are sorted and merged into
// the best 32 (lane l keeps the better of best[l] and cand[31 - l], which
// leaves the best 32 of both as a bitonic sequence; five steps sort it) and
// the k-th best moves up.  An entry that does not beat the k-th best when it
// is read ranks after k entries of the row, so the filter drops nothing of
// the result; the candidates left at the end of the row are merged last.
// A random order of m entries brings about k ln(m / k) candidates, so most
// chunks of 32 entries cost a ballot instead of a 32-wide sort.  Two chunks
// are read per step to keep more loads in flight.  The first k of the row go
// to tkey / tcol at row * k, and kept[row] = min(k, entries - diagonal).
constexpr int kSelectWarps = 8;

template <typename I, typename V>
__global__ void __launch_bounds__(kSelectWarps * 32)
    topk_select_kernel(const I* __restrict__ crp, const I* __restrict__ cci, const V* __restrict__ cval,
                       const I* __restrict__ arp, int64_t n, int k, uint64_t* __restrict__ tkey,
                       I* __restrict__ tcol, int64_t* __restrict__ kept) {
  __shared__ uint64_t s_key[kSelectWarps][64];
  __shared__ int64_t s_col[kSelectWarps][64];
  const int64_t i = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;  // one row per warp
  const int lane = threadIdx.x & 31;
  if (i >= n || k <= 0) return;  // kept[] is zeroed by the caller
  uint64_t* const buf_k = s_key[threadIdx.x >> 5];
  int64_t* const buf_c = s_col[threadIdx.x >> 5];
  const unsigned below = (1u << lane) - 1u;
  const int64_t e0 = crp[i], e1 = crp[i + 1];
  const int64_t li = (int64_t)arp[i + 1] - (int64_t)arp[i];
  uint64_t bk = kDiagKey;  // padding sorts after every entry, the diagonal included
  int64_t bc = INT64_MAX;
  uint64_t tk = kDiagKey;  // the k-th best so far: a candidate must rank before it
  int64_t tc = INT64_MAX;
  int nbuf = 0, diag = 0;
  auto merge = [&](uint64_t ck, int64_t cc) {
    warp_sort32(ck, cc);
    const uint64_t rk = __shfl_sync(0xffffffffu, ck, 31 - lane);
    const int64_t rc = __shfl_sync(0xffffffffu, cc, 31 - lane);
    if (rank_less(rk, rc, bk, bc)) {
      bk = rk;
      bc = rc;
    }
    for (int j = 16; j > 0; j >>= 1) warp_cx(bk, bc, j, true);
    tk = __shfl_sync(0xffffffffu, bk, k - 1);
    tc = __shfl_sync(0xffffffffu, bc, k - 1);
  };
  auto offer = [&](uint64_t key, int64_t col, bool ok) {
    const bool cand = ok && rank_less(key, col, tk, tc);
    const unsigned m = __ballot_sync(0xffffffffu, cand);
    if (cand) {
      const int p = nbuf + __popc(m & below);  // nbuf <= 31 before, so p <= 62
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
  };
  auto entry_key = [&](int64_t col, V inter) {
    const int64_t u = li + ((int64_t)arp[col + 1] - (int64_t)arp[col]) - (int64_t)inter;
    return desc_key(u == 0 ? V(0) : V(1) * inter / (V)u);
  };
  for (int64_t base = e0; base < e1; base += 64) {
    const int64_t ea = base + lane, eb = ea + 32;
    const bool ha = ea < e1, hb = eb < e1;
    const int64_t ca = ha ? (int64_t)cci[ea] : -1, cb = hb ? (int64_t)cci[eb] : -1;
    const V va = ha ? cval[ea] : V(0), vb = hb ? cval[eb] : V(0);
    const bool oa = ha && ca != i, ob = hb && cb != i;
    diag |= (ha && ca == i) || (hb && cb == i);
    const uint64_t ka = oa ? entry_key(ca, va) : kDiagKey;
    const uint64_t kb = ob ? entry_key(cb, vb) : kDiagKey;
    offer(ka, ca, oa);
    offer(kb, cb, ob);
  }
  if (nbuf > 0) {
    __syncwarp();
    const uint64_t ck = lane < nbuf ? buf_k[lane] : kDiagKey;
    const int64_t cc = lane < nbuf ? buf_c[lane] : INT64_MAX;
    merge(ck, cc);
  }
  diag = __any_sync(0xffffffffu, diag);
  if (lane < k) {
    tkey[i * k + lane] = bk;
    tcol[i * k + lane] = (I)(bc == INT64_MAX ? 0 : bc);
  }
  if (lane == 0) {
    const int64_t avail = e1 - e0 - diag;
    kept[i] = avail < k ? avail : k;
  }
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

template <typename I, typename V>
spops_status_t topk_t(Context* ctx, Matrix* A, int64_t top_k, Matrix** out) {
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
  // 3. keys and the best k per row: a warp selection for k <= 32, else a
  //    per-row stable sort
  ArenaScope scope(ctx);  // this call's temporaries come from the arena
  PoolBuf key(ctx), skey(ctx), col(ctx), scol(ctx), diag(ctx), kept(ctx), orp(ctx), tmp(ctx);
  if (top_k <= 32) {
    const int k = (int)std::max<int64_t>(top_k, 0);
    const size_t nk = (size_t)std::max<int64_t>(n * k, 1);
    SPOPS_TRY(skey.alloc(nk * 8));
    SPOPS_TRY(scol.alloc(nk * sizeof(I)));
    SPOPS_TRY(kept.alloc((size_t)(n + 1) * 8));
    SPOPS_TRY(orp.alloc((size_t)(n + 1) * 8));
    SPOPS_CUDA(cudaMemsetAsync(kept.p, 0, (size_t)(n + 1) * 8, st));
    if (n > 0) {
      topk_select_kernel<I, V><<<grid_for(n * 32), kSelectWarps * 32, 0, st>>>(Cn->row.as<I>(), Cn->col.as<I>(), Cn->val.as<V>(),
                                                                 A->row.as<I>(), n, k, skey.as<uint64_t>(),
                                                                 scol.as<I>(), kept.as<int64_t>());
      SPOPS_LAUNCH_CHECK();
    }
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
    return SPOPS_OK;
  }
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

// COO -> CSR on the device, with the reference's duplicate summation.
//
// Replaces coo_to_csr (reference include/sparse_conversion.h:37-99): rows by
// a counting sort that keeps the file order of the entries within a row
// (here a stable radix sort by row, done once by the COO handle's analysis).
// With compact = true the reference then runs sum_csr_duplicates
// (include/sparse_operation.h:21-69), which, row by row, adds the values of
// equal columns in file order, lists the distinct columns in REVERSE order of
// their first appearance (it pushes every new column on the front of a
// list), and drops columns whose sum is exactly zero.  The device version
// reproduces that result bit for bit:
//   1. stable sort of (row, column) keys carrying the entry position;
//   2. one thread per (row, column) group adds its values in file order,
//      starting from zero, and records the group's first position;
//   3. groups with a non-zero sum are sorted by (row, first position
//      descending) and written out; row offsets from per-row counts.
#include <cub/cub.cuh>

#include <algorithm>
#include <cstring>

#include "spops_internal.h"

namespace spops {
namespace {

inline unsigned grid_of(int64_t work, int threads = 256) {
  int64_t g = (work + threads - 1) / threads;
  return (unsigned)(g < 1 ? 1 : g);
}

template <typename I>
__global__ void entry_key_kernel(const I* __restrict__ rp, int64_t n, const I* __restrict__ ci,
                                 uint64_t* __restrict__ key, int64_t* __restrict__ pos) {
  const int64_t r = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (r >= n) return;
  for (int64_t e = (int64_t)rp[r] + lane; e < (int64_t)rp[r + 1]; e += 32) {
    key[e] = ((uint64_t)r << 32) | (uint64_t)(uint32_t)ci[e];
    pos[e] = e;
  }
}

__global__ void group_flag_kernel(const uint64_t* __restrict__ key, int64_t m, int64_t* __restrict__ flag) {
  const int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (e < m) flag[e] = (e == 0 || key[e] != key[e - 1]) ? 1 : 0;
}

// group g = entries [start[g], start[g+1]) of the sorted keys
__global__ void group_start_kernel(const int64_t* __restrict__ flag, const int64_t* __restrict__ gid, int64_t m,
                                   int64_t* __restrict__ start) {
  const int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (e < m && flag[e]) start[gid[e] - 1] = e;
  if (e == 0) start[gid[m - 1]] = m;
}

template <typename I, typename V>
__global__ void group_sum_kernel(const uint64_t* __restrict__ key, const int64_t* __restrict__ pos,
                                 const int64_t* __restrict__ start, int64_t ngroups, const I* __restrict__ rp,
                                 const V* __restrict__ val, V* __restrict__ gsum, uint64_t* __restrict__ okey,
                                 int64_t* __restrict__ gidx, unsigned long long* __restrict__ kept,
                                 unsigned long long* __restrict__ rowcnt) {
  const int64_t g = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (g >= ngroups) return;
  const int64_t a = start[g], b = start[g + 1];
  V s = V(0);
  for (int64_t t = a; t < b; ++t) s += val[pos[t]];  // file order: positions ascend within a group
  gsum[g] = s;
  if (s != V(0)) {
    const uint64_t r = key[a] >> 32;
    const uint64_t first = (uint64_t)(pos[a] - (int64_t)rp[r]);  // position within the row
    const unsigned long long slot = atomicAdd(kept, 1ULL);
    okey[slot] = (r << 32) | (uint64_t)(0xffffffffu - (uint32_t)first);
    gidx[slot] = g;
    atomicAdd(rowcnt + r, 1ULL);
  }
}

template <typename I, typename V>
__global__ void compact_write_kernel(const uint64_t* __restrict__ key, const int64_t* __restrict__ start,
                                     const int64_t* __restrict__ gidx_sorted, const V* __restrict__ gsum, int64_t m,
                                     I* __restrict__ col, V* __restrict__ val) {
  const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (t >= m) return;
  const int64_t g = gidx_sorted[t];
  col[t] = (I)(uint32_t)(key[start[g]] & 0xffffffffu);
  val[t] = gsum[g];
}

template <typename I>
__global__ void offsets_kernel(const unsigned long long* __restrict__ scan, int64_t n1, I* __restrict__ rp) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i < n1) rp[i] = (I)scan[i];
}

Matrix* new_csr(Context* ctx, const Matrix* like, int64_t nnz) {
  Matrix* C = new Matrix();
  C->ctx = ctx;
  C->format = SPOPS_FMT_CSR;
  C->itype = like->itype;
  C->vtype = like->vtype;
  C->rows = like->rows;
  C->cols = like->cols;
  C->nnz = nnz;
  return C;
}

template <typename I, typename V>
spops_status_t coo_to_csr_t(Context* ctx, Matrix* coo, bool compact, Matrix** out) {
  cudaStream_t st = ctx->stream;
  if (!coo->csr_view) SPOPS_TRY(coo_analyse(ctx, coo));
  const Matrix* S = coo->csr_view;  // rows sorted, file order within rows
  const int64_t n = S->rows, nz = S->nnz;
  const size_t n1 = (size_t)n + 1;
  if (!compact) {
    Matrix* C = new_csr(ctx, S, nz);
    spops_status_t s = C->row.alloc(n1 * sizeof(I));
    if (s == SPOPS_OK) s = C->col.alloc((size_t)std::max<int64_t>(nz, 1) * sizeof(I));
    if (s == SPOPS_OK) s = C->val.alloc((size_t)std::max<int64_t>(nz, 1) * sizeof(V));
    if (s == SPOPS_OK) {
      SPOPS_CUDA(cudaMemcpyAsync(C->row.p, S->row.p, n1 * sizeof(I), cudaMemcpyDeviceToDevice, st));
      if (nz) {
        SPOPS_CUDA(cudaMemcpyAsync(C->col.p, S->col.p, (size_t)nz * sizeof(I), cudaMemcpyDeviceToDevice, st));
        SPOPS_CUDA(cudaMemcpyAsync(C->val.p, S->val.p, (size_t)nz * sizeof(V), cudaMemcpyDeviceToDevice, st));
      }
      SPOPS_CUDA(cudaStreamSynchronize(st));
    }
    if (s != SPOPS_OK) {
      C->release_all();
      delete C;
      return s;
    }
    *out = C;
    return SPOPS_OK;
  }
  if (n > (int64_t)0xffffffffLL || S->cols > (int64_t)0xffffffffLL)
    return fail(SPOPS_ERR_UNSUPPORTED, "coo_to_csr (compact): more than 2^32 rows or columns");
  const size_t m1 = (size_t)std::max<int64_t>(nz, 1);
  DevBuf key, skey, pos, spos, flag, gid, start, gsum, okey, sokey, gidx, sgidx, cnt, scan, tmp;
  SPOPS_TRY(key.alloc(m1 * 8));
  SPOPS_TRY(skey.alloc(m1 * 8));
  SPOPS_TRY(pos.alloc(m1 * 8));
  SPOPS_TRY(spos.alloc(m1 * 8));
  SPOPS_TRY(flag.alloc(m1 * 8));
  SPOPS_TRY(gid.alloc(m1 * 8));
  SPOPS_TRY(cnt.alloc((n1 + 1) * 8));
  SPOPS_TRY(scan.alloc((n1 + 1) * 8));
  SPOPS_CUDA(cudaMemsetAsync(cnt.p, 0, (n1 + 1) * 8, st));  // per-row counts, then the kept total at [n + 1]
  int64_t ngroups = 0, kept = 0;
  if (nz > 0) {
    entry_key_kernel<I><<<grid_of(n * 32), 256, 0, st>>>(S->row.as<I>(), n, S->col.as<I>(), key.as<uint64_t>(),
                                                         pos.as<int64_t>());
    SPOPS_LAUNCH_CHECK();
    size_t c1 = 0, c2 = 0;
    SPOPS_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, c1, key.as<uint64_t>(), skey.as<uint64_t>(), pos.as<int64_t>(),
                                               spos.as<int64_t>(), nz, 0, 64, st));
    SPOPS_CUDA(cub::DeviceScan::InclusiveSum(nullptr, c2, flag.as<int64_t>(), gid.as<int64_t>(), nz, st));
    SPOPS_TRY(tmp.alloc(std::max(c1, c2) + 256));
    SPOPS_CUDA(cub::DeviceRadixSort::SortPairs(tmp.p, c1, key.as<uint64_t>(), skey.as<uint64_t>(), pos.as<int64_t>(),
                                               spos.as<int64_t>(), nz, 0, 64, st));
    group_flag_kernel<<<grid_of(nz), 256, 0, st>>>(skey.as<uint64_t>(), nz, flag.as<int64_t>());
    SPOPS_LAUNCH_CHECK();
    SPOPS_CUDA(cub::DeviceScan::InclusiveSum(tmp.p, c2, flag.as<int64_t>(), gid.as<int64_t>(), nz, st));
    SPOPS_CUDA(cudaMemcpyAsync(&ngroups, gid.as<int64_t>() + nz - 1, 8, cudaMemcpyDeviceToHost, st));
    SPOPS_CUDA(cudaStreamSynchronize(st));
    SPOPS_TRY(start.alloc(((size_t)ngroups + 1) * 8));
    SPOPS_TRY(gsum.alloc((size_t)ngroups * sizeof(V)));
    SPOPS_TRY(okey.alloc((size_t)ngroups * 8));
    SPOPS_TRY(sokey.alloc((size_t)ngroups * 8));
    SPOPS_TRY(gidx.alloc((size_t)ngroups * 8));
    SPOPS_TRY(sgidx.alloc((size_t)ngroups * 8));
    group_start_kernel<<<grid_of(nz), 256, 0, st>>>(flag.as<int64_t>(), gid.as<int64_t>(), nz, start.as<int64_t>());
    unsigned long long* kept_d = cnt.as<unsigned long long>() + n1;
    group_sum_kernel<I, V><<<grid_of(ngroups), 256, 0, st>>>(
        skey.as<uint64_t>(), spos.as<int64_t>(), start.as<int64_t>(), ngroups, S->row.as<I>(), S->val.as<V>(),
        gsum.as<V>(), okey.as<uint64_t>(), gidx.as<int64_t>(), kept_d, cnt.as<unsigned long long>());
    SPOPS_LAUNCH_CHECK();
    unsigned long long hk = 0;
    SPOPS_CUDA(cudaMemcpyAsync(&hk, kept_d, 8, cudaMemcpyDeviceToHost, st));
    SPOPS_CUDA(cudaStreamSynchronize(st));
    kept = (int64_t)hk;
    if (kept > 0) {
      size_t c3 = 0;
      SPOPS_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, c3, okey.as<uint64_t>(), sokey.as<uint64_t>(),
                                                 gidx.as<int64_t>(), sgidx.as<int64_t>(), kept, 0, 64, st));
      if (c3 + 256 > tmp.bytes) SPOPS_TRY(tmp.alloc(c3 + 256));
      SPOPS_CUDA(cub::DeviceRadixSort::SortPairs(tmp.p, c3, okey.as<uint64_t>(), sokey.as<uint64_t>(),
                                                 gidx.as<int64_t>(), sgidx.as<int64_t>(), kept, 0, 64, st));
    }
  }
  Matrix* C = new_csr(ctx, S, kept);
  spops_status_t s = C->row.alloc(n1 * sizeof(I));
  if (s == SPOPS_OK) s = C->col.alloc((size_t)std::max<int64_t>(kept, 1) * sizeof(I));
  if (s == SPOPS_OK) s = C->val.alloc((size_t)std::max<int64_t>(kept, 1) * sizeof(V));
  if (s == SPOPS_OK) {
    size_t c4 = 0;
    SPOPS_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, c4, cnt.as<unsigned long long>(),
                                             scan.as<unsigned long long>(), (int64_t)n1, st));
    if (c4 + 256 > tmp.bytes) SPOPS_TRY(tmp.alloc(c4 + 256));
    SPOPS_CUDA(cub::DeviceScan::ExclusiveSum(tmp.p, c4, cnt.as<unsigned long long>(), scan.as<unsigned long long>(),
                                             (int64_t)n1, st));
    offsets_kernel<I><<<grid_of((int64_t)n1), 256, 0, st>>>(scan.as<unsigned long long>(), (int64_t)n1, C->row.as<I>());
    if (kept > 0)
      compact_write_kernel<I, V><<<grid_of(kept), 256, 0, st>>>(skey.as<uint64_t>(), start.as<int64_t>(),
                                                                sgidx.as<int64_t>(), gsum.as<V>(), kept,
                                                                C->col.as<I>(), C->val.as<V>());
    SPOPS_LAUNCH_CHECK();
    SPOPS_CUDA(cudaStreamSynchronize(st));
  }
  if (s != SPOPS_OK) {
    C->release_all();
    delete C;
    return s;
  }
  *out = C;
  return SPOPS_OK;
}

// ---- csr_reorder_rows (include/sparse_conversion.h:1879-1998): row i of the
// result is row perm[i] of the input.
template <typename I>
__global__ void reorder_len_kernel(const I* __restrict__ rp, const I* __restrict__ perm, int64_t n,
                                   unsigned long long* __restrict__ len, unsigned int* __restrict__ seen,
                                   int* __restrict__ bad) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int64_t p = (int64_t)perm[i];
  if (p < 0 || p >= n) {
    atomicExch(bad, 1);
    len[i] = 0;
    return;
  }
  atomicAdd(seen + p, 1u);
  len[i] = (unsigned long long)((int64_t)rp[p + 1] - (int64_t)rp[p]);
}

__global__ void perm_check_kernel(const unsigned int* __restrict__ seen, int64_t n, int* __restrict__ bad) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i < n && seen[i] != 1u) atomicExch(bad, 1);
}

// one warp per result row
template <typename I, typename V>
__global__ void reorder_copy_kernel(const I* __restrict__ rp, const I* __restrict__ ci, const V* __restrict__ val,
                                    const I* __restrict__ perm, const unsigned long long* __restrict__ off, int64_t n,
                                    I* __restrict__ nci, V* __restrict__ nval) {
  const int64_t r = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (r >= n) return;
  const int64_t p = (int64_t)perm[r];
  const int64_t s = (int64_t)rp[p], m = (int64_t)rp[p + 1] - s, o = (int64_t)off[r];
  for (int64_t k = lane; k < m; k += 32) {
    nci[o + k] = ci[s + k];
    nval[o + k] = val[s + k];
  }
}

template <typename I, typename V>
spops_status_t reorder_t(Context* ctx, Matrix* A, const void* perm_host, Matrix** out) {
  cudaStream_t st = ctx->stream;
  const int64_t n = A->rows, nz = A->nnz;
  PoolBuf perm(ctx), len(ctx), seen(ctx), flag(ctx), scan(ctx), tmp(ctx);
  SPOPS_TRY(perm.alloc((size_t)std::max<int64_t>(n, 1) * sizeof(I)));
  SPOPS_TRY(len.alloc((size_t)(n + 1) * 8));
  SPOPS_TRY(scan.alloc((size_t)(n + 1) * 8));
  SPOPS_TRY(seen.alloc((size_t)std::max<int64_t>(n, 1) * 4));
  SPOPS_TRY(flag.alloc(16));
  if (n > 0) SPOPS_CUDA(cudaMemcpyAsync(perm.p, perm_host, (size_t)n * sizeof(I), cudaMemcpyHostToDevice, st));
  SPOPS_CUDA(cudaMemsetAsync(seen.p, 0, (size_t)std::max<int64_t>(n, 1) * 4, st));
  SPOPS_CUDA(cudaMemsetAsync(flag.p, 0, 16, st));
  SPOPS_CUDA(cudaMemsetAsync(len.as<unsigned long long>() + n, 0, 8, st));
  if (n > 0) {
    reorder_len_kernel<I><<<grid_of(n), 256, 0, st>>>(A->row.as<I>(), perm.as<I>(), n, len.as<unsigned long long>(),
                                                      seen.as<unsigned int>(), flag.as<int>());
    perm_check_kernel<<<grid_of(n), 256, 0, st>>>(seen.as<unsigned int>(), n, flag.as<int>());
    SPOPS_LAUNCH_CHECK();
  }
  int bad = 0;
  SPOPS_CUDA(cudaMemcpyAsync(&bad, flag.p, 4, cudaMemcpyDeviceToHost, st));
  SPOPS_CUDA(cudaStreamSynchronize(st));
  if (bad) return fail(SPOPS_ERR_INVALID, "csr_reorder_rows: the row permutation is not a permutation of 0..%lld",
                       (long long)(n - 1));
  size_t tb = 0;
  SPOPS_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tb, len.as<unsigned long long>(), scan.as<unsigned long long>(),
                                           n + 1, st));
  SPOPS_TRY(tmp.alloc(tb + 256));
  SPOPS_CUDA(cub::DeviceScan::ExclusiveSum(tmp.p, tb, len.as<unsigned long long>(), scan.as<unsigned long long>(),
                                           n + 1, st));
  Matrix* C = new_csr(ctx, A, nz);
  spops_status_t s = C->row.alloc((size_t)(n + 1) * sizeof(I));
  if (s == SPOPS_OK) s = C->col.alloc((size_t)std::max<int64_t>(nz, 1) * sizeof(I));
  if (s == SPOPS_OK) s = C->val.alloc((size_t)std::max<int64_t>(nz, 1) * sizeof(V));
  if (s == SPOPS_OK) {
    offsets_kernel<I><<<grid_of(n + 1), 256, 0, st>>>(scan.as<unsigned long long>(), n + 1, C->row.as<I>());
    if (n > 0)
      reorder_copy_kernel<I, V><<<grid_of(n * 32), 256, 0, st>>>(A->row.as<I>(), A->col.as<I>(), A->val.as<V>(),
                                                                 perm.as<I>(), scan.as<unsigned long long>(), n,
                                                                 C->col.as<I>(), C->val.as<V>());
    if (cudaGetLastError() != cudaSuccess || cudaStreamSynchronize(st) != cudaSuccess)
      s = fail(SPOPS_ERR_CUDA, "csr_reorder_rows: launch failed");
  }
  if (s != SPOPS_OK) {
    C->release_all();
    delete C;
    return s;
  }
  *out = C;
  return SPOPS_OK;
}

}  // namespace
}  // namespace spops

using namespace spops;

extern "C" spops_status_t spops_coo_to_csr(spops_context_t ctx, spops_matrix_t coo, int32_t compact,
                                           spops_matrix_t* csr) {
  if (!ctx || !coo || !csr) return fail(SPOPS_ERR_INVALID, "spops_coo_to_csr: null argument");
  if (coo->format != SPOPS_FMT_COO) return fail(SPOPS_ERR_INVALID, "spops_coo_to_csr: not a COO matrix");
  DeviceGuard g(ctx->device);
  Matrix* out = nullptr;
  const bool c = compact != 0;
  spops_status_t s;
  if (coo->itype == SPOPS_INDEX_I32)
    s = coo->vtype == SPOPS_VALUE_F64 ? coo_to_csr_t<int32_t, double>(ctx, coo, c, &out)
                                      : coo_to_csr_t<int32_t, float>(ctx, coo, c, &out);
  else
    s = coo->vtype == SPOPS_VALUE_F64 ? coo_to_csr_t<int64_t, double>(ctx, coo, c, &out)
                                      : coo_to_csr_t<int64_t, float>(ctx, coo, c, &out);
  if (s != SPOPS_OK) return s;
  *csr = static_cast<spops_matrix_s*>(out);
  return SPOPS_OK;
}

extern "C" spops_status_t spops_csr_reorder_rows(spops_context_t ctx, spops_matrix_t csr, const void* perm,
                                                 spops_matrix_t* out) {
  if (!ctx || !csr || !out || (!perm && csr->rows > 0))
    return fail(SPOPS_ERR_INVALID, "spops_csr_reorder_rows: null argument");
  if (csr->format != SPOPS_FMT_CSR) return fail(SPOPS_ERR_INVALID, "spops_csr_reorder_rows: needs a CSR matrix");
  DeviceGuard g(ctx->device);
  if (!csr->plan.ready) SPOPS_TRY(csr_analyse(ctx, csr));  // validates the pattern
  Matrix* C = nullptr;
  spops_status_t s;
  if (csr->itype == SPOPS_INDEX_I32)
    s = csr->vtype == SPOPS_VALUE_F64 ? reorder_t<int32_t, double>(ctx, csr, perm, &C)
                                      : reorder_t<int32_t, float>(ctx, csr, perm, &C);
  else
    s = csr->vtype == SPOPS_VALUE_F64 ? reorder_t<int64_t, double>(ctx, csr, perm, &C)
                                      : reorder_t<int64_t, float>(ctx, csr, perm, &C);
  if (s != SPOPS_OK) return s;
  *out = static_cast<spops_matrix_s*>(C);
  return SPOPS_OK;
}

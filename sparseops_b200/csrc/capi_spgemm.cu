// C ABI of the LeSpGEMM path: MinHash signatures, LSH candidate pairs,
// hierarchical clustering and the cluster-wise SpGEMM.
#include <chrono>
#include <cstring>
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "spops_internal.h"

using namespace spops;

struct spops_pairs_s : spops::PairSet {
  spops::Context* ctx = nullptr;
};

namespace {

// The CSR pattern of A as int64 host arrays (for the host clustering), copied
// once per handle and kept on it: a handle's pattern never changes
// (spops_csr_set_values replaces values only).
spops_status_t host_pattern(Context* ctx, Matrix* A, const std::vector<int64_t>** rp_out,
                            const std::vector<int64_t>** ci_out) {
  *rp_out = &A->host_rp;
  *ci_out = &A->host_ci;
  if (A->host_rp.size() == (size_t)A->rows + 1) return SPOPS_OK;
  std::vector<int64_t> rp((size_t)A->rows + 1), ci((size_t)A->nnz);
  cudaStream_t st = ctx->stream;
  if (A->itype == SPOPS_INDEX_I64) {
    SPOPS_CUDA(cudaMemcpyAsync(rp.data(), A->row.p, rp.size() * 8, cudaMemcpyDeviceToHost, st));
    if (A->nnz) SPOPS_CUDA(cudaMemcpyAsync(ci.data(), A->col.p, ci.size() * 8, cudaMemcpyDeviceToHost, st));
    SPOPS_CUDA(cudaStreamSynchronize(st));
  } else {
    std::vector<int32_t> r32(rp.size()), c32(ci.size());
    SPOPS_CUDA(cudaMemcpyAsync(r32.data(), A->row.p, r32.size() * 4, cudaMemcpyDeviceToHost, st));
    if (A->nnz) SPOPS_CUDA(cudaMemcpyAsync(c32.data(), A->col.p, c32.size() * 4, cudaMemcpyDeviceToHost, st));
    SPOPS_CUDA(cudaStreamSynchronize(st));
    std::copy(r32.begin(), r32.end(), rp.begin());
    std::copy(c32.begin(), c32.end(), ci.begin());
  }
  A->host_rp.swap(rp);
  A->host_ci.swap(ci);
  return SPOPS_OK;
}

void put_stats(const SpgemmStats& s, spops_spgemm_stats_t* o) {
  if (!o) return;
  o->flops = s.flops;
  o->clusters = s.clusters;
  o->dense_clusters = s.dense_clusters;
  o->pairs = s.pairs;
  o->cluster_columns = s.cluster_columns;
  o->c_cluster_columns = s.c_cluster_columns;
  o->minhash_ms = s.minhash_ms;
  o->lsh_ms = s.lsh_ms;
  o->hc_ms = s.hc_ms;
  o->cluster_ms = s.cluster_ms;
  o->symbolic_ms = s.symbolic_ms;
  o->numeric_ms = s.numeric_ms;
  o->to_csr_ms = s.to_csr_ms;
}

double ms_since(std::chrono::steady_clock::time_point t0) {
  return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
}

}  // namespace

extern "C" {

spops_status_t spops_minhash(spops_context_t ctx, spops_matrix_t A, int32_t k, uint64_t seed, void* sig) {
  if (!ctx || !A || (!sig && A->rows > 0)) return fail(SPOPS_ERR_INVALID, "spops_minhash: null argument");
  DeviceGuard g(ctx->device);
  return minhash_signatures(ctx, A, k, seed, static_cast<uint64_t*>(sig));
}

spops_status_t spops_minhash_host(spops_context_t ctx, spops_matrix_t A, int32_t k, uint64_t seed, void* sig_host) {
  if (!ctx || !A || (!sig_host && A->rows > 0)) return fail(SPOPS_ERR_INVALID, "spops_minhash_host: null argument");
  if (k <= 0) return fail(SPOPS_ERR_INVALID, "spops_minhash_host: k must be positive");
  DeviceGuard g(ctx->device);
  const size_t bytes = (size_t)std::max<int64_t>(A->rows, 1) * (size_t)k * 8;
  DevBuf sig;
  SPOPS_TRY(sig.alloc(bytes));
  spops_status_t s = minhash_signatures(ctx, A, k, seed, sig.as<uint64_t>());
  if (s == SPOPS_OK && A->rows > 0) {
    const cudaError_t e = cudaMemcpyAsync(sig_host, sig.p, (size_t)A->rows * (size_t)k * 8, cudaMemcpyDeviceToHost,
                                          ctx->stream);
    const cudaError_t e2 = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess || e2 != cudaSuccess)
      s = fail(SPOPS_ERR_CUDA, "spops_minhash_host: %s", cudaGetErrorString(e != cudaSuccess ? e : e2));
  }
  sig.release();
  return s;
}

spops_status_t spops_lsh_pairs_from_signatures(spops_context_t ctx, const void* sig, int64_t rows, int32_t k,
                                               int32_t bands, int32_t constrain, spops_pairs_t* out) {
  if (!ctx || !out || (!sig && rows > 0)) return fail(SPOPS_ERR_INVALID, "spops_lsh_pairs_from_signatures: null");
  DeviceGuard g(ctx->device);
  spops_pairs_s* P = new spops_pairs_s();
  P->ctx = ctx;
  spops_status_t s = lsh_pairs(ctx, static_cast<const uint64_t*>(sig), rows, k, bands, constrain != 0, P);
  if (s != SPOPS_OK) {
    P->release();
    delete P;
    return s;
  }
  *out = P;
  return SPOPS_OK;
}

spops_status_t spops_lsh_pairs(spops_context_t ctx, spops_matrix_t A, int32_t k, int32_t bands, uint64_t seed,
                               int32_t constrain, spops_pairs_t* out) {
  if (!ctx || !A || !out) return fail(SPOPS_ERR_INVALID, "spops_lsh_pairs: null argument");
  if (k <= 0) return fail(SPOPS_ERR_INVALID, "spops_lsh_pairs: k must be positive");
  DeviceGuard g(ctx->device);
  DevBuf sig;
  SPOPS_TRY(sig.alloc((size_t)std::max<int64_t>(A->rows, 1) * k * 8));
  spops_status_t s = minhash_signatures(ctx, A, k, seed, sig.as<uint64_t>());
  if (s == SPOPS_OK) s = spops_lsh_pairs_from_signatures(ctx, sig.p, A->rows, k, bands, constrain, out);
  SPOPS_CUDA(cudaStreamSynchronize(ctx->stream));
  sig.release();
  return s;
}

spops_status_t spops_pairs_create(spops_context_t ctx, const int64_t* i, const int64_t* j, const double* score,
                                  int64_t count, spops_mem_t mem, spops_pairs_t* pairs) {
  if (!ctx || !pairs || count < 0 || (count > 0 && (!i || !j || !score)))
    return fail(SPOPS_ERR_INVALID, "spops_pairs_create: null or negative argument");
  DeviceGuard g(ctx->device);
  spops_pairs_s* P = new spops_pairs_s();
  P->ctx = ctx;
  P->count = count;
  const size_t n = (size_t)std::max<int64_t>(count, 1);
  spops_status_t s = P->pi.alloc(n * 8);
  if (s == SPOPS_OK) s = P->pj.alloc(n * 8);
  if (s == SPOPS_OK) s = P->score.alloc(n * 8);
  const cudaMemcpyKind kind = mem == SPOPS_MEM_HOST ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice;
  if (s == SPOPS_OK && count > 0 &&
      (cudaMemcpyAsync(P->pi.p, i, (size_t)count * 8, kind, ctx->stream) != cudaSuccess ||
       cudaMemcpyAsync(P->pj.p, j, (size_t)count * 8, kind, ctx->stream) != cudaSuccess ||
       cudaMemcpyAsync(P->score.p, score, (size_t)count * 8, kind, ctx->stream) != cudaSuccess ||
       cudaStreamSynchronize(ctx->stream) != cudaSuccess))
    s = fail(SPOPS_ERR_CUDA, "spops_pairs_create: copy failed: %s", cudaGetErrorString(cudaGetLastError()));
  if (s != SPOPS_OK) {
    P->release();
    delete P;
    return s;
  }
  *pairs = P;
  return SPOPS_OK;
}

spops_status_t spops_pairs_count(spops_pairs_t P, int64_t* count) {
  if (!P || !count) return fail(SPOPS_ERR_INVALID, "spops_pairs_count: null argument");
  *count = P->count;
  return SPOPS_OK;
}

spops_status_t spops_pairs_arrays(spops_pairs_t P, const int64_t** i, const int64_t** j, const double** score) {
  if (!P) return fail(SPOPS_ERR_INVALID, "spops_pairs_arrays: null pairs");
  if (i) *i = P->pi.as<int64_t>();
  if (j) *j = P->pj.as<int64_t>();
  if (score) *score = P->score.as<double>();
  return SPOPS_OK;
}

spops_status_t spops_pairs_download(spops_pairs_t P, int64_t* i, int64_t* j, double* score) {
  if (!P) return fail(SPOPS_ERR_INVALID, "spops_pairs_download: null pairs");
  if (P->count == 0) return SPOPS_OK;
  DeviceGuard g(P->ctx->device);
  cudaStream_t st = P->ctx->stream;
  const size_t b = (size_t)P->count * 8;
  if (i) SPOPS_CUDA(cudaMemcpyAsync(i, P->pi.p, b, cudaMemcpyDeviceToHost, st));
  if (j) SPOPS_CUDA(cudaMemcpyAsync(j, P->pj.p, b, cudaMemcpyDeviceToHost, st));
  if (score) SPOPS_CUDA(cudaMemcpyAsync(score, P->score.p, b, cudaMemcpyDeviceToHost, st));
  SPOPS_CUDA(cudaStreamSynchronize(st));
  return SPOPS_OK;
}

spops_status_t spops_pairs_destroy(spops_pairs_t P) {
  if (!P) return SPOPS_OK;
  DeviceGuard g(P->ctx->device);
  cudaStreamSynchronize(P->ctx->stream);
  P->release();
  delete P;
  return SPOPS_OK;
}

spops_status_t spops_hierarchical_clustering(const int64_t* row_ptr, const int64_t* col_index, int64_t rows,
                                             const int64_t* pi, const int64_t* pj, const double* score,
                                             int64_t npairs, int64_t cluster_size, int64_t* permutation,
                                             int64_t* offsets, int64_t* nclusters) {
  if (rows < 0 || npairs < 0 || (rows > 0 && (!row_ptr || !permutation || !offsets)) ||
      (npairs > 0 && (!pi || !pj || !score)) || !nclusters)
    return fail(SPOPS_ERR_INVALID, "spops_hierarchical_clustering: null argument");
  std::vector<int64_t> perm, offs;
  SPOPS_TRY(hierarchical_clustering(row_ptr, col_index, rows, pi, pj, score, npairs, cluster_size, perm, offs));
  std::memcpy(permutation, perm.data(), perm.size() * 8);
  std::memcpy(offsets, offs.data(), offs.size() * 8);
  *nclusters = (int64_t)offs.size() - 1;
  return SPOPS_OK;
}

spops_status_t spops_pairs_cluster(spops_context_t ctx, spops_matrix_t A, spops_pairs_t pairs, int64_t cluster_size,
                                   int64_t* permutation, int64_t* offsets, int64_t* nclusters) {
  if (!ctx || !A || !pairs || !nclusters || (A->rows > 0 && (!permutation || !offsets)))
    return fail(SPOPS_ERR_INVALID, "spops_pairs_cluster: null argument");
  if (A->format != SPOPS_FMT_CSR) return fail(SPOPS_ERR_INVALID, "spops_pairs_cluster: A must be a CSR matrix");
  DeviceGuard g(ctx->device);
  const PairSet& P = *pairs;
  ArenaScope scope(ctx);  // this call's temporaries come from the arena
  PoolBuf perm(ctx), offs(ctx);
  SPOPS_TRY(perm.alloc((size_t)std::max<int64_t>(A->rows, 1) * 8));
  SPOPS_TRY(offs.alloc(((size_t)A->rows + 1) * 8));
  int64_t ncl = 0;
  SPOPS_TRY(hierarchical_clustering_device(ctx, A, P.pi.as<int64_t>(), P.pj.as<int64_t>(), P.score.as<double>(),
                                           P.count, cluster_size, perm.as<int64_t>(), offs.as<int64_t>(), &ncl,
                                           nullptr));
  if (A->rows > 0)
    SPOPS_CUDA(cudaMemcpyAsync(permutation, perm.p, (size_t)A->rows * 8, cudaMemcpyDeviceToHost, ctx->stream));
  if (offsets) SPOPS_CUDA(cudaMemcpyAsync(offsets, offs.p, ((size_t)ncl + 1) * 8, cudaMemcpyDeviceToHost, ctx->stream));
  SPOPS_CUDA(cudaStreamSynchronize(ctx->stream));
  *nclusters = ncl;
  return SPOPS_OK;
}

spops_status_t spops_spgemm_clustered(spops_context_t ctx, spops_matrix_t A, spops_matrix_t B,
                                      const int64_t* permutation, const int64_t* offsets, int64_t nclusters,
                                      int32_t sort_output, double l2_budget_bytes, spops_matrix_t* C,
                                      spops_spgemm_stats_t* stats) {
  if (!ctx || !A || !B || !C || !offsets || (A->rows > 0 && !permutation))
    return fail(SPOPS_ERR_INVALID, "spops_spgemm_clustered: null argument");
  DeviceGuard g(ctx->device);
  SpgemmStats s;
  Matrix* out = nullptr;
  SPOPS_TRY(cluster_spgemm(ctx, A, B, permutation, offsets, nclusters, sort_output != 0, l2_budget_bytes, &out, &s));
  *C = static_cast<spops_matrix_s*>(out);
  put_stats(s, stats);
  return SPOPS_OK;
}

spops_status_t spops_spgemm_rowwise(spops_context_t ctx, spops_matrix_t A, spops_matrix_t B, int32_t kernel_flag,
                                    int32_t sort_output, spops_matrix_t* C, spops_spgemm_stats_t* stats) {
  if (!ctx || !A || !B || !C) return fail(SPOPS_ERR_INVALID, "spops_spgemm_rowwise: null argument");
  (void)kernel_flag;  // kernels 1-3 give the same entries; columns always ascending here
  DeviceGuard g(ctx->device);
  SpgemmStats s;
  Matrix* out = nullptr;
  SPOPS_TRY(rowwise_spgemm(ctx, A, B, sort_output != 0, &out, &s));
  *C = static_cast<spops_matrix_s*>(out);
  put_stats(s, stats);
  return SPOPS_OK;
}

spops_status_t spops_spgemm_topk(spops_context_t ctx, spops_matrix_t A, int64_t top_k, spops_matrix_t* C) {
  if (!ctx || !A || !C) return fail(SPOPS_ERR_INVALID, "spops_spgemm_topk: null argument");
  DeviceGuard g(ctx->device);
  Matrix* out = nullptr;
  SPOPS_TRY(topk_spgemm(ctx, A, top_k, &out));
  *C = static_cast<spops_matrix_s*>(out);
  return SPOPS_OK;
}

spops_status_t spops_spgemm_lsh(spops_context_t ctx, spops_matrix_t A, spops_matrix_t B, int32_t k, int32_t bands,
                                uint64_t seed, int64_t cluster_size, int32_t sort_output, double l2_budget_bytes,
                                spops_matrix_t* C, spops_spgemm_stats_t* stats) {
  if (!ctx || !A || !B || !C) return fail(SPOPS_ERR_INVALID, "spops_spgemm_lsh: null argument");
  DeviceGuard g(ctx->device);
  SpgemmStats s;
  auto t0 = std::chrono::steady_clock::now();
  ArenaScope scope(ctx);  // this call's temporaries come from the arena
  PoolBuf sig(ctx);
  SPOPS_TRY(sig.alloc((size_t)std::max<int64_t>(A->rows, 1) * (size_t)std::max(k, 1) * 8));
  spops_status_t st = minhash_signatures(ctx, A, k, seed, sig.as<uint64_t>());
  if (st != SPOPS_OK) {
    sig.release();
    return st;
  }
  cudaStreamSynchronize(ctx->stream);
  s.minhash_ms = ms_since(t0);
  t0 = std::chrono::steady_clock::now();
  PairSet P;
  st = lsh_pairs(ctx, sig.as<uint64_t>(), A->rows, k, bands, true, &P);
  cudaStreamSynchronize(ctx->stream);
  sig.release();
  if (st != SPOPS_OK) return st;
  s.lsh_ms = ms_since(t0);
  s.pairs = P.count;
  t0 = std::chrono::steady_clock::now();
  // clustering on the device; permutation and offsets stay there
  PoolBuf perm(ctx), offs(ctx);
  SPOPS_TRY(perm.alloc((size_t)std::max<int64_t>(A->rows, 1) * 8));
  SPOPS_TRY(offs.alloc(((size_t)A->rows + 1) * 8));
  int64_t ncl = 0;
  st = hierarchical_clustering_device(ctx, A, P.pi.as<int64_t>(), P.pj.as<int64_t>(), P.score.as<double>(), P.count,
                                      cluster_size, perm.as<int64_t>(), offs.as<int64_t>(), &ncl, nullptr);
  P.release();
  if (st != SPOPS_OK) return st;
  s.hc_ms = ms_since(t0);
  Matrix* out = nullptr;
  SpgemmStats s2;
  SPOPS_TRY(cluster_spgemm(ctx, A, B, perm.as<int64_t>(), offs.as<int64_t>(), ncl, sort_output != 0, l2_budget_bytes,
                           &out, &s2, false, false, true));
  s2.minhash_ms = s.minhash_ms;
  s2.lsh_ms = s.lsh_ms;
  s2.hc_ms = s.hc_ms;
  s2.pairs = s.pairs;
  *C = static_cast<spops_matrix_s*>(out);
  put_stats(s2, stats);
  return SPOPS_OK;
}

// ------------------------------------------------ clustered (VLength) form
spops_status_t spops_vlcluster_create(spops_context_t ctx, spops_matrix_t* M, int64_t csr_rows, int64_t clusters,
                                      int64_t cols, int64_t nnzc, int64_t nnzv, const void* cluster_sz,
                                      const void* rowptr, const void* colids, const void* rowptr_val,
                                      const void* values, spops_index_t itype, spops_value_t vtype, spops_mem_t mem) {
  if (!ctx || !M || clusters < 0 || csr_rows < 0 || cols < 0 || nnzc < 0 || nnzv < 0 ||
      (clusters > 0 && (!cluster_sz || !rowptr || !rowptr_val)) || (nnzc > 0 && !colids) || (nnzv > 0 && !values))
    return fail(SPOPS_ERR_INVALID, "spops_vlcluster_create: null or negative argument");
  if ((itype != SPOPS_INDEX_I32 && itype != SPOPS_INDEX_I64) || (vtype != SPOPS_VALUE_F32 && vtype != SPOPS_VALUE_F64))
    return fail(SPOPS_ERR_INVALID, "spops_vlcluster_create: bad index or value type");
  DeviceGuard g(ctx->device);
  cudaStream_t st = ctx->stream;
  const size_t is = itype == SPOPS_INDEX_I32 ? 4 : 8, vs = vtype == SPOPS_VALUE_F32 ? 4 : 8;
  const cudaMemcpyKind kind = mem == SPOPS_MEM_HOST ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice;
  const cudaMemcpyKind back = mem == SPOPS_MEM_HOST ? cudaMemcpyHostToHost : cudaMemcpyDeviceToHost;
  // the small per-cluster arrays on the host for the checks
  std::vector<int64_t> sz((size_t)clusters), rp((size_t)clusters + 1), rpv((size_t)clusters + 1);
  {
    std::vector<char> a((size_t)clusters * is), b(((size_t)clusters + 1) * is), c(((size_t)clusters + 1) * is);
    if (clusters > 0) {
      SPOPS_CUDA(cudaMemcpy(a.data(), cluster_sz, a.size(), back));
      SPOPS_CUDA(cudaMemcpy(b.data(), rowptr, b.size(), back));
      SPOPS_CUDA(cudaMemcpy(c.data(), rowptr_val, c.size(), back));
    }
    auto get = [&](const std::vector<char>& v, size_t i) -> int64_t {
      return is == 4 ? (int64_t)reinterpret_cast<const int32_t*>(v.data())[i] : reinterpret_cast<const int64_t*>(v.data())[i];
    };
    for (int64_t i = 0; i < clusters; ++i) sz[(size_t)i] = get(a, (size_t)i);
    for (int64_t i = 0; clusters > 0 && i <= clusters; ++i) {
      rp[(size_t)i] = get(b, (size_t)i);
      rpv[(size_t)i] = get(c, (size_t)i);
    }
  }
  std::vector<int64_t> off((size_t)clusters + 1, 0);
  for (int64_t i = 0; i < clusters; ++i) {
    if (sz[(size_t)i] < 0) return fail(SPOPS_ERR_INVALID, "spops_vlcluster_create: negative cluster size");
    off[(size_t)i + 1] = off[(size_t)i] + sz[(size_t)i];
  }
  if (off[(size_t)clusters] != csr_rows)
    return fail(SPOPS_ERR_INVALID, "spops_vlcluster_create: cluster sizes add up to %lld, not %lld rows",
                (long long)off[(size_t)clusters], (long long)csr_rows);
  if (clusters > 0) {
    if (rp[0] != 0 || rpv[0] != 0 || rp[(size_t)clusters] != nnzc || rpv[(size_t)clusters] != nnzv)
      return fail(SPOPS_ERR_INVALID, "spops_vlcluster_create: rowptr / rowptr_val do not span nnzc / nnzv");
    for (int64_t i = 0; i < clusters; ++i)
      if (rp[(size_t)i + 1] < rp[(size_t)i] ||
          rpv[(size_t)i + 1] - rpv[(size_t)i] != (rp[(size_t)i + 1] - rp[(size_t)i]) * sz[(size_t)i])
        return fail(SPOPS_ERR_INVALID, "spops_vlcluster_create: cluster %lld: rowptr_val does not match", (long long)i);
  } else if (nnzc || nnzv || csr_rows) {
    return fail(SPOPS_ERR_INVALID, "spops_vlcluster_create: entries without clusters");
  }
  Matrix* A = new spops_matrix_s();
  A->ctx = ctx;
  A->format = SPOPS_FMT_VLCLUSTER;
  A->itype = itype;
  A->vtype = vtype;
  A->rows = csr_rows;
  A->cols = cols;
  A->nnz = nnzc;
  A->clusters = clusters;
  A->cl_nnzv = nnzv;
  spops_status_t s = A->row.alloc(((size_t)clusters + 1) * is);
  if (s == SPOPS_OK) s = A->cl_rpv.alloc(((size_t)clusters + 1) * is);
  if (s == SPOPS_OK) s = A->col.alloc((size_t)std::max<int64_t>(nnzc, 1) * is);
  if (s == SPOPS_OK) s = A->val.alloc((size_t)std::max<int64_t>(nnzv, 1) * vs);
  if (s == SPOPS_OK && clusters > 0) {
    if (cudaMemcpyAsync(A->row.p, rowptr, ((size_t)clusters + 1) * is, kind, st) != cudaSuccess ||
        cudaMemcpyAsync(A->cl_rpv.p, rowptr_val, ((size_t)clusters + 1) * is, kind, st) != cudaSuccess ||
        (nnzc > 0 && cudaMemcpyAsync(A->col.p, colids, (size_t)nnzc * is, kind, st) != cudaSuccess) ||
        (nnzv > 0 && cudaMemcpyAsync(A->val.p, values, (size_t)nnzv * vs, kind, st) != cudaSuccess))
      s = fail(SPOPS_ERR_CUDA, "spops_vlcluster_create: copy failed");
  }
  if (s == SPOPS_OK && nnzc > 0) s = validate_columns(ctx, A->col.p, nnzc, itype, cols, false);
  if (s == SPOPS_OK) s = vlcluster_finish(ctx, A, off.data());
  if (s != SPOPS_OK) {
    A->release_all();
    delete static_cast<spops_matrix_s*>(A);
    return s;
  }
  *M = static_cast<spops_matrix_s*>(A);
  return SPOPS_OK;
}

spops_status_t spops_csr_to_vlength_cluster(spops_context_t ctx, spops_matrix_t csr, const int64_t* offsets,
                                            int64_t clusters, spops_matrix_t* cluster) {
  if (!ctx || !csr || !offsets || !cluster) return fail(SPOPS_ERR_INVALID, "spops_csr_to_vlength_cluster: null argument");
  DeviceGuard g(ctx->device);
  Matrix* out = nullptr;
  SPOPS_TRY(vlcluster_from_csr(ctx, csr, offsets, clusters, &out));
  *cluster = static_cast<spops_matrix_s*>(out);
  return SPOPS_OK;
}

spops_status_t spops_vlength_cluster_to_csr(spops_context_t ctx, spops_matrix_t cluster, spops_matrix_t* csr) {
  if (!ctx || !cluster || !csr) return fail(SPOPS_ERR_INVALID, "spops_vlength_cluster_to_csr: null argument");
  DeviceGuard g(ctx->device);
  Matrix* out = nullptr;
  SPOPS_TRY(vlcluster_to_csr(ctx, cluster, &out));
  *csr = static_cast<spops_matrix_s*>(out);
  return SPOPS_OK;
}

spops_status_t spops_spgemm_vlength(spops_context_t ctx, spops_matrix_t A_cluster, spops_matrix_t B,
                                    int32_t sort_output, double l2_budget_bytes, spops_matrix_t* C_cluster,
                                    spops_spgemm_stats_t* stats) {
  if (!ctx || !A_cluster || !B || !C_cluster) return fail(SPOPS_ERR_INVALID, "spops_spgemm_vlength: null argument");
  if (A_cluster->format != SPOPS_FMT_VLCLUSTER)
    return fail(SPOPS_ERR_INVALID, "spops_spgemm_vlength: A must be a clustered matrix");
  DeviceGuard g(ctx->device);
  const int64_t ncl = A_cluster->clusters, n = A_cluster->rows;
  std::vector<int64_t> off((size_t)ncl + 1), perm((size_t)std::max<int64_t>(n, 1));
  SPOPS_CUDA(cudaMemcpy(off.data(), A_cluster->cl_off.p, ((size_t)ncl + 1) * 8, cudaMemcpyDeviceToHost));
  for (int64_t r = 0; r < n; ++r) perm[(size_t)r] = r;
  Matrix* A = nullptr;
  SPOPS_TRY(vlcluster_to_csr(ctx, A_cluster, &A));
  SpgemmStats s;
  Matrix* out = nullptr;
  spops_status_t rc =
      cluster_spgemm(ctx, A, B, perm.data(), off.data(), ncl, sort_output != 0, l2_budget_bytes, &out, &s, false, true);
  A->release_all();
  delete static_cast<spops_matrix_s*>(A);
  SPOPS_TRY(rc);
  *C_cluster = static_cast<spops_matrix_s*>(out);
  put_stats(s, stats);
  return SPOPS_OK;
}

}  // extern "C"
